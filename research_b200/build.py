"""Build recipe for the native libraries (no GPU needed; nvcc cross-compiles).

    python -m research_b200.build            # librr_cuda.so + the CPU checker
    python -m research_b200.build --ptxas-v  # also print register/spill reports

Outputs (git-ignored, shipped in-tree):
    research_b200/lib/librr_cuda.so   CUDA kernels + C ABI (include/rr_cuda.h)
    research_b200/lib/librr_passes.so the RenderPass adapters (only with the reference's headers)
    oracle/librr_oracle.so            CPU checker, built by oracle/Makefile
    oracle/librr_inputs.so            the seeded scene/camera generators without CUDA (CPU reference arm)
    oracle/_ref/librr_slangref.so     the reference's shader text rewritten to C++ (only with the reference checkout)

Numerics flags: the kernels are compiled without FMA contraction and with
IEEE-rounded division and square root (-fmad=false -prec-div=true
-prec-sqrt=true -ftz=false), host code with -ffp-contract=off, so device and
CPU evaluate the same binary32 operations in the same order.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "research_b200"
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
BUILD = ROOT / "_build"
LIB = LIBDIR / "librr_cuda.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-O2,-ffp-contract=off,-fno-fast-math",
    f"-I{ROOT / 'include'}", f"-I{CSRC}",
]
SOURCES = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
HEADERS = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))


def _nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found")
    return exe


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, quiet=False):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(map(str, cmd))}\n{r.stdout}\n{r.stderr}")
    if not quiet and (r.stderr.strip() or r.stdout.strip()):
        sys.stderr.write(r.stdout + r.stderr)
    return r


def build_cuda(force: bool = False, ptxas_v: bool = False, jobs: int | None = None) -> Path:
    """Compile every kernel source for sm_100a and link librr_cuda.so."""
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    nvcc = _nvcc()
    objs = []
    todo = []
    for src in SOURCES:
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if force or ptxas_v or _stale(obj, [src, *HEADERS]):
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
            if ptxas_v and src.suffix == ".cu":
                cmd += ["-Xptxas", "-v"]
            todo.append(cmd)
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            for r in ex.map(lambda c: _run(c, quiet=not ptxas_v), todo):
                if ptxas_v:
                    pass
    if force or todo or _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lpthread"])
    return LIB


REFERENCE = Path("/root/reference")
PASSES_LIB = LIBDIR / "librr_passes.so"
ADAPTERS = PKG / "adapters"


def build_passes(force: bool = False) -> Path | None:
    """The RenderPass adapters (adapters/rr_passes.*) for a host that keeps the
    reference's pass interface: compiled against that host's headers
    (src/render/RenderPass.h and what it includes), here the reference
    checkout's; skipped where it is absent. Links librr_cuda.so."""
    hdr = REFERENCE / "src" / "render" / "RenderPass.h"
    if not hdr.exists():
        return PASSES_LIB if PASSES_LIB.exists() else None
    src = ADAPTERS / "rr_passes.cpp"
    deps = [src, ADAPTERS / "rr_passes.h", LIB, ROOT / "include" / "rr_cuda.h", ROOT / "include" / "rr_layouts.h"]
    if force or _stale(PASSES_LIB, deps):
        cuda = Path(_nvcc()).resolve().parent.parent
        _run(["g++", "-O2", "-std=c++20", "-fPIC", "-Wall", "-shared", f"-I{REFERENCE / 'src'}",
              f"-I{ROOT / 'include'}", f"-I{cuda / 'include'}", "-o", str(PASSES_LIB), str(src),
              f"-L{LIBDIR}", "-lrr_cuda", f"-L{cuda / 'lib64'}", "-lcudart", "-Wl,-rpath,$ORIGIN",
              f"-Wl,-rpath,{cuda / 'lib64'}"])
    return PASSES_LIB


def build_oracle(force: bool = False) -> Path:
    """Build the CPU checker (test infrastructure) via oracle/Makefile: the
    hand-written restatement, the seeded-input library and, where the
    reference checkout is present, the reference's own shader text rewritten
    to C++ (oracle/_ref/librr_slangref.so)."""
    out = ROOT / "oracle" / "librr_oracle.so"
    if force and out.exists():
        out.unlink()
    _run(["make", "-s", "-C", str(ROOT / "oracle")], quiet=True)
    if (REFERENCE / "assets" / "shaders").is_dir():
        _run(["make", "-s", "-C", str(ROOT / "oracle"), "ref", f"REFERENCE={REFERENCE}", f"PYTHON={sys.executable}"],
             quiet=True)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print ptxas register/spill reports")
    ap.add_argument("--no-oracle", action="store_true")
    a = ap.parse_args(argv)
    lib = build_cuda(force=a.force, ptxas_v=a.ptxas_v)
    print(f"built {lib}")
    passes = build_passes(force=a.force)
    if passes:
        print(f"built {passes}")
    if not a.no_oracle:
        print(f"built {build_oracle(force=a.force)}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
