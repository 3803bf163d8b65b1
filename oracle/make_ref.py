"""Mechanical rewrite of the reference's Slang shaders into C++ (TEST
INFRASTRUCTURE ONLY: the output is a checker, never shipped or measured).

    python oracle/make_ref.py [--reference DIR] [--out oracle/_ref]

reads the reference's own shader files from DIR (default: the reference
checkout at /root/reference) and writes oracle/_ref/slang_ref_gen.h, which
oracle/slang_ref_harness.cpp compiles against oracle/slang_shim.h into
oracle/_ref/librr_slangref.so (recipe: oracle/Makefile, target `ref`). The
output directory is git-ignored: the reference's text is never committed.

Each pass becomes one C++ namespace (nested in `slang`, so that the shim's
intrinsics hide the C library's) holding the flattened text of the pass and
of the includes it pulls in, each include once, in first-use order. The
rewrite changes syntax only:
  - `[shader(...)]`, `[numthreads(...)]` and `: SV_...` semantics are dropped;
    `[[vk::push_constant]] PushConstants pc;` becomes a namespace-scope
    `static` object the harness fills; `#include "BindlessHeap.slang"` is
    replaced by the shim's heap arrays; `import "X";` includes X once;
  - `inout T x` / `out T x` parameters become `T& x`;
  - multi-letter swizzles `.xyz`, `.rgb`, `.xy` become calls `.xyz()` /
    `.xy()` (single components are members);
  - `(float3x3)expr` becomes `to_float3x3(expr)`, `(Struct)0` becomes
    `Struct{}` (a zero-initialised struct);
  - unsuffixed floating literals get an `f` suffix (Slang floats are 32-bit);
  - vector constructor calls `floatN(a, b)` become `floatN{a, b}`, and a call
    with several random-number draws among its arguments evaluates them into
    temporaries first, so that arguments are evaluated left to right as in
    Slang (C++ leaves their order unspecified).
Nothing else is touched: every expression, constant, branch and loop is the
reference's.
"""
from __future__ import annotations

import argparse
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
DEFAULT_REF = Path("/root/reference")
SHADERS = Path("assets/shaders")
INCLUDE_DIR = SHADERS / "include"

# (namespace, shader file relative to assets/shaders)
PASSES = [
    ("ref_inc", None),   # only the shared includes, for function-level checks
    ("ref_pt", "passes/pathtracer_reference/pathtracer.slang"),
    ("ref_acc", "passes/accumulate/accumulate.slang"),
    ("ref_di", "passes/restir_di/restir_di.slang"),
    ("ref_atrous", "passes/denoise/atrous.slang"),
    ("ref_rpt", "passes/restir_pt/restir_pt.slang"),
    ("ref_rgi", "passes/restir_gi/restir_gi.slang"),
]
# the includes the function-level namespace pulls in
SHARED_INCLUDES = ["Common.slang", "Sampling.slang", "BRDF.slang", "GpuScene.slang", "GuidingGrid.slang"]
SKIP_INCLUDES = {"BindlessHeap.slang"}

VEC_TYPES = r"(?:float|int|uint|bool)[234]"


def _match_paren(s: str, i: int) -> int:
    """Index of the ')' closing the '(' at s[i]."""
    depth = 0
    for j in range(i, len(s)):
        c = s[j]
        if c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
            if depth == 0:
                return j
    raise ValueError("unbalanced parentheses")


def _split_args(body: str) -> list[str]:
    """Top-level comma split of an argument list."""
    out, depth, cur = [], 0, []
    for c in body:
        if c in "([{":
            depth += 1
        elif c in ")]}":
            depth -= 1
        if c == "," and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(c)
    out.append("".join(cur))
    return out


def _strip_comments(src: str) -> str:
    src = re.sub(r"/\*.*?\*/", lambda m: "\n" * m.group(0).count("\n"), src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def _vector_ctors_to_braces(s: str) -> str:
    """floatN(a, b, ...) -> floatN{a, b, ...} (left-to-right evaluation)."""
    pat = re.compile(r"\b(" + VEC_TYPES + r")\s*\(")
    i = 0
    out = []
    while True:
        m = pat.search(s, i)
        if not m:
            out.append(s[i:])
            break
        open_i = m.end() - 1
        close_i = _match_paren(s, open_i)
        inner = _vector_ctors_to_braces(s[open_i + 1:close_i])
        out.append(s[i:m.start()])
        out.append(m.group(1) + "{" + inner + "}")
        i = close_i + 1
    return "".join(out)


RAND_CALL = re.compile(r"\brand_float2?\s*\(")


def _sequence_random_arguments(s: str) -> str:
    """f(rand_float(seed), rand_float(seed), x) -> an immediately invoked
    lambda that draws the arguments in order, then calls f."""
    pat = re.compile(r"\b([A-Za-z_]\w*)\s*\(")
    i = 0
    out = []
    keywords = {"if", "for", "while", "switch", "return", "sizeof"}
    while True:
        m = pat.search(s, i)
        if not m:
            out.append(s[i:])
            break
        name = m.group(1)
        open_i = m.end() - 1
        close_i = _match_paren(s, open_i)
        body = s[open_i + 1:close_i]
        args = _split_args(body)
        draws = [a for a in args if RAND_CALL.search(a)]
        if name not in keywords and len(args) > 1 and len(draws) > 1 and "{" not in body:
            temps, call_args = [], []
            for k, a in enumerate(args):
                if RAND_CALL.search(a):
                    temps.append(f"auto __arg{k} = ({a.strip()});")
                    call_args.append(f"__arg{k}")
                else:
                    call_args.append(a.strip())
            out.append(s[i:m.start()])
            out.append("[&] { " + " ".join(temps) + f" return {name}(" + ", ".join(call_args) + "); }()")
            i = close_i + 1
        else:
            out.append(s[i:open_i + 1])
            i = open_i + 1
    return "".join(out)


FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")


def rewrite(src: str) -> str:
    s = _strip_comments(src)
    s = re.sub(r"^\s*\[shader\([^)]*\)\]\s*$", "", s, flags=re.M)
    s = re.sub(r"^\s*\[numthreads\([^)]*\)\]\s*$", "", s, flags=re.M)
    s = re.sub(r"\[\[vk::push_constant\]\]\s*", "static ", s)
    s = re.sub(r"\s*:\s*SV_\w+", "", s)
    s = re.sub(r"\b(?:inout|out)\s+(\w+)\s+(\w+)", r"\1& \2", s)
    s = re.sub(r"\.(xyz|rgb)\b(?!\s*\()", ".xyz()", s)
    s = re.sub(r"\.(xy)\b(?!\s*\()", ".xy()", s)
    s = re.sub(r"\(float3x3\)\s*([A-Za-z_]\w*(?:\.\w+)*)", r"to_float3x3(\1)", s)
    s = re.sub(r"\(([A-Z]\w*)\)\s*0\b", r"\1{}", s)   # (Struct)0: a zero-initialised struct
    s = FLOAT_LIT.sub(lambda m: m.group(1) + "f", s)
    s = _sequence_random_arguments(s)
    s = _vector_ctors_to_braces(s)
    return s


def flatten(path: Path, seen: set[str]) -> str:
    """The file's text with its includes/imports expanded once each."""
    text = path.read_text(encoding="utf-8")
    parts = []
    for line in text.splitlines(keepends=True):
        m = re.match(r'\s*#include\s+"([^"]+)"', line) or re.match(r'\s*import\s+"([^"]+)"\s*;', line)
        if m:
            name = m.group(1)
            if not name.endswith(".slang"):
                name += ".slang"
            if name in SKIP_INCLUDES or name in seen:
                parts.append("\n")
                continue
            seen.add(name)
            inc = path.parent / name                       # an include importing another
            if not inc.exists():
                inc = path.parents[2] / "include" / name   # a pass under passes/<name>/
            parts.append(flatten(inc.resolve(), seen))
            continue
        parts.append(line)
    return "".join(parts)


def generate(ref_root: Path) -> str:
    out = ["// Generated by oracle/make_ref.py from the reference's shader files; do not edit or commit.\n",
           "#pragma once\n#include \"slang_shim.h\"\n\n"]
    for ns, rel in PASSES:
        seen: set[str] = set()
        if rel is None:
            chunks = []
            for f in SHARED_INCLUDES:
                if f not in seen:
                    seen.add(f)
                    chunks.append(flatten(ref_root / INCLUDE_DIR / f, seen))
            text = "".join(chunks)
            src_name = ", ".join(str(INCLUDE_DIR / f) for f in SHARED_INCLUDES)
        else:
            p = ref_root / SHADERS / rel
            text = flatten(p, seen)
            src_name = str(SHADERS / rel)
        out.append(f"// ── {ns}: {src_name}\n")
        out.append(f"namespace slang {{ namespace {ns} {{\n")
        out.append(rewrite(text))
        out.append(f"\n}} }} // namespace slang::{ns}\n\n")
    return "".join(out)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", type=Path, default=DEFAULT_REF)
    ap.add_argument("--out", type=Path, default=HERE / "_ref")
    a = ap.parse_args(argv)
    if not (a.reference / SHADERS).is_dir():
        print(f"make_ref: no reference shaders under {a.reference / SHADERS}", file=sys.stderr)
        return 2
    a.out.mkdir(parents=True, exist_ok=True)
    target = a.out / "slang_ref_gen.h"
    text = generate(a.reference)
    if not target.exists() or target.read_text() != text:
        target.write_text(text)
    print(target)
    return 0


if __name__ == "__main__":
    sys.exit(main())
