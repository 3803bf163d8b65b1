"""Writes the regression fixtures of tests/golden/ from the reference's own
shader text, run here on the CPU.

The reference cannot run as shipped (Vulkan ray queries, Slang, a Windows
toolchain) and ships no golden data. oracle/make_ref.py rewrites its shader
files mechanically into C++ and oracle/slang_ref_harness.cpp runs their
compute entry points (oracle/_ref/librr_slangref.so, built from the
reference checkout): these fixtures are that run's outputs on small seeded
inputs. The script also requires the hand-written oracle to produce the same
bits before it writes anything. Regenerate only when a semantic change is
intended (needs the reference checkout):

    python tests/golden/make_golden.py

Fixtures (RGBA32F images as float32 arrays, bit-exact expectations):
  cornell_pt.npz    Cornell box (Scene::build_cornell_box), camera defaults,
                    32x24, frame seeds 3..4 (2 spp), 8 bounces
  restir_di.npz     Cornell box, 24x16, ReSTIR DI frame 0 (M=8, K=4, R=15):
                    G-buffer, reservoir, shaded output
  atrous.npz        A-trous 5 iterations over restir_di's output and G-buffer
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

CORNELL_PT = dict(width=32, height=24, frame_seed=3, max_bounces=8, spp=2)
DI = dict(width=24, height=16, frame_seed=0, candidates=8, neighbors=4, radius=15)
ATROUS_ITERATIONS = 5


def compute(rr, O):
    """The fixtures' contents from the hand-written oracle."""
    hs = rr.HostScene.cornell(0)
    osc = O.OracleScene(hs.arrays, use_bvh=False)
    c = CORNELL_PT
    cam = rr.camera_data(rr.camera_desc(c["width"], c["height"]))
    pt, _ = O.pathtrace(osc, cam, c["frame_seed"], c["max_bounces"], c["spp"])
    d = DI
    cam = rr.camera_data(rr.camera_desc(d["width"], d["height"]))
    p = O.di_params(d["frame_seed"], d["candidates"], 1, 1, d["neighbors"], d["radius"], 20)
    z = lambda: np.zeros((d["height"], d["width"], 4), np.float32)
    gpos, gnrm, res, out = z(), z(), z(), z()
    O.restir_di_initial(osc, cam, p, gpos, gnrm, res)
    O.restir_di_spatial_shade(osc, cam, p, gpos, gnrm, res, out)
    den = O.atrous(out, gpos, gnrm, ATROUS_ITERATIONS)
    hs.close()
    return {"cornell_pt": {"images": pt},
            "restir_di": {"gbuf_pos": gpos, "gbuf_norm": gnrm, "reservoir": res, "output": out},
            "atrous": {"output": den}}


def compute_reference_text(rr, O, S):
    """The same contents from the reference's shader text (S = slang_ref);
    cs_temporal is not dispatched, as in compute()."""
    hs = rr.HostScene.cornell(0)
    osc = O.OracleScene(hs.arrays, use_bvh=False)
    ref = S.RefScene(hs.arrays, osc)
    c = CORNELL_PT
    cam = rr.camera_data(rr.camera_desc(c["width"], c["height"]))
    pt = S.pathtrace(ref, cam, c["frame_seed"], c["max_bounces"], c["spp"])
    d = DI
    cam = rr.camera_data(rr.camera_desc(d["width"], d["height"]))
    p = O.di_params(d["frame_seed"], d["candidates"], 1, 1, d["neighbors"], d["radius"], 20)
    z = lambda: np.zeros((d["height"], d["width"], 4), np.float32)
    gpos, gnrm, res, prev, out = z(), z(), z(), z(), z()
    S.restir_di(0, ref, cam, p, gpos, gnrm, res, prev, out)
    S.restir_di(2, ref, cam, p, gpos, gnrm, res, prev, out)
    den = S.atrous(out, gpos, gnrm, ATROUS_ITERATIONS)
    ref.close()
    hs.close()
    return {"cornell_pt": {"images": pt},
            "restir_di": {"gbuf_pos": gpos, "gbuf_norm": gnrm, "reservoir": res, "output": out},
            "atrous": {"output": den}}


def main():
    from research_b200 import build, rr
    import oracle as O
    import slang_ref as S
    build.build_oracle()
    if not S.available():
        sys.exit("make_golden: the reference-text checker is not built (needs the reference checkout)")
    fixtures = compute_reference_text(rr, O, S)
    mine = compute(rr, O)
    for name, arrays in fixtures.items():
        for k, v in arrays.items():
            if not np.array_equal(v.view(np.uint32), mine[name][k].view(np.uint32)):
                sys.exit(f"make_golden: the oracle differs from the reference text in {name}.{k}; nothing written")
    for name, arrays in fixtures.items():
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        print("wrote", HERE / f"{name}.npz", {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
