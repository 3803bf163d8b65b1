"""Writes the regression fixtures of tests/golden/ with the CPU oracle.

They are OUR oracle's outputs on small seeded inputs, not the reference's
(the reference cannot run anywhere here and ships no golden data): they pin
the oracle and the CUDA kernels to fixed bit patterns across changes and
machines. Regenerate only when a semantic change is intended:

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


def main():
    from research_b200 import build, rr
    import oracle as O
    build.build_oracle()
    for name, arrays in compute(rr, O).items():
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        print("wrote", HERE / f"{name}.npz", {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
