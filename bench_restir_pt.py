"""ReSTIR PT (ReSTIRPTPass::execute) timing on one B200: the config-2 frame —
seeded 1M-triangle room, 1920x1080 — with the reference pass defaults
(8 candidates, 4 bounces, temporal and spatial reuse with 4 neighbours in a
12-pixel radius, guiding grid of 2^20 cells, alpha 0.5). Per frame: ReSTIR DI
(G-buffer and direct light, M = 32), then ReSTIR PT initial, temporal, spatial
shade and the guiding fit. Device time per stage from CUDA events after
--warmup frames; the camera orbits slowly so that the temporal pass
reprojects. Prints one JSON line.

    python bench_restir_pt.py [--width 1920 --height 1080 --frames 8 --warmup 3]
"""
import argparse
import ctypes as C
import json
import math
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--frames", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--triangles", type=int, default=1_000_000)
    ap.add_argument("--initial", choices=["wavefront", "per_pixel"], default="wavefront",
                    help="form of the initial pass (rr_reuse_set_wavefront)")
    args = ap.parse_args()

    import torch
    from research_b200 import rr
    torch.cuda.set_device(0)
    L = rr.lib()
    ctx = rr.Context(0)
    ctx.check(rr.lib().rr_reuse_set_wavefront(ctx.handle, 1 if args.initial == "wavefront" else 0))
    hs = rr.HostScene.procedural(target_triangles=args.triangles)
    scene = rr.Scene(ctx, hs.arrays)
    W, H = args.width, args.height
    st = torch.cuda.current_stream().cuda_stream
    dev = lambda: torch.zeros((H, W, 4), device="cuda")
    gpos, gnrm, dres, dprev, direct, out = (dev() for _ in range(6))
    res = [[dev() for _ in range(4)] for _ in range(2)]
    hist = [[dev() for _ in range(2)] for _ in range(2)]
    for h in hist:
        h[0][..., 3] = -1.0
    cells = 1 << 20
    accum = torch.zeros((cells, 4), dtype=torch.int32, device="cuda")
    fitted = torch.zeros((cells, 4), device="cuda")
    p = rr.pt_reuse_params()
    di = rr.DIParams(0, 32, 1, 1, 5, 30, 20, 0)
    imgs = rr.PtReuseImages()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    names = ("restir_di", "pt_initial", "pt_temporal", "pt_spatial_shade", "guiding_fit")
    tot = dict.fromkeys(names, 0.0)
    prev_desc = None
    for f in range(args.warmup + args.frames):
        a = 0.002 * f
        desc = rr.camera_desc(W, H, eye=(34.0 * math.sin(a), 4.0, 34.0 * math.cos(a)), center=(0.0, -3.0, 0.0))
        cam = rr.camera_data(desc, prev_desc)
        c, pv = f & 1, 1 - (f & 1)
        di.frame_seed = p.frame_seed = f
        imgs.gbuf_pos, imgs.gbuf_norm, imgs.direct = gpos.data_ptr(), gnrm.data_ptr(), direct.data_ptr()
        for k in range(4):
            imgs.reservoir_curr[k], imgs.reservoir_prev[k] = res[c][k].data_ptr(), res[pv][k].data_ptr()
        for k in range(2):
            imgs.history_curr[k], imgs.history_prev[k] = hist[c][k].data_ptr(), hist[pv][k].data_ptr()
        imgs.output, imgs.guiding_accum, imgs.guiding_fitted = out.data_ptr(), accum.data_ptr(), fitted.data_ptr()
        ev[0].record()
        ctx.check(L.rr_restir_di_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(di), gpos.data_ptr(),
                                         gnrm.data_ptr(), (dres if c else dprev).data_ptr(),
                                         (dprev if c else dres).data_ptr(), direct.data_ptr(), st))
        ev[1].record()
        ctx.check(L.rr_restir_pt_initial(ctx.handle, scene.handle, C.byref(cam), C.byref(p), C.byref(imgs), st))
        ev[2].record()
        ctx.check(L.rr_restir_pt_temporal(ctx.handle, scene.handle, C.byref(cam), C.byref(p), C.byref(imgs), st))
        ev[3].record()
        ctx.check(L.rr_restir_pt_spatial_shade(ctx.handle, scene.handle, C.byref(cam), C.byref(p), C.byref(imgs),
                                               st))
        ev[4].record()
        ctx.check(L.rr_guiding_fit(ctx.handle, accum.data_ptr(), fitted.data_ptr(), C.byref(p.guiding), st))
        ev[5].record()
        torch.cuda.synchronize()
        if f >= args.warmup:
            for k, n in enumerate(names):
                tot[n] += ev[k].elapsed_time(ev[k + 1])
        prev_desc = desc
    ms = {n: round(v / args.frames, 3) for n, v in tot.items()}
    frame_ms = sum(ms.values())
    o = out[..., :3]
    line = {"metric": "ReSTIR PT frame time, 1xB200", "unit": "ms/frame", "value": round(frame_ms, 3),
            "stages_ms": ms, "frames": args.frames, "warmup": args.warmup,
            "mpixels_per_s": round(W * H / frame_ms / 1e3, 2),
            "config": {"workload": f"procedural-room-1M-tris, {W}x{H}", "candidates": 8, "max_bounces": 4,
                       "spatial_neighbors": 4, "spatial_radius": 12, "guiding_cells": cells, "di_candidates": 32,
                       "initial": args.initial},
            "output_mean": float(o.mean()), "output_finite": bool(torch.isfinite(o).all())}
    print(json.dumps(line), flush=True)
    scene.close()
    ctx.close()


if __name__ == "__main__":
    main()
