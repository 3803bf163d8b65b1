"""Large-scene guiding on one B200: the seeded instanced scene of 10.24M fp32
triangles (4096 instances of 16 base meshes of 2,500 triangles under random
rotations, scales [0.2, 3] and translations in a box of half-size
--box-half (250: a sparse cloud seen mostly against the sky; 40: dense
clutter where indirect light dominates); 16,384
emissive triangles, each also a point light), 3840 x 2160, 1 sample per
pixel per frame over --frames frames. Every frame runs ReSTIR DI (32
candidates, temporal M-cap 20, 5 spatial neighbours in 30 px) and a path
tracer — unguided, guided by the dense vMF grid (64^3 x 8 lobes, FP64 EM) or
by the learned BF16 MLP — followed by the guide update and accumulation.

Judge. The unguided tracer at --judge-spp samples per pixel (two FP64
halves A, B) over the --crop x --crop centre crop of the view (a camera with
the same eye and the field of view narrowed to the crop, whose pixel rays are
those of the full view's centre pixels). Its own noise s2_J = MSE(A, B)/4 is
subtracted from every method's MSE against J = (A + B)/2.

Equal-RMSE comparison. Each method's accumulated image after --frames
frames is compared with J on the crop (judge-corrected relative RMSE), and
its own noise is estimated from its even/odd frames (s2_x = MSE(even,
odd)/4). An unbiased estimator's MSE falls as 1/t, so the time a method needs
to reach the grid guide's final error is t * s2_x / s2_grid; the learned
guide's speed-up at equal RMSE is the grid's time over that. Frame time is
device time (CUDA events) of DI + trace + guide update + accumulate; the
crop bookkeeping runs outside it. Prints one JSON line.

    python bench_large.py [--frames 64 --judge-spp 4096 --crop 128]
"""
import argparse
import ctypes as C
import json
import math
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CENTER = (0.0, 0.0, 0.0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=3840)
    ap.add_argument("--height", type=int, default=2160)
    ap.add_argument("--frames", type=int, default=64)
    ap.add_argument("--bounces", type=int, default=5)
    ap.add_argument("--crop", type=int, default=128)
    ap.add_argument("--judge-spp", type=int, default=4096)
    ap.add_argument("--methods", default="unguided,grid,mlp")
    ap.add_argument("--mlp-batch", type=int, default=1 << 18)
    ap.add_argument("--instances", type=int, default=4096)
    ap.add_argument("--box-half", type=float, default=250.0,
                    help="half-size of the instance placement box (250: sparse, 40: dense clutter)")
    ap.add_argument("--emitters", action="store_true",
                    help="no centroid point lights; the tracers, the judge and ReSTIR DI sample the emissive "
                         "triangles (RR_PT_FLAG_EMITTERS, RR_DI_FLAG_EMITTERS)")
    args = ap.parse_args()

    import torch
    from research_b200 import rr
    torch.cuda.set_device(0)
    L = rr.lib()
    ctx = rr.Context(0)
    t0 = time.perf_counter()
    hs = rr.HostScene.instanced(instance_count=args.instances, box_half=args.box_half,
                                flags=rr.SCENE_NO_EMITTER_LIGHTS if args.emitters else 0)
    ptf = rr.PT_FLAG_EMITTERS if args.emitters else 0
    dif = rr.DI_FLAG_EMITTERS if args.emitters else 0
    scene = rr.Scene(ctx, hs.arrays)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    n_tris = hs.triangle_count()
    W, H, c = args.width, args.height, args.crop
    x0, y0 = (W - c) // 2, (H - c) // 2
    # the eye 1.32 box half-sizes out on +z, a little above the centre plane
    eye = (0.0, 0.12 * args.box_half, 1.32 * args.box_half)
    desc = rr.camera_desc(W, H, eye=eye, center=CENTER)
    cam = rr.camera_data(desc)
    cdesc = rr.camera_desc(c, c, eye=eye, center=CENTER)
    cdesc.fov_y_deg = 2.0 * math.degrees(math.atan(math.tan(math.radians(desc.fov_y_deg) / 2.0) * c / H))
    ccam = rr.camera_data(cdesc)
    st = torch.cuda.current_stream().cuda_stream

    # ── judge ──────────────────────────────────────────────────────────────
    t0 = time.perf_counter()
    jspp = 256
    jrad = torch.empty((jspp, c, c, 4), device="cuda")
    halves = []
    for h in range(2):
        acc = torch.zeros((c, c, 4), device="cuda")
        s64 = torch.zeros((c, c, 4), device="cuda", dtype=torch.float64)
        done = 0
        while done < args.judge_spp // 2:
            p = rr.PtParams((1 << 28) * (h + 1) + done, args.bounces, jspp, ptf)
            ctx.check(L.rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(ccam), C.byref(p), jrad.data_ptr(),
                                              st))
            a = rr.AccParams(c, c, 1 if done == 0 else 0, done)
            ctx.check(L.rr_accumulate_execute(ctx.handle, jrad.data_ptr(), jspp, acc.data_ptr(), s64.data_ptr(),
                                              C.byref(a), st))
            done += jspp
        torch.cuda.synchronize()
        halves.append((s64 / done)[..., :3])
    A, B = halves
    J = (A + B) / 2
    finite = torch.isfinite(A).all(-1) & torch.isfinite(B).all(-1)
    judge_mean = float(J[finite].mean())

    def mse(x, y, ok):
        d = x[ok] - y[ok]
        return float((d * d).mean())

    s2_J = mse(A, B, finite) / 4.0
    judge_s = time.perf_counter() - t0
    del jrad

    # ── methods ────────────────────────────────────────────────────────────
    rad = torch.empty((1, H, W, 4), device="cuda")
    acc = torch.zeros((H, W, 4), device="cuda")
    gpos, gnrm, dres0, dres1, direct = (torch.zeros((H, W, 4), device="cuda") for _ in range(5))
    di = rr.DIParams(0, 32, 1, 1, 5, 30, 20, dif)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    results = {}
    for method in args.methods.split(","):
        guide = None
        if method != "unguided":
            kind = rr.GUIDE_GRID if method == "grid" else rr.GUIDE_MLP
            bh = args.box_half + 10.0
            d = rr.GuideDesc(kind, 64, 0.5, 0.9, (C.c_float * 3)(-bh, -bh, -bh), (C.c_float * 3)(bh, bh, bh),
                             1 << 22, args.mlp_batch, 1e-2, 11)
            guide = C.c_void_p()
            ctx.check(L.rr_guide_create(ctx.handle, C.byref(d), C.byref(guide)))
        par = [torch.zeros((c, c, 3), device="cuda", dtype=torch.float64) for _ in range(2)]
        tot = dict(restir_di=0.0, trace=0.0, guide_update=0.0, accumulate=0.0)
        dres0.zero_(); dres1.zero_()
        for f in range(args.frames):
            di.frame_seed = f
            ev[0].record()
            ctx.check(L.rr_restir_di_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(di), gpos.data_ptr(),
                                             gnrm.data_ptr(), (dres0 if f & 1 else dres1).data_ptr(),
                                             (dres1 if f & 1 else dres0).data_ptr(), direct.data_ptr(), st))
            ev[1].record()
            p = rr.PtParams(f, args.bounces, 1, ptf)
            if guide is None:
                ctx.check(L.rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), rad.data_ptr(),
                                                  st))
            else:
                ctx.check(L.rr_guided_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), guide,
                                                         rad.data_ptr(), st))
            ev[2].record()
            if guide is not None:
                ctx.check(L.rr_guide_update(ctx.handle, guide, st))
            ev[3].record()
            a = rr.AccParams(W, H, 1 if f == 0 else 0, f)
            ctx.check(L.rr_accumulate_execute(ctx.handle, rad.data_ptr(), 1, acc.data_ptr(), None, C.byref(a), st))
            ev[4].record()
            par[f & 1] += rad[0, y0:y0 + c, x0:x0 + c, :3].double()   # outside the timed region
            torch.cuda.synchronize()
            for k, n in enumerate(tot):
                tot[n] += ev[k].elapsed_time(ev[k + 1])
        x = acc[y0:y0 + c, x0:x0 + c, :3].double()
        ok = finite & torch.isfinite(x).all(-1) & torch.isfinite(par[0]).all(-1) & torch.isfinite(par[1]).all(-1)
        half = args.frames // 2
        s2_x = mse(par[0] / half, par[1] / (args.frames - half), ok) / 4.0
        corrected = mse(x, J, ok) - s2_J
        frame_ms = sum(tot.values()) / args.frames
        stats = None
        if guide is not None:
            gs = rr.GuideStats()
            ctx.check(L.rr_guide_get_stats(ctx.handle, guide, C.byref(gs)))
            stats = {"samples_per_frame": gs.samples_recorded, "samples_used": gs.samples_used,
                     "cells_valid": gs.cells_valid, "loss": round(gs.last_loss, 4)}
            L.rr_guide_destroy(guide)
        results[method] = {
            "ms_per_frame": round(frame_ms, 3), "stages_ms": {k: round(v / args.frames, 3) for k, v in tot.items()},
            "trace_mpaths_s": round(W * H * args.frames / tot["trace"] / 1e3, 2),
            "final_rel_rmse_vs_judge": round(math.sqrt(max(corrected, 0.0)) / judge_mean, 5),
            "rel_rmse_self": round(math.sqrt(s2_x) / judge_mean, 5),
            "mse_x_time": s2_x * frame_ms * args.frames,
            "mse_x_time_trace_only": s2_x * (frame_ms - tot["restir_di"] / args.frames) * args.frames,
            "image_mean_ratio": round(float(x[ok].mean()) / judge_mean, 5),
            "nonfinite_pixels": int((~ok).sum()), "guide": stats}

    def speedup(key):
        g, m = results.get("grid", {}).get(key), results.get("mlp", {}).get(key)
        return round(g / m, 3) if g and m else None

    if "grid" in results:
        ref_mse = (results["grid"]["rel_rmse_self"] * judge_mean) ** 2
        for r in results.values():
            r["time_to_grid_rmse_ms"] = round(r["mse_x_time"] / ref_mse, 1) if ref_mse > 0 else None
    line = {"metric": "time to equal RMSE, learned vs vMF-grid guiding, 10M-triangle instanced scene at 4K, 1xB200",
            "unit": "x (grid time / learned time at the grid's final RMSE)",
            "value": speedup("mse_x_time"), "learned_speedup_trace_only": speedup("mse_x_time_trace_only"),
            "config": {"workload": "instanced 4096 x 2.5k-tri meshes (10.24M tris), 16384 emissive tris, 3840x2160",
                       "light_sampling": "emitter triangles (RR_PT_FLAG_EMITTERS, RR_DI_FLAG_EMITTERS), no centroid "
                                         "point lights" if args.emitters else "reference (centroid point lights)",
                       "box_half": args.box_half, "eye": list(eye),
                       "triangles": n_tris, "frames": args.frames, "spp_per_frame": 1, "max_bounces": args.bounces,
                       "restir_di": "32 candidates, M-cap 20, 5 neighbours r=30",
                       "crop": c, "judge": f"unguided tracer, 2 x {args.judge_spp // 2} spp, FP64",
                       "grid": "64^3 x 8 vMF lobes, FP64 EM, alpha 0.5",
                       "mlp": f"80-64x4-48 BF16 tcgen05 MLP, Adam lr 1e-2, {args.mlp_batch} samples/frame"},
            "judge": {"mean": round(judge_mean, 5), "rel_rmse_own": round(math.sqrt(s2_J) / judge_mean, 5),
                      "seconds": round(judge_s, 1), "nonfinite_pixels": int((~finite).sum())},
            "scene_build_s": round(build_s, 1), "results": results}
    print(json.dumps(line), flush=True)
    scene.close()
    hs.close()
    ctx.close()


if __name__ == "__main__":
    main()
