"""Time-to-RMSE of path guiding on one B200: the unguided reference tracer vs
the dense vMF-grid guide (64^3 cells x 8 lobes, FP64 EM statistics) vs the
learned BF16 MLP guide, on the seeded 1M-triangle procedural room.

Region. RMSE is taken where the reference's Application::compute_mse takes
it (Application.cpp:892-949): the 64 x 64 centre crop of the 1920 x 1080 view,
linear radiance, RGB, in FP64. The crop is rendered as its own 64 x 64 camera
(same eye and direction, vertical field of view narrowed by 64/1080).

Judge. The unguided tracer accumulated in FP64 (rr_accumulate's FP64 sum)
as two independent halves A and B of --judge-spp/2 samples per pixel. The
judge J = (A + B)/2 has its own noise, estimated as s2_J = MSE(A, B)/4 and
subtracted: MSE_true(x) ~ MSE(x, J) - s2_J (independent seeds, unbiased
estimators). Pixels that are not finite in any image are left out and
counted (the reference's arithmetic yields a non-finite sample about once
per 10^9 paths on this scene).

Methods. Each starts from scratch (fresh guide) and renders frames of
--spp samples per pixel, guide update per frame, accumulating a running mean.
Device time per frame (render + guide update + accumulate) is taken with
CUDA events; the RMSE evaluation is outside the timed region. Each method
also keeps its even and odd frames in two accumulators, whose difference
estimates its own MSE without the judge: s2_x = MSE(even, odd)/4.

Time to target. The judge-corrected relative RMSE
sqrt(MSE(x,J) - s2_J) / mean(J) is taken after every frame. Its samples are
heavy-tailed (a rare bright path lifts the error long after it first dipped
under the target), so the measured time is the one after which the error
stays at or under --target up to the end of the --budget-s run
(time_to_target_ms; the first dip is reported too). The time is also
extrapolated from the run's efficiency: an unbiased estimator's MSE falls as
1/t, so t_target = t * s2_x / (target * mean(J))^2, which uses the whole run
(time_to_target_extrapolated_ms). learned_speedup_vs_grid is the grid's
extrapolated time over the MLP's.

    python bench_guiding.py [--target 0.01 --budget-s 15 --judge-spp 2097152]
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

EYE, CENTER = (0.0, 4.0, 34.0), (0.0, -3.0, 0.0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--crop", type=int, default=64)
    ap.add_argument("--view-height", type=int, default=1080)
    ap.add_argument("--spp", type=int, default=256, help="samples per pixel per frame")
    ap.add_argument("--bounces", type=int, default=5)
    ap.add_argument("--judge-spp", type=int, default=1 << 21)
    ap.add_argument("--target", type=float, default=0.01)
    ap.add_argument("--budget-s", type=float, default=15.0, help="device-time budget per method")
    ap.add_argument("--triangles", type=int, default=1_000_000)
    ap.add_argument("--methods", default="unguided,grid,mlp")
    ap.add_argument("--mlp-batch", type=int, default=1 << 18)
    args = ap.parse_args()

    import torch
    from research_b200 import rr
    torch.cuda.set_device(0)
    L = rr.lib()
    ctx = rr.Context(0)
    hs = rr.HostScene.procedural(target_triangles=args.triangles)
    scene = rr.Scene(ctx, hs.arrays)
    W = H = args.crop
    desc = rr.camera_desc(W, H, eye=EYE, center=CENTER)
    full_fov = desc.fov_y_deg
    desc.fov_y_deg = 2.0 * math.degrees(math.atan(math.tan(math.radians(full_fov) / 2.0) * H / args.view_height))
    cam = rr.camera_data(desc)
    stream = torch.cuda.current_stream().cuda_stream
    spp = args.spp
    rad = torch.empty((spp, H, W, 4), device="cuda")

    def trace(seed, guide=None):
        p = rr.PtParams(seed, args.bounces, spp, 0)
        if guide is None:
            ctx.check(L.rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), rad.data_ptr(),
                                              stream))
        else:
            ctx.check(L.rr_guided_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), guide,
                                                     rad.data_ptr(), stream))

    def accumulate(acc, s64, first, done):
        a = rr.AccParams(W, H, 1 if first else 0, done)
        ctx.check(L.rr_accumulate_execute(ctx.handle, rad.data_ptr(), spp, acc.data_ptr(),
                                          s64.data_ptr() if s64 is not None else None, C.byref(a), stream))

    # ── judge: two independent FP64 halves of the unguided tracer ──────────
    t0 = time.perf_counter()
    halves = []
    for h in range(2):
        acc = torch.zeros((H, W, 4), device="cuda")
        s64 = torch.zeros((H, W, 4), device="cuda", dtype=torch.float64)
        done = 0
        while done < args.judge_spp // 2:
            trace((1 << 28) * (h + 1) + done)
            accumulate(acc, s64, done == 0, done)
            done += spp
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

    results = {}
    target_mse = (args.target * judge_mean) ** 2
    for method in args.methods.split(","):
        guide = None
        if method != "unguided":
            kind = rr.GUIDE_GRID if method == "grid" else rr.GUIDE_MLP
            d = rr.GuideDesc(kind, 64, 0.5, 0.9, (C.c_float * 3)(-20.5, -20.5, -20.5),
                             (C.c_float * 3)(20.5, 20.5, 20.5), 1 << 22, args.mlp_batch, 1e-2, 11)
            guide = C.c_void_p()
            ctx.check(L.rr_guide_create(ctx.handle, C.byref(d), C.byref(guide)))
        acc = torch.zeros((H, W, 4), device="cuda")
        par = [torch.zeros((H, W, 4), device="cuda") for _ in range(2)]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        elapsed_ms, frame, reached, curve = 0.0, 0, None, []
        stable = None   # (ms, spp) of the first frame of the final run of frames at or under the target
        next_log = 1
        while elapsed_ms < args.budget_s * 1e3:
            e0.record()
            trace(frame * spp, guide)
            if guide is not None:
                ctx.check(L.rr_guide_update(ctx.handle, guide, stream))
            accumulate(acc, None, frame == 0, frame * spp)
            e1.record()
            accumulate(par[frame & 1], None, frame < 2, (frame >> 1) * spp)   # outside the timed region
            torch.cuda.synchronize()
            elapsed_ms += e0.elapsed_time(e1)
            frame += 1
            x = acc[..., :3].double()
            ok = finite & torch.isfinite(x).all(-1)
            corrected = mse(x, J, ok) - s2_J
            if frame >= next_log:
                curve.append((round(elapsed_ms, 1), frame * spp, round(math.sqrt(max(corrected, 0.0)) / judge_mean, 5)))
                next_log *= 2
            if frame >= 4 and corrected <= target_mse:
                if reached is None:
                    reached = (elapsed_ms, frame * spp)
                if stable is None:
                    stable = (elapsed_ms, frame * spp)
            else:
                stable = None
        x = acc[..., :3].double()
        ok = finite & torch.isfinite(x).all(-1)
        bad = int((~ok).sum())
        corrected = mse(x, J, ok) - s2_J
        s2_x = mse(par[0][..., :3].double(), par[1][..., :3].double(), ok) / 4.0 if frame >= 2 else float("nan")
        stats = None
        if guide is not None:
            st = rr.GuideStats()
            ctx.check(L.rr_guide_get_stats(ctx.handle, guide, C.byref(st)))
            stats = {"samples_per_frame": st.samples_recorded, "samples_used": st.samples_used,
                     "update_ms": round(st.ms_update, 3), "cells_valid": st.cells_valid,
                     "loss": round(st.last_loss, 4)}
            L.rr_guide_destroy(guide)
        results[method] = {
            "time_to_target_ms": round(stable[0], 1) if stable else None,
            "spp_to_target": stable[1] if stable else None,
            "first_under_target_ms": round(reached[0], 1) if reached else None,
            "time_to_target_extrapolated_ms": round(elapsed_ms * s2_x / target_mse, 1),
            "final_rel_rmse_vs_judge": round(math.sqrt(max(corrected, 0.0)) / judge_mean, 5),
            "final_rel_rmse_self": round(math.sqrt(s2_x) / judge_mean, 5),
            "rel_sigma_per_spp": round(math.sqrt(s2_x * frame * spp) / judge_mean, 3),
            "image_mean_ratio": round(float(x[ok].mean()) / judge_mean, 5),
            "frames": frame, "spp": frame * spp, "ms_per_frame": round(elapsed_ms / frame, 3),
            "nonfinite_pixels": bad, "curve": curve, "guide": stats}

    def ratio(a, b, key):
        va, vb = results.get(a, {}).get(key), results.get(b, {}).get(key)
        return round(va / vb, 3) if va and vb else None

    line = {"metric": "time-to-RMSE 1e-2, learned vs vMF-grid guiding, 1xB200", "target_rel_rmse": args.target,
            "config": {"workload": "procedural-room-1M-tris, 64x64 centre crop of the 1920x1080 view",
                       "crop": W, "spp_per_frame": spp, "max_bounces": args.bounces,
                       "judge": f"unguided tracer, 2 x {args.judge_spp // 2} spp, FP64 accumulation",
                       "grid": "64^3 x 8 vMF lobes, FP64 EM, alpha 0.5",
                       "mlp": f"80-64x4-48 BF16 tcgen05 MLP, Adam lr 1e-2, {args.mlp_batch} samples/frame, alpha 0.5"},
            "judge": {"mean": round(judge_mean, 5), "rel_rmse_own": round(math.sqrt(s2_J) / judge_mean, 5),
                      "seconds": round(judge_s, 1), "nonfinite_pixels": int((~finite).sum())},
            "results": results,
            "learned_speedup_vs_grid": ratio("grid", "mlp", "time_to_target_extrapolated_ms"),
            "learned_speedup_vs_grid_measured": ratio("grid", "mlp", "time_to_target_ms")}
    print(json.dumps(line), flush=True)
    scene.close()
    ctx.close()


if __name__ == "__main__":
    main()
