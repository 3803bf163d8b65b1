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

    python bench_guiding.py [--target 0.01 --budget-s 15 --repeats 3 --judge-spp 2097152]
                            [--grid-resolution 64 --alpha 0.5 --decay 0.9]

bench.py calls measure() for the `time_to_rmse` key of its JSON line.
"""
import argparse
import ctypes as C
import json
import math
import statistics
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

EYE, CENTER = (0.0, 4.0, 34.0), (0.0, -3.0, 0.0)


GRID_BOUNDS = 20.5


class Workload:
    """The crop camera, the scene and the render / accumulate calls."""

    def __init__(self, rr, torch, ctx, scene, crop=64, view_height=1080, spp=256, bounces=5, flags=0):
        self.rr, self.torch, self.ctx, self.scene = rr, torch, ctx, scene
        self.flags = flags
        self.L = rr.lib()
        self.W = self.H = crop
        desc = rr.camera_desc(crop, crop, eye=EYE, center=CENTER)
        full_fov = desc.fov_y_deg
        desc.fov_y_deg = 2.0 * math.degrees(math.atan(math.tan(math.radians(full_fov) / 2.0) * crop / view_height))
        self.cam = rr.camera_data(desc)
        self.stream = torch.cuda.current_stream().cuda_stream
        self.spp, self.bounces = spp, bounces
        self.rad = torch.empty((spp, crop, crop, 4), device="cuda")

    def trace(self, seed, guide=None):
        p = self.rr.PtParams(seed, self.bounces, self.spp, self.flags)
        if guide is None:
            self.ctx.check(self.L.rr_pathtracer_execute(self.ctx.handle, self.scene.handle, C.byref(self.cam),
                                                        C.byref(p), self.rad.data_ptr(), self.stream))
        else:
            self.ctx.check(self.L.rr_guided_pathtracer_execute(self.ctx.handle, self.scene.handle, C.byref(self.cam),
                                                               C.byref(p), guide, self.rad.data_ptr(), self.stream))

    def accumulate(self, acc, s64, first, done):
        a = self.rr.AccParams(self.W, self.H, 1 if first else 0, done)
        self.ctx.check(self.L.rr_accumulate_execute(self.ctx.handle, self.rad.data_ptr(), self.spp, acc.data_ptr(),
                                                    s64.data_ptr() if s64 is not None else None, C.byref(a),
                                                    self.stream))


def _mse(x, y, ok):
    d = x[ok] - y[ok]
    return float((d * d).mean())


def make_judge(w: Workload, judge_spp: int):
    """Two independent FP64 halves of the unguided tracer (seeds disjoint
    from every method's)."""
    torch = w.torch
    t0 = time.perf_counter()
    halves = []
    for h in range(2):
        acc = torch.zeros((w.H, w.W, 4), device="cuda")
        s64 = torch.zeros((w.H, w.W, 4), device="cuda", dtype=torch.float64)
        done = 0
        while done < judge_spp // 2:
            w.trace((1 << 28) * (h + 1) + done)
            w.accumulate(acc, s64, done == 0, done)
            done += w.spp
        torch.cuda.synchronize()
        halves.append((s64 / done)[..., :3])
    A, B = halves
    J = (A + B) / 2
    finite = torch.isfinite(A).all(-1) & torch.isfinite(B).all(-1)
    return {"J": J, "finite": finite, "mean": float(J[finite].mean()), "s2": _mse(A, B, finite) / 4.0,
            "seconds": time.perf_counter() - t0, "spp": judge_spp}


def run_method(w: Workload, judge, method: str, target: float, budget_s: float, seed_base: int = 0,
               grid_resolution: int = 64, alpha: float = 0.5, decay: float = 0.9, mlp_batch: int = 1 << 18):
    """One method from scratch for `budget_s` of device time; returns its record."""
    rr, torch, ctx, L = w.rr, w.torch, w.ctx, w.L
    J, finite, judge_mean, s2_J = judge["J"], judge["finite"], judge["mean"], judge["s2"]
    target_mse = (target * judge_mean) ** 2
    spp = w.spp
    guide = None
    if method != "unguided":
        kind = rr.GUIDE_GRID if method == "grid" else rr.GUIDE_MLP
        d = rr.GuideDesc(kind, grid_resolution, alpha, decay, (C.c_float * 3)(*([-GRID_BOUNDS] * 3)),
                         (C.c_float * 3)(*([GRID_BOUNDS] * 3)), 1 << 22, mlp_batch, 1e-2, 11)
        guide = C.c_void_p()
        ctx.check(L.rr_guide_create(ctx.handle, C.byref(d), C.byref(guide)))
    acc = torch.zeros((w.H, w.W, 4), device="cuda")
    par = [torch.zeros((w.H, w.W, 4), device="cuda") for _ in range(2)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    elapsed_ms, frame, reached, curve = 0.0, 0, None, []
    stable = None   # (ms, spp) of the first frame of the final run of frames at or under the target
    next_log = 1
    while elapsed_ms < budget_s * 1e3:
        e0.record()
        w.trace(seed_base + frame * spp, guide)
        if guide is not None:
            ctx.check(L.rr_guide_update(ctx.handle, guide, w.stream))
        w.accumulate(acc, None, frame == 0, frame * spp)
        e1.record()
        w.accumulate(par[frame & 1], None, frame < 2, (frame >> 1) * spp)   # outside the timed region
        torch.cuda.synchronize()
        elapsed_ms += e0.elapsed_time(e1)
        frame += 1
        x = acc[..., :3].double()
        ok = finite & torch.isfinite(x).all(-1)
        corrected = _mse(x, J, ok) - s2_J
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
    corrected = _mse(x, J, ok) - s2_J
    s2_x = _mse(par[0][..., :3].double(), par[1][..., :3].double(), ok) / 4.0 if frame >= 2 else float("nan")
    stats = None
    if guide is not None:
        st = rr.GuideStats()
        ctx.check(L.rr_guide_get_stats(ctx.handle, guide, C.byref(st)))
        stats = {"samples_per_frame": st.samples_recorded, "samples_used": st.samples_used,
                 "update_ms": round(st.ms_update, 3), "cells_valid": st.cells_valid, "loss": round(st.last_loss, 4)}
        L.rr_guide_destroy(guide)
    return {"time_to_target_ms": round(stable[0], 1) if stable else None,
            "spp_to_target": stable[1] if stable else None,
            "first_under_target_ms": round(reached[0], 1) if reached else None,
            "time_to_target_extrapolated_ms": round(elapsed_ms * s2_x / target_mse, 1),
            "final_rel_rmse_vs_judge": round(math.sqrt(max(corrected, 0.0)) / judge_mean, 5),
            "final_rel_rmse_self": round(math.sqrt(s2_x) / judge_mean, 5),
            "rel_sigma_per_spp": round(math.sqrt(s2_x * frame * spp) / judge_mean, 3),
            "image_mean_ratio": round(float(x[ok].mean()) / judge_mean, 5),
            "frames": frame, "spp": frame * spp, "ms_per_frame": round(elapsed_ms / frame, 3),
            "nonfinite_pixels": bad, "curve": curve, "guide": stats}


def _ratio(a, b):
    return round(a / b, 3) if a and b else None


def measure(rr, torch, ctx, scene, methods=("unguided", "grid", "mlp"), target=0.01, budget_s=15.0, repeats=1,
            judge_spp=1 << 21, crop=64, spp=256, bounces=5, mlp_batch=1 << 18, grid_resolution=64, alpha=0.5,
            decay=0.9, flags=0, grid_variants=()):
    """Time to the target relative RMSE for each method, `repeats` times each
    (fresh guides, disjoint seeds), against one shared judge. flags: the
    tracers' RR_PT_FLAG_* (RR_PT_FLAG_EMITTERS: every method, the judge
    included, samples the emissive triangles). grid_variants: extra grid
    settings (resolution, decay, alpha), each measured as method
    "grid:<res>:<decay>:<alpha>"."""
    w = Workload(rr, torch, ctx, scene, crop=crop, spp=spp, bounces=bounces, flags=flags)
    judge = make_judge(w, judge_spp)
    all_methods = list(methods) + [f"grid:{r}:{d}:{a}" for r, d, a in grid_variants]
    runs = {m: [] for m in all_methods}
    for r in range(repeats):
        for m in all_methods:
            if m.startswith("grid:"):
                _, res, dec, alp = m.split(":")
                runs[m].append(run_method(w, judge, "grid", target, budget_s, seed_base=r * (1 << 24),
                                          grid_resolution=int(res), alpha=float(alp), decay=float(dec),
                                          mlp_batch=mlp_batch))
                continue
            runs[m].append(run_method(w, judge, m, target, budget_s, seed_base=r * (1 << 24),
                                      grid_resolution=grid_resolution, alpha=alpha, decay=decay, mlp_batch=mlp_batch))
    summary = {}
    for m, rs in runs.items():
        ext = [x["time_to_target_extrapolated_ms"] for x in rs]
        meas = [x["time_to_target_ms"] for x in rs]
        # a run that never stayed under the target counts as slower than
        # every run that did (null when that decides the median)
        med = statistics.median([x if x is not None else math.inf for x in meas])
        summary[m] = {"extrapolated_ms": ext, "extrapolated_ms_median": statistics.median(ext),
                      "measured_ms": meas,
                      "measured_ms_median": med if math.isfinite(med) else None,
                      "runs_not_reaching_target": sum(x is None for x in meas),
                      "rel_sigma_per_spp": [x["rel_sigma_per_spp"] for x in rs],
                      "image_mean_ratio": [x["image_mean_ratio"] for x in rs],
                      "ms_per_frame": statistics.median([x["ms_per_frame"] for x in rs])}
    out = {"target_rel_rmse": target, "budget_s_per_run": budget_s, "repeats": repeats,
           "judge": {"mean": round(judge["mean"], 5), "rel_rmse_own": round(math.sqrt(judge["s2"]) / judge["mean"], 5),
                     "spp": judge_spp, "seconds": round(judge["seconds"], 1),
                     "nonfinite_pixels": int((~judge["finite"]).sum())},
           "methods": summary, "runs": runs}

    def pair(num, den):
        if num not in summary or den not in summary:
            return None
        e = [_ratio(a, b) for a, b in zip(summary[num]["extrapolated_ms"], summary[den]["extrapolated_ms"])]
        mm = [_ratio(a, b) for a, b in zip(summary[num]["measured_ms"], summary[den]["measured_ms"])]
        return {"extrapolated_median": _ratio(summary[num]["extrapolated_ms_median"],
                                              summary[den]["extrapolated_ms_median"]),
                "extrapolated_per_repeat": e, "measured_median": _ratio(summary[num]["measured_ms_median"],
                                                                         summary[den]["measured_ms_median"]),
                "measured_per_repeat": mm}
    out["learned_speedup_vs_grid"] = pair("grid", "mlp")
    out["grid_speedup_vs_unguided"] = pair("unguided", "grid")
    out["learned_speedup_vs_unguided"] = pair("unguided", "mlp")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--crop", type=int, default=64)
    ap.add_argument("--spp", type=int, default=256, help="samples per pixel per frame")
    ap.add_argument("--bounces", type=int, default=5)
    ap.add_argument("--judge-spp", type=int, default=1 << 21)
    ap.add_argument("--target", type=float, default=0.01)
    ap.add_argument("--budget-s", type=float, default=15.0, help="device-time budget per method and repeat")
    ap.add_argument("--repeats", type=int, default=1)
    ap.add_argument("--triangles", type=int, default=1_000_000)
    ap.add_argument("--methods", default="unguided,grid,mlp")
    ap.add_argument("--mlp-batch", type=int, default=1 << 18)
    ap.add_argument("--grid-resolution", type=int, default=64)
    ap.add_argument("--alpha", type=float, default=0.5)
    ap.add_argument("--decay", type=float, default=0.9)
    ap.add_argument("--emitters", action="store_true",
                    help="the emitter-sampling mode (RR_PT_FLAG_EMITTERS) on the scene without the emitters' point "
                         "lights, for every method and the judge")
    ap.add_argument("--grid-variants", default="",
                    help="extra grid settings res:decay:alpha[,res:decay:alpha...] measured beside the methods")
    args = ap.parse_args()

    import torch
    from research_b200 import rr
    torch.cuda.set_device(0)
    ctx = rr.Context(0)
    hs = rr.HostScene.procedural(target_triangles=args.triangles,
                                 flags=rr.SCENE_NO_EMITTER_LIGHTS if args.emitters else 0)
    scene = rr.Scene(ctx, hs.arrays)
    variants = [tuple(v.split(":")) for v in args.grid_variants.split(",") if v]
    variants = [(int(r), float(d), float(a)) for r, d, a in variants]
    res = measure(rr, torch, ctx, scene, methods=tuple(m for m in args.methods.split(",") if m),
                  target=args.target, budget_s=args.budget_s, repeats=args.repeats, judge_spp=args.judge_spp,
                  crop=args.crop, spp=args.spp, bounces=args.bounces, mlp_batch=args.mlp_batch,
                  grid_resolution=args.grid_resolution, alpha=args.alpha, decay=args.decay,
                  flags=rr.PT_FLAG_EMITTERS if args.emitters else 0, grid_variants=variants)
    for rs in res["runs"].values():
        for x in rs:
            x.pop("curve", None)
    line = {"metric": "time-to-RMSE 1e-2, learned vs vMF-grid guiding, 1xB200",
            "config": {"workload": f"procedural-room-1M-tris, {args.crop}x{args.crop} centre crop of the 1920x1080 "
                                   "view", "spp_per_frame": args.spp, "max_bounces": args.bounces,
                       "light_sampling": "emitter triangles (RR_PT_FLAG_EMITTERS), no centroid point lights"
                       if args.emitters else "reference (point lights at the emitters' centroids)",
                       "judge": f"unguided tracer, 2 x {args.judge_spp // 2} spp, FP64 accumulation",
                       "grid": f"{args.grid_resolution}^3 x 8 vMF lobes, FP64 EM, decay {args.decay}, "
                               f"alpha {args.alpha}",
                       "mlp": f"80-64x4-48 BF16 tcgen05 MLP, Adam lr 1e-2, {args.mlp_batch} samples/frame, "
                              f"alpha {args.alpha}"},
            **res}
    print(json.dumps(line), flush=True)
    scene.close()
    ctx.close()


if __name__ == "__main__":
    main()
