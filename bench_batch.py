"""Config 4 on one B200: 64 independent seeded scenes of the config-2 kind
(procedural rooms) with triangle counts log-uniform in [10k, 500k] and square
images with pixel counts log-uniform in [256^2, 1024^2], 8 spp each, depth 5.
All scenes are rendered by one batch call (rr_batch_execute) in the form
the batch autotuner picked with the traversal variants: one set of wavefront
launches for all scenes (one raygen and, per bounce, one extend, one shade
and one shadow launch), replayed from a captured CUDA graph, or the scenes
one after another. Reported beside it: the wavefront form with and without
the graph, the scenes rendered one rr_pathtracer_execute call after another,
and the same forms at small images (128^2, 1 spp: the launch-bound regime,
tuned again).
Then guiding per scene (rr_batch_execute_guided): every scene gets its own
guide (a 32^3 vMF grid, or its own BF16 MLP run by one grouped tensor-core
launch per bounce for all scenes), the 8 spp are rendered as frames of
--guided-spp with every guide updated after each frame (rr_guides_update),
against the same work scene by scene.
Device time from CUDA events; prints one JSON line (Mpaths/s over the batch).

    python bench_batch.py [--scenes 64 --spp 8 --frames 3 --warmup 1]
"""
import argparse
import json
import math
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=64)
    ap.add_argument("--spp", type=int, default=8)
    ap.add_argument("--bounces", type=int, default=5)
    ap.add_argument("--frames", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--seed", type=int, default=0x5EED0004)
    ap.add_argument("--small-side", type=int, default=128)
    ap.add_argument("--small-spp", type=int, default=1)
    ap.add_argument("--guided-spp", type=int, default=2,
                    help="guided batches: spp per frame; each frame is followed by one update of every guide")
    ap.add_argument("--guides", default="grid,mlp", help="guide kinds to run per scene ('' for none)")
    ap.add_argument("--no-guided-sequential", action="store_true")
    args = ap.parse_args()

    import numpy as np
    import torch
    from research_b200 import rr
    torch.cuda.set_device(0)
    ctx = rr.Context(0)
    rng = np.random.default_rng(args.seed)
    tris = np.exp(rng.uniform(math.log(10_000), math.log(500_000), args.scenes)).astype(int)
    pixels = np.exp(rng.uniform(math.log(256 * 256), math.log(1024 * 1024), args.scenes))
    sides = (np.round(np.sqrt(pixels) / 8) * 8).astype(int)
    t0 = time.perf_counter()
    scenes, cams = [], []
    built_tris = 0
    for i in range(args.scenes):
        hs = rr.HostScene.procedural(seed=args.seed + i, target_triangles=int(tris[i]),
                                     emissive_triangles=max(16, int(tris[i]) * 4096 // 1_000_000))
        built_tris += hs.triangle_count()
        scenes.append(rr.Scene(ctx, hs.arrays))
        hs.close()
        a = rng.uniform(-0.4, 0.4)
        cams.append(rr.camera_data(rr.camera_desc(int(sides[i]), int(sides[i]),
                                                  eye=(34.0 * math.sin(a), 4.0, 34.0 * math.cos(a)),
                                                  center=(0.0, -3.0, 0.0))))
    build_s = time.perf_counter() - t0
    st = torch.cuda.current_stream().cuda_stream
    outs = [torch.empty((args.spp, int(s), int(s), 4), device="cuda") for s in sides]
    ptrs = [o.data_ptr() for o in outs]
    paths = int(sum(int(s) * int(s) for s in sides)) * args.spp
    batch = rr.Batch(ctx, scenes)
    tune = batch.tune(cams, rr.PtParams(0, args.bounces, args.spp, 0), ptrs, st)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for f in range(args.warmup):
            fn(1000 + f)
        torch.cuda.synchronize()
        ms = 0.0
        for f in range(args.frames):
            ev0.record()
            fn(2000 + 64 * f)
            ev1.record()
            torch.cuda.synchronize()
            ms += ev0.elapsed_time(ev1)
        return ms / args.frames

    mode_names = {rr.BATCH_WAVEFRONT: "wavefront", rr.BATCH_PER_SCENE: "per_scene"}
    tuned_mode = batch.mode
    ms_tuned = timed(lambda seed: batch.execute(cams, rr.PtParams(seed, args.bounces, args.spp, rr.PT_FLAG_GRAPH),
                                                ptrs, st))
    batch.set_mode(rr.BATCH_WAVEFRONT)
    ms_graph = timed(lambda seed: batch.execute(cams, rr.PtParams(seed, args.bounces, args.spp, rr.PT_FLAG_GRAPH),
                                                ptrs, st))
    ms_plain = timed(lambda seed: batch.execute(cams, rr.PtParams(seed, args.bounces, args.spp, 0), ptrs, st))

    def sequential(seed):
        import ctypes as C
        p = rr.PtParams(seed, args.bounces, args.spp, 0)
        for sc, cam, o in zip(scenes, cams, outs):
            ctx.check(rr.lib().rr_pathtracer_execute(ctx.handle, sc.handle, C.byref(cam), C.byref(p), o.data_ptr(),
                                                     st))
    ms_seq = timed(sequential)
    finite = bool(all(torch.isfinite(o).all() for o in outs))
    # the same 64 scenes at small images (launch-bound regime): one batch frame
    # is then a few milliseconds, and per-scene launches dominate the sequential form
    sm_cams = [rr.camera_data(rr.camera_desc(args.small_side, args.small_side, eye=(0.0, 4.0, 34.0),
                                             center=(0.0, -3.0, 0.0))) for _ in scenes]
    sm_outs = [torch.empty((args.small_spp, args.small_side, args.small_side, 4), device="cuda") for _ in scenes]
    sm_ptrs = [o.data_ptr() for o in sm_outs]
    sm_paths = args.scenes * args.small_side * args.small_side * args.small_spp
    sm_tune = batch.tune(sm_cams, rr.PtParams(0, args.bounces, args.small_spp, 0), sm_ptrs, st)
    sm = {"autotune": {"mode": mode_names[batch.mode], "best_extend": sm_tune.best_extend,
                       "best_shadow": sm_tune.best_shadow}}
    ms = timed(lambda seed: batch.execute(sm_cams, rr.PtParams(seed, args.bounces, args.small_spp, rr.PT_FLAG_GRAPH),
                                          sm_ptrs, st))
    sm["tuned"] = {"ms": round(ms, 3), "mpaths_s": round(sm_paths / ms / 1e3, 2)}
    batch.set_mode(rr.BATCH_WAVEFRONT)
    for name, flags in (("graph", rr.PT_FLAG_GRAPH), ("plain", 0)):
        ms = timed(lambda seed, fl=flags: batch.execute(sm_cams, rr.PtParams(seed, args.bounces, args.small_spp, fl),
                                                        sm_ptrs, st))
        sm[name] = {"ms": round(ms, 3), "mpaths_s": round(sm_paths / ms / 1e3, 2)}

    def sm_sequential(seed):
        import ctypes as C
        p = rr.PtParams(seed, args.bounces, args.small_spp, 0)
        for sc, cam, o in zip(scenes, sm_cams, sm_outs):
            ctx.check(rr.lib().rr_pathtracer_execute(ctx.handle, sc.handle, C.byref(cam), C.byref(p), o.data_ptr(),
                                                     st))
    ms = timed(sm_sequential)
    sm["sequential"] = {"ms": round(ms, 3), "mpaths_s": round(sm_paths / ms / 1e3, 2)}
    sm["config"] = {"side": args.small_side, "spp": args.small_spp, "paths_per_batch": sm_paths}
    # back to the large images' tuning for the guided section
    ctx.check(rr.lib().rr_pathtracer_set_variants(ctx.handle, tune.best_extend, tune.best_shadow))
    batch.set_mode(tuned_mode)

    # learned (or grid) guiding per scene: the batch's spp rendered as frames
    # of --guided-spp with one guide per scene, every guide updated after each
    # frame (rr_guides_update: one host wait for all sample counts), against
    # the same work scene by scene (rr_guided_pathtracer_execute +
    # rr_guide_update per scene)
    import ctypes as C
    L = rr.lib()
    gspp = args.guided_spp
    gframes = max(1, args.spp // gspp)
    g_outs = [torch.empty((gspp, int(s), int(s), 4), device="cuda") for s in sides]
    g_ptrs = [o.data_ptr() for o in g_outs]
    guided = {}
    for kind in [k for k in args.guides.split(",") if k]:
        gk = rr.GUIDE_GRID if kind == "grid" else rr.GUIDE_MLP
        guides = []
        for i in range(args.scenes):
            d = rr.GuideDesc(gk, 32, 0.5, 0.8, (C.c_float * 3)(-52.0, -52.0, -52.0), (C.c_float * 3)(52.0, 52.0, 52.0),
                             1 << 20, 1 << 16, 1e-2, 100 + i)
            h = C.c_void_p()
            ctx.check(L.rr_guide_create(ctx.handle, C.byref(d), C.byref(h)))
            guides.append(h)
        garr = (C.c_void_p * len(guides))(*[g.value for g in guides])

        def batch_frames(seed, update=True):
            for j in range(gframes):
                batch.execute_guided(cams, rr.PtParams(seed + j * gspp, args.bounces, gspp, rr.PT_FLAG_GRAPH),
                                     [g.value for g in guides], g_ptrs, st)
                if update:
                    ctx.check(L.rr_guides_update(ctx.handle, garr, len(guides), st))

        ms_g = timed(batch_frames)
        ms_render = timed(lambda seed: batch_frames(seed, update=False))
        entry = {"ms_per_batch": round(ms_g, 3), "mpaths_s": round(paths / ms_g / 1e3, 2),
                 "render_only": {"ms": round(ms_render, 3), "mpaths_s": round(paths / ms_render / 1e3, 2)},
                 "frames_per_batch": gframes, "spp_per_frame": gspp}
        if not args.no_guided_sequential:
            def seq_frames(seed):
                for j in range(gframes):
                    p = rr.PtParams(seed + j * gspp, args.bounces, gspp, 0)
                    for sc, cam, o, g in zip(scenes, cams, g_outs, guides):
                        ctx.check(L.rr_guided_pathtracer_execute(ctx.handle, sc.handle, C.byref(cam), C.byref(p), g,
                                                                 o.data_ptr(), st))
                        ctx.check(L.rr_guide_update(ctx.handle, g, st))
            ms_s = timed(seq_frames)
            entry["sequential_scenes"] = {"ms": round(ms_s, 3), "mpaths_s": round(paths / ms_s / 1e3, 2)}
        gst = rr.GuideStats()
        rec = []
        for g in guides:
            ctx.check(L.rr_guide_get_stats(ctx.handle, g, C.byref(gst)))
            rec.append(gst.samples_recorded)
        entry["samples_recorded_per_scene"] = {"min": int(min(rec)), "max": int(max(rec))}
        entry["finite"] = bool(all(torch.isfinite(o).all() for o in g_outs))
        if gk == rr.GUIDE_MLP:
            err = C.c_int(0)
            bad = 0
            for g in guides:
                ctx.check(L.rr_guide_mlp_params(ctx.handle, g, None, None, None, rr.MLP_PARAM_COUNT, C.byref(err)))
                bad += err.value
            entry["tensor_core_wait_errors"] = bad
        guided[kind] = entry
        for g in guides:
            L.rr_guide_destroy(g)
    line = {"metric": "Mpaths/s, 64-scene batch (autotuned form, RR_PT_FLAG_GRAPH), 1xB200",
            "value": round(paths / ms_tuned / 1e3, 2), "unit": "Mpaths/s", "ms_per_batch": round(ms_tuned, 3),
            "wavefront_graph_batch": {"ms": round(ms_graph, 3), "mpaths_s": round(paths / ms_graph / 1e3, 2)},
            "plain_batch": {"ms": round(ms_plain, 3), "mpaths_s": round(paths / ms_plain / 1e3, 2)},
            "sequential_scenes": {"ms": round(ms_seq, 3), "mpaths_s": round(paths / ms_seq / 1e3, 2)},
            "autotune": {"mode": mode_names[tuned_mode], "best_extend": tune.best_extend,
                         "best_shadow": tune.best_shadow,
                         "extend_ms": [round(x, 2) for x in tune.extend_ms],
                         "shadow_ms": [round(x, 2) for x in tune.shadow_ms]},
            "config": {"workload": "64 procedural rooms, 10k-500k triangles, 256^2-1024^2 pixels", "scenes": args.scenes,
                       "spp": args.spp, "max_bounces": args.bounces, "paths_per_batch": paths,
                       "triangles_total": int(built_tris), "pixels_total": int(sum(int(s) ** 2 for s in sides)),
                       "guiding": "none (the reference path tracer)"},
            "small_images": sm,
            "guided_per_scene": {"config": {"grid": "32^3 cells x 8 vMF lobes per scene",
                                            "mlp": "80-64-64-64-64-48 BF16 MLP per scene, Adam lr 1e-2, "
                                                   "2^16 samples per update",
                                            "max_samples_per_scene": 1 << 20},
                                 **guided},
            "frames": args.frames, "warmup": args.warmup, "scene_build_s": round(build_s, 1), "finite": finite}
    print(json.dumps(line), flush=True)
    batch.close()
    for sc in scenes:
        sc.close()
    ctx.close()


if __name__ == "__main__":
    main()
