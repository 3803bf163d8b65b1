"""Benchmark: Mpaths/s at 1080p on the procedural 1M-triangle scene.

One step = one full frame of the configuration "1M-triangle procedural room,
1920x1080, 4 spp, ReSTIR DI 32 candidates / temporal M-cap 20*M / 5 spatial
neighbours r=30 px, A-trous 5 iterations":
    path tracer (4 consecutive frame seeds, depth 5) -> accumulate (4 images)
    -> ReSTIR DI (initial, temporal, spatial+shade) -> A-trous x5.
value = W*H*spp paths per step / device time of the whole step (max over
ranks). Multi-GPU runs are independent replicas (each rank renders its own
frame sequence; only the timing is reduced).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints exactly one JSON line on rank 0. Beside the timed frames it reports,
outside the timed region: `parity` (the benchmarked frame against the
oracle), `cpu_baseline`, and `time_to_rmse` (the metric's second half:
bench_guiding.measure on the same scene).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mpaths/s at 1080p"
UNIT = "Mpaths/s"
WORKLOAD = "procedural-room-1M-tris-1080p-4spp-restirdi32-atrous5"
CFG = dict(width=1920, height=1080, spp=4, max_bounces=5, di_candidates=32, di_neighbors=5, di_radius=30,
           m_cap_factor=20, atrous_iterations=5, scene_seed=0x5EED0002, triangles=1_000_000, emitters=4096,
           box_half=20.0, eye=(0.0, 4.0, 34.0), center=(0.0, -3.0, 0.0))
# Algorithmic bytes (per unit): a ray record 32 B in + 16 B hit out, a BVH2
# node (two child boxes) 64 B, a triangle (3 vertices) 36 B.
# A node of the 4-wide tree (the wide traversal variants) holds four child
# boxes: 128 B (rr_pathtracer_variant_width).
RAY_BYTES, NODE_BYTES, TRI_BYTES = 48, 64, 36


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--width", type=int, default=CFG["width"])
    ap.add_argument("--height", type=int, default=CFG["height"])
    ap.add_argument("--triangles", type=int, default=CFG["triangles"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle check of the benchmarked frame")
    ap.add_argument("--no-time-to-rmse", action="store_true", help="skip the guiding time-to-RMSE measurement")
    ap.add_argument("--no-emitter-mode", action="store_true",
                    help="skip the frame measured with emitter sampling on the scene without centroid point lights")
    ap.add_argument("--rmse-budget-s", type=float, default=6.0,
                    help="device seconds per method and repeat of the time-to-RMSE measurement")
    ap.add_argument("--rmse-repeats", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU-baseline sample budget")
    ap.add_argument("--variants", default=None,
                    help="E,S: traversal variants for extension and shadow rays instead of the autotuner's choice "
                         "(profilers distort the tuner's timings)")
    ap.add_argument("--serial-passes", action="store_true",
                    help="run ReSTIR DI and A-trous after the path tracer on one stream")
    return ap.parse_args()


def dist_init(args):
    from research_b200 import replicas
    return replicas.init("nccl")


def barrier(ws):
    from research_b200 import replicas
    replicas.barrier(ws)


def max_over_ranks(ws, x: float) -> float:
    from research_b200 import replicas
    return replicas.max_over_ranks(ws, x, "cuda")


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """DRAM bytes of `kernel` over one frame (its launches summed, ncu with cold
    caches) from the committed ncu summary, if any."""
    f = ROOT / "profiles" / f"{kernel}_traffic.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith(f"dram_bytes_per_frame_{kernel}:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        u = str(uuid)
        self.device = u if u.startswith("GPU-") else f"GPU-{u}"
        self.rows = []
        self._stop = threading.Event()
        self._th = None

    def mark(self):
        """Only samples taken from now on are reported."""
        self.first = len(self.rows)

    def start(self):
        self.first = 0
        def run():
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.rows.append([x.strip() for x in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)
        self._th = threading.Thread(target=run, daemon=True)
        self._th.start()

    def stop(self):
        self._stop.set()
        if self._th:
            self._th.join(timeout=10)
        rows = self.rows[self.first:] or self.rows[-1:]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def build_scene(rr, args):
    hs = rr.HostScene.procedural(seed=CFG["scene_seed"], target_triangles=args.triangles,
                                 emissive_triangles=CFG["emitters"], box_half=CFG["box_half"])
    return hs


# ─────────────────────────────── reference arm ──────────────────────────────
def cpu_frame_sample(O, rr, oscene, args, budget_s: float, nthreads: int, L=None):
    """Times the oracle (CPU restatement of the reference passes) on a centre
    crop of the same frame (PT 4 spp + accumulate + DI + A-trous), repeating
    until `budget_s` of work; returns (Mpaths/s, description, seconds).
    `L` is the library whose camera helpers build the camera blocks."""
    import numpy as np
    W, H = args.width, args.height
    cw, ch = min(256, W), min(256, H)
    x0, y0 = (W - cw) // 2, (H - ch) // 2
    cam_full = rr.camera_data(rr.camera_desc(W, H, eye=CFG["eye"], center=CFG["center"], L=L), L=L)
    cam_crop = rr.camera_data(rr.camera_desc(cw, ch, eye=CFG["eye"], center=CFG["center"], L=L), L=L)
    acc = np.zeros((ch, cw, 4), np.float32)
    z = lambda: np.zeros((ch, cw, 4), np.float32)
    gpos, gnrm, res, prev, out = z(), z(), z(), z(), z()
    paths = 0
    frames = 0
    t0 = time.perf_counter()
    while True:
        img, _ = O.pathtrace(oscene, cam_full, frames * CFG["spp"], CFG["max_bounces"], CFG["spp"],
                             region=(x0, y0, cw, ch), nthreads=nthreads)
        for k in range(CFG["spp"]):
            O.accumulate(np.ascontiguousarray(img[k]), acc, 1 if (frames == 0 and k == 0) else 0,
                         frames * CFG["spp"] + k)
        p = O.di_params(frames, CFG["di_candidates"], 1, 1, CFG["di_neighbors"], CFG["di_radius"],
                        CFG["m_cap_factor"])
        O.restir_di_initial(oscene, cam_crop, p, gpos, gnrm, res, nthreads)
        O.restir_di_temporal(oscene, cam_crop, p, gpos, gnrm, res, prev, nthreads)
        O.restir_di_spatial_shade(oscene, cam_crop, p, gpos, gnrm, res, out, nthreads)
        O.atrous(out, gpos, gnrm, CFG["atrous_iterations"])
        res, prev = prev, res
        paths += cw * ch * CFG["spp"]
        frames += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    desc = (f"oracle port, {cw}x{ch} centre crop of the 1920x1080 frame, {frames} frame(s) of PT {CFG['spp']} spp "
            f"+ accumulate + ReSTIR DI + A-trous ({dt:.1f} s, {nthreads} threads)")
    return paths / dt / 1e6, desc, dt


def run_reference(args, ws, rank):
    """The reference arm: the CPU restatement of the reference passes (the
    reference itself cannot run here) on the host cores. Its scene and camera
    come from oracle/librr_inputs.so, the same seeded generators built
    without CUDA: this arm loads no library of the GPU path. A step is one
    bounded sample of the workload (centre-crop frames for a fixed time);
    ms_per_step is that step's measured duration."""
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    from research_b200 import build
    build.build_oracle()
    from research_b200 import rr   # ctypes layouts only; librr_cuda.so is not loaded
    import oracle as O
    inputs = O.inputs_lib()
    hs = rr.HostScene.procedural(seed=CFG["scene_seed"], target_triangles=args.triangles,
                                 emissive_triangles=CFG["emitters"], box_half=CFG["box_half"], L=inputs)
    oscene = O.OracleScene(hs.arrays, use_bvh=True)
    nth = O.threads()
    per_step = max(2.0, min(30.0, 120.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_frame_sample(O, rr, oscene, args, 0.5, nth, L=inputs)
    vals, descs, secs = [], [], []
    for _ in range(args.steps):
        v, d, dt = cpu_frame_sample(O, rr, oscene, args, per_step, nth, L=inputs)
        vals.append(v)
        descs.append(d)
        secs.append(dt)
    oscene.close()
    value = statistics.median(vals)
    full_ms = args.width * args.height * CFG["spp"] / (value * 1e6) * 1e3
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.mean(secs) * 1e3,
            "step": f"one bounded sample: centre-crop frames of the workload for about {per_step:.1f} s",
            "full_frame_ms_extrapolated": full_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(args),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nth, "kind": "port", "sample": descs[-1]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_dict(args):
    return {"workload": WORKLOAD, "width": args.width, "height": args.height, "spp": CFG["spp"],
            "max_bounces": CFG["max_bounces"], "triangles": args.triangles, "emissive_triangles": CFG["emitters"],
            "restir_di": {"candidates": CFG["di_candidates"], "m_cap": CFG["m_cap_factor"] * CFG["di_candidates"],
                          "neighbors": CFG["di_neighbors"], "radius_px": CFG["di_radius"]},
            "atrous_iterations": CFG["atrous_iterations"], "parallelism": f"replicas{args.gpus}",
            "pass_schedule": ("one stream; A-trous strides 1-4 through TMA-staged tiles" if args.serial_passes else
                              "ReSTIR DI + A-trous (direct loads) on a second stream beside path tracer + accumulate"),
            "l2": "per-step working set (ray queues + images) > 126 MB L2; no explicit flush"}


# ───────────────────────────────── our arm ──────────────────────────────────
class Frame:
    """One config frame through the C ABI on device buffers."""

    def __init__(self, rr, torch, ctx, scene, W, H):
        self.rr, self.torch, self.ctx, self.scene = rr, torch, ctx, scene
        self.W, self.H = W, H
        self.L = rr.lib()
        f = lambda *s: torch.zeros(s, device="cuda", dtype=torch.float32)
        self.rad = f(CFG["spp"], H, W, 4)
        self.acc = f(H, W, 4)
        self.gpos, self.gnrm, self.out = f(H, W, 4), f(H, W, 4), f(H, W, 4)
        self.res = [f(H, W, 4), f(H, W, 4)]
        self.ping = [f(H, W, 4), f(H, W, 4)]
        self.frame = 0
        self.spp_acc = 0
        self.pt_mode = 0      # RR_PT_FLAG_EMITTERS for the emitter-sampling frame
        self.di_flags = 0     # RR_DI_FLAG_EMITTERS likewise
        self.slot = C.c_uint32()
        self.desc = rr.camera_desc(W, H, eye=CFG["eye"], center=CFG["center"])
        self.cam = rr.camera_data(self.desc)
        self.stage_events = []
        # ReSTIR DI and A-trous do not read the path tracer's or the
        # accumulation's buffers (nor they theirs): with `concurrent`, they run
        # on a second stream that forks from the frame's stream at the start
        # of the step and joins it at the end
        self.concurrent = False
        self.di_stream = torch.cuda.Stream()
        self.fork, self.join = torch.cuda.Event(), torch.cuda.Event()

    def step(self, stream, pt_flags=0, seed_base=0, stage_timing=False):
        rr, L, ctx = self.rr, self.L, self.ctx
        cam = self.cam
        ev = []
        mark = (lambda: ev.append(self.torch.cuda.Event(enable_timing=True))) if stage_timing else (lambda: None)
        rec = (lambda: ev[-1].record()) if stage_timing else (lambda: None)
        fork = self.concurrent and not stage_timing
        di_st = stream
        if fork:
            main = self.torch.cuda.current_stream()
            self.fork.record(main)
            self.di_stream.wait_event(self.fork)
            di_st = self.di_stream.cuda_stream
        mark(); rec()
        p = rr.PtParams(seed_base + self.frame * CFG["spp"], CFG["max_bounces"], CFG["spp"], pt_flags | self.pt_mode)
        ctx.check(L.rr_pathtracer_execute(ctx.handle, self.scene.handle, C.byref(cam), C.byref(p),
                                          self.rad.data_ptr(), stream))
        mark(); rec()
        ap = rr.AccParams(self.W, self.H, 1 if self.spp_acc == 0 else 0, self.spp_acc)
        ctx.check(L.rr_accumulate_execute(ctx.handle, self.rad.data_ptr(), CFG["spp"], self.acc.data_ptr(), None,
                                          C.byref(ap), stream))
        self.spp_acc += CFG["spp"]
        mark(); rec()
        dp = rr.DIParams(seed_base + self.frame, CFG["di_candidates"], 1, 1, CFG["di_neighbors"], CFG["di_radius"],
                         CFG["m_cap_factor"], self.di_flags)
        cur, prev = self.res[self.frame & 1], self.res[(self.frame & 1) ^ 1]
        ctx.check(L.rr_restir_di_execute(ctx.handle, self.scene.handle, C.byref(cam), C.byref(dp),
                                         self.gpos.data_ptr(), self.gnrm.data_ptr(), cur.data_ptr(), prev.data_ptr(),
                                         self.out.data_ptr(), di_st))
        mark(); rec()
        atp = rr.AtrousParams(self.W, self.H, CFG["atrous_iterations"], 0, 0.25, 0.20, 1.0, 0)
        ctx.check(L.rr_atrous_execute(ctx.handle, self.out.data_ptr(), self.gpos.data_ptr(), self.gnrm.data_ptr(),
                                      self.ping[0].data_ptr(), self.ping[1].data_ptr(), C.byref(atp),
                                      C.byref(self.slot), di_st))
        if fork:
            self.join.record(self.di_stream)
            main.wait_event(self.join)
        mark(); rec()
        if stage_timing:
            self.stage_events.append(ev)
        self.frame += 1

    def denoised(self):
        return self.ping[self.slot.value]

    def stage_ms(self):
        self.torch.cuda.synchronize()
        names = ["pathtracer", "accumulate", "restir_di", "atrous"]
        tot = {n: 0.0 for n in names}
        for ev in self.stage_events:
            for k, n in enumerate(names):
                tot[n] += ev[k].elapsed_time(ev[k + 1])
        cnt = max(1, len(self.stage_events))
        return {n: v / cnt for n, v in tot.items()}


def parity_check(rr, O, torch, ctx, scene, oscene, args, frame_index, seed_base, concurrent, pt_mode=0, di_flags=0):
    """The benchmarked frame against the oracle, outside the timed region:
    two frames rendered exactly as the timed loop renders them (fresh
    reservoirs; the second frame uses the first timed frame's seeds). The
    path tracer's 4 images and the accumulated image are compared on the
    256x256 centre crop (the oracle traces that region of the same camera
    with the same frame seeds); the ReSTIR DI G-buffer and output and the
    A-trous output on the whole 1920x1080 frame. Tolerance zero: every
    compared float must have the same bits. pt_mode / di_flags: the
    emitter-sampling frame's RR_PT_FLAG_EMITTERS / RR_DI_FLAG_EMITTERS."""
    import numpy as np
    W, H = args.width, args.height
    spp = CFG["spp"]
    cw, ch = min(256, W), min(256, H)
    x0, y0 = (W - cw) // 2, (H - ch) // 2
    t0 = time.perf_counter()
    pf = Frame(rr, torch, ctx, scene, W, H)
    pf.concurrent = concurrent
    pf.pt_mode, pf.di_flags = pt_mode, di_flags
    pf.frame = frame_index - 1
    stream = torch.cuda.current_stream().cuda_stream
    frames = [pf.frame, pf.frame + 1]
    rad_crops = []
    for _ in frames:
        pf.step(stream, seed_base=seed_base)
        torch.cuda.synchronize()
        rad_crops.append(pf.rad[:, y0:y0 + ch, x0:x0 + cw].contiguous().cpu().numpy())
    g_acc = pf.acc[y0:y0 + ch, x0:x0 + cw].contiguous().cpu().numpy()
    g_pos, g_nrm, g_out = pf.gpos.cpu().numpy(), pf.gnrm.cpu().numpy(), pf.out.cpu().numpy()
    g_den = pf.denoised().cpu().numpy()
    t_gpu = time.perf_counter() - t0

    cam = pf.cam
    o_acc = np.zeros((ch, cw, 4), np.float32)
    mism = {}
    nth = O.threads()
    for j, f in enumerate(frames):
        img, _ = O.pathtrace(oscene, cam, seed_base + f * spp, CFG["max_bounces"], spp,
                             region=(x0, y0, cw, ch), nthreads=nth, flags=O.PT_EMITTERS if pt_mode else 0)
        for k in range(spp):
            O.accumulate(np.ascontiguousarray(img[k]), o_acc, 1 if (j == 0 and k == 0) else 0, j * spp + k)
        mism[f"pathtracer_frame{j}"] = int((img.view(np.uint32) != rad_crops[j].view(np.uint32)).any(-1).sum())
    mism["accumulated"] = int((o_acc.view(np.uint32) != g_acc.view(np.uint32)).any(-1).sum())
    z = lambda: np.zeros((H, W, 4), np.float32)
    gpos, gnrm, out = z(), z(), z()
    res = [z(), z()]
    for j, f in enumerate(frames):
        dp = O.di_params(seed_base + f, CFG["di_candidates"], 1, 1, CFG["di_neighbors"], CFG["di_radius"],
                         CFG["m_cap_factor"], flags=O.DI_EMITTERS if di_flags else 0)
        cur, prev = res[f & 1], res[(f & 1) ^ 1]
        O.restir_di_initial(oscene, cam, dp, gpos, gnrm, cur, nth)
        O.restir_di_temporal(oscene, cam, dp, gpos, gnrm, cur, prev, nth)
        O.restir_di_spatial_shade(oscene, cam, dp, gpos, gnrm, cur, out, nth)
    den = O.atrous(out, gpos, gnrm, CFG["atrous_iterations"])
    for name, a, b in (("gbuffer_pos", gpos, g_pos), ("gbuffer_normal", gnrm, g_nrm), ("restir_di_output", out, g_out),
                       ("atrous_output", den, g_den)):
        mism[name] = int((a.view(np.uint32) != b.view(np.uint32)).any(-1).sum())
    return {"bit_exact": all(v == 0 for v in mism.values()), "mismatched_pixels": mism,
            "pathtracer_and_accumulate": f"{cw}x{ch} centre crop at ({x0},{y0}), {spp} spp per frame",
            "restir_di_and_atrous": f"full {W}x{H} frame", "frames": 2,
            "seeds": f"path tracer frame seeds {seed_base + frames[0] * spp}..{seed_base + frames[1] * spp + spp - 1}, "
                     f"DI frame seeds {seed_base + frames[0]}, {seed_base + frames[1]} (the second frame is the "
                     f"first timed frame)",
            "gpu_s": round(t_gpu, 2), "oracle_s": round(time.perf_counter() - t0 - t_gpu, 2), "oracle_threads": nth}


def run_ours(args, ws, rank, local):
    import torch
    from research_b200 import rr
    torch.cuda.set_device(local)
    ctx = rr.Context(local)
    hs = build_scene(rr, args)
    scene = rr.Scene(ctx, hs.arrays)
    sst = scene.stats()
    W, H = args.width, args.height
    stream = torch.cuda.current_stream().cuda_stream
    fr = Frame(rr, torch, ctx, scene, W, H)
    fr.concurrent = not args.serial_passes
    # A-trous beside the path tracer uses direct loads: its TMA-staged tiles
    # need shared memory on the SMs whose traversal blocks run on a full L1
    # (measured: 37.6 ms per frame with the tiles, 35.8 with direct loads)
    ctx.check(rr.lib().rr_atrous_set_tma(ctx.handle, 0 if fr.concurrent else 1))
    from research_b200 import replicas
    seed_base = replicas.seed_base(rank)
    replicas.check_seed_budget((args.warmup + 3 * args.steps + 8) * CFG["spp"])

    st = rr.PtStats()
    # autotune the traversal variants on this scene and frame (setup, untimed)
    if args.variants:
        ev, sv = (int(x) for x in args.variants.split(","))
        ctx.check(rr.lib().rr_pathtracer_set_variants(ctx.handle, ev, sv))
        tuned = {"extend_variant": ev, "shadow_variant": sv, "fixed": True}
    else:
        tune = rr.PtTuneResult()
        ctx.check(rr.lib().rr_pathtracer_tune(ctx.handle, scene.handle, C.byref(fr.cam),
                                              C.byref(rr.PtParams(seed_base, CFG["max_bounces"], CFG["spp"], 0)),
                                              fr.rad.data_ptr(), stream, C.byref(tune)))
        tuned = {"extend_variant": tune.best_extend, "shadow_variant": tune.best_shadow,
                 "extend_ms": [round(x, 3) for x in tune.extend_ms],
                 "shadow_ms": [round(x, 3) for x in tune.shadow_ms]}
    clocks = ClockSampler(torch.cuda.get_device_properties(local).uuid)
    clocks.start()
    # 1) warm-up
    for _ in range(args.warmup):
        fr.step(stream, seed_base=seed_base)
    torch.cuda.synchronize()
    ctx.check(rr.lib().rr_pathtracer_stats(ctx.handle, C.byref(st), 1))
    launches0 = st.launches_total
    # 2) timed region: K device-resident steps (the path tracer overlaps each
    #    bounce's shadow rays with the next bounce's extension rays)
    first_timed = fr.frame
    barrier(ws)
    torch.cuda.synchronize()
    clocks.mark()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        fr.step(stream, seed_base=seed_base)
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(ws)
    ms_total = e0.elapsed_time(e1)
    ms_step = max_over_ranks(ws, ms_total / args.steps)
    ctx.check(rr.lib().rr_pathtracer_stats(ctx.handle, C.byref(st), 1))
    launches = st.launches_total - launches0

    # 2b) stage times: the same K frames again, each stage timed alone with
    #     CUDA events on one stream (untimed as a whole)
    fr.frame = first_timed
    for _ in range(args.steps):
        fr.step(stream, pt_flags=rr.PT_FLAG_TIME_STAGES, seed_base=seed_base, stage_timing=True)
    torch.cuda.synchronize()
    ctx.check(rr.lib().rr_pathtracer_stats(ctx.handle, C.byref(st), 1))
    stage = fr.stage_ms()
    pt_stage = {"raygen": st.ms_raygen / args.steps, "extend": st.ms_extend / args.steps,
                "shade": st.ms_shade / args.steps, "shadow": st.ms_shadow / args.steps}
    paths_per_step = W * H * CFG["spp"]
    value = replicas.job_throughput(paths_per_step, ws, ms_step)

    # 3) algorithmic work of the timed frames: replay the same K frame seeds
    #    with traversal counters on (untimed; the kernels are deterministic)
    keys = ("extension_rays", "shadow_rays", "extension_nodes", "extension_tris", "shadow_nodes", "shadow_tris")
    counted = {k: 0 for k in keys}
    fr.frame = first_timed
    for _ in range(args.steps):
        fr.step(stream, pt_flags=rr.PT_FLAG_COUNT_TRAVERSAL, seed_base=seed_base)
        ctx.check(rr.lib().rr_pathtracer_stats(ctx.handle, C.byref(st), 1))
        for k in keys:
            counted[k] += getattr(st, k)
    counted = {k: v // args.steps for k, v in counted.items()}

    # 4) e2e through the public API with host buffers: the per-frame input is
    #    the host GpuCameraData block, handed to rr_pathtracer_execute and
    #    rr_restir_di_execute (the library forwards it in launch parameters);
    #    the frame's results, the accumulated and the denoised images, are read
    #    back into pinned host memory every step. The read-back is pipelined as
    #    a renderer's presentation path would be: each frame's two images are
    #    snapshot on the compute stream into one of two device slots, and a
    #    second stream copies that slot to its pinned host pair while the next
    #    frame renders; a slot is reused only after its copy has finished, and
    #    the timed region ends after the last copy.
    compute = torch.cuda.current_stream()
    copier = torch.cuda.Stream()
    snap = [[torch.empty((H, W, 4), device="cuda") for _ in range(2)] for _ in range(2)]
    host = [[torch.empty((H, W, 4), dtype=torch.float32).pin_memory() for _ in range(2)] for _ in range(2)]
    snapped = [torch.cuda.Event() for _ in range(2)]
    copied = [torch.cuda.Event() for _ in range(2)]
    h2d = 2 * C.sizeof(rr.GpuCameraData)
    d2h = 2 * H * W * 16
    barrier(ws)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(compute)
    for k in range(args.steps):
        j = k & 1
        fr.cam = rr.camera_data(fr.desc)
        fr.step(stream, seed_base=seed_base)
        if k >= 2:
            compute.wait_event(copied[j])
        snap[j][0].copy_(fr.acc, non_blocking=True)
        snap[j][1].copy_(fr.denoised(), non_blocking=True)
        snapped[j].record(compute)
        copier.wait_event(snapped[j])
        with torch.cuda.stream(copier):
            host[j][0].copy_(snap[j][0], non_blocking=True)
            host[j][1].copy_(snap[j][1], non_blocking=True)
            copied[j].record(copier)
    compute.wait_stream(copier)
    f1.record(compute)
    torch.cuda.synchronize()
    # the last frame's images arrived intact
    last = (args.steps - 1) & 1
    if not (torch.equal(host[last][0], fr.acc.cpu()) and torch.equal(host[last][1], fr.denoised().cpu())):
        raise RuntimeError("pipelined read-back does not match the device images")
    e2e_ms = max_over_ranks(ws, f0.elapsed_time(f1) / args.steps)
    e2e_value = replicas.job_throughput(paths_per_step, ws, e2e_ms)

    # roofline of the dominant kernel (BVH traversal of extension rays)
    peak, peak_kind = load_peaks()
    node_bytes = {k: NODE_BYTES * rr.lib().rr_pathtracer_variant_width(tuned[k + "_variant"]) // 2
                  for k in ("extend", "shadow")}
    ext_bytes = (counted["extension_rays"] * RAY_BYTES + counted["extension_nodes"] * node_bytes["extend"] +
                 counted["extension_tris"] * TRI_BYTES)
    ext_ms = pt_stage["extend"]
    shadow_bytes = (counted["shadow_rays"] * RAY_BYTES + counted["shadow_nodes"] * node_bytes["shadow"] +
                    counted["shadow_tris"] * TRI_BYTES)
    achieved = ext_bytes / (ext_ms * 1e-3) / 1e9 if ext_ms > 0 else 0.0
    # DRAM bytes are not measured in this run (that needs ncu): the figure of
    # the committed ncu capture of the same frame is reported beside the
    # roofline, labelled as such, and `traffic` stays null
    prof = ncu_traffic("extend")
    from_profile = None
    if prof is not None:
        per_launch = prof / CFG["max_bounces"]
        dram_gbs = prof / (ext_ms * 1e-3) / 1e9 if ext_ms > 0 else 0.0
        from_profile = {"dram_bytes_per_launch": per_launch, "dram_gbs": dram_gbs, "dram_frac": dram_gbs / peak,
                        "source": "ncu capture of one frame's extend launches, summarised in "
                                  "profiles/extend_traffic.txt; not measured in this run"}
    roofline = {"kernel": "extend_kernel (closest-hit BVH traversal, all bounces of one frame)",
                "bound": "latency (L1/L2-served node fetches, SIMT divergence)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": f"{peak_kind} hbm_gbs", "traffic": None, "from_profile": from_profile,
                "achieved_scope": "algorithmic bytes (rays, BVH nodes and triangles the traversal touches, counted by "
                                  "the kernel) per second of extend time; most are served by L1/L2, not HBM",
                "algorithmic_bytes_per_step": ext_bytes, "launches_per_step": CFG["max_bounces"],
                "node_bytes": node_bytes,
                "shadow_achieved_gbs": shadow_bytes / (pt_stage["shadow"] * 1e-3) / 1e9 if pt_stage["shadow"] else 0}
    rays = counted["extension_rays"] + counted["shadow_rays"]

    cpu = None
    parity = None
    if rank == 0 and not (args.no_cpu_baseline and args.no_parity):
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O
        oscene = O.OracleScene(hs.arrays, use_bvh=True)
        if not args.no_parity:
            parity = parity_check(rr, O, torch, ctx, scene, oscene, args, first_timed, seed_base, fr.concurrent)
        if ws == 1 and not args.no_cpu_baseline:
            v, d, _ = cpu_frame_sample(O, rr, oscene, args, args.cpu_seconds, O.threads())
            cpu = {"value": v, "unit": UNIT, "cores": O.threads(), "kind": "port", "sample": d}
        oscene.close()

    # the same frame lit by its emissive triangles alone (no centroid point
    # lights), with the path tracer and ReSTIR DI sampling the triangles
    # (RR_PT_FLAG_EMITTERS, RR_DI_FLAG_EMITTERS); device-timed like the main
    # frames, reported beside them
    emitter_mode = None
    if not args.no_emitter_mode:
        hs_e = rr.HostScene.procedural(seed=CFG["scene_seed"], target_triangles=args.triangles,
                                       emissive_triangles=CFG["emitters"], box_half=CFG["box_half"],
                                       flags=rr.SCENE_NO_EMITTER_LIGHTS)
        scene_e = rr.Scene(ctx, hs_e.arrays)
        fe = Frame(rr, torch, ctx, scene_e, W, H)
        fe.concurrent = fr.concurrent
        fe.pt_mode, fe.di_flags = rr.PT_FLAG_EMITTERS, rr.DI_FLAG_EMITTERS
        for _ in range(args.warmup):
            fe.step(stream, seed_base=seed_base)
        first_timed_e = fe.frame
        barrier(ws)
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record()
        for _ in range(args.steps):
            fe.step(stream, seed_base=seed_base)
        g1.record()
        torch.cuda.synchronize()
        em_ms = max_over_ranks(ws, g0.elapsed_time(g1) / args.steps)
        fe.frame = args.warmup
        for _ in range(args.steps):
            fe.step(stream, pt_flags=rr.PT_FLAG_TIME_STAGES, seed_base=seed_base, stage_timing=True)
        ctx.check(rr.lib().rr_pathtracer_stats(ctx.handle, C.byref(st), 1))
        em_stage = fe.stage_ms()
        em_parity = None
        if rank == 0 and not args.no_parity:
            sys.path.insert(0, str(ROOT / "oracle"))
            import oracle as O
            osc_e = O.OracleScene(hs_e.arrays, use_bvh=True)
            em_parity = parity_check(rr, O, torch, ctx, scene_e, osc_e, args, first_timed_e, seed_base, fr.concurrent,
                                     pt_mode=rr.PT_FLAG_EMITTERS, di_flags=rr.DI_FLAG_EMITTERS)
            osc_e.close()
        emitter_mode = {"value": replicas.job_throughput(paths_per_step, ws, em_ms), "unit": UNIT,
                        "ms_per_step": em_ms,
                        "workload": "the same frame on the same scene without its centroid point lights: the path "
                                    "tracer's NEE and ReSTIR DI's candidates sample the 4096 emissive triangles "
                                    "(RR_PT_FLAG_EMITTERS, RR_DI_FLAG_EMITTERS)",
                        "parity": em_parity,
                        "stages_ms": {**{k: round(v, 4) for k, v in em_stage.items()},
                                      "pt_extend": round(st.ms_extend / args.steps, 4),
                                      "pt_shade": round(st.ms_shade / args.steps, 4),
                                      "pt_shadow": round(st.ms_shadow / args.steps, 4)}}
        del fe
        scene_e.close()

    # the metric's second half: time to a relative RMSE of 1e-2, learned vs
    # grid guiding (and unguided), on the same scene, one GPU
    rmse = None
    if rank == 0 and ws == 1 and not args.no_time_to_rmse:
        import bench_guiding
        rclocks = ClockSampler(torch.cuda.get_device_properties(local).uuid)
        rclocks.start()
        r = bench_guiding.measure(rr, torch, ctx, scene, budget_s=args.rmse_budget_s, repeats=args.rmse_repeats)
        r["clocks"] = rclocks.stop()
        for rs in r["runs"].values():
            for x in rs:
                x.pop("curve", None)
        rmse = {"metric": "time to relative RMSE 1e-2 (learned vs vMF-grid guiding vs unguided)",
                "workload": "procedural-room-1M-tris, 64x64 centre crop of the 1920x1080 view "
                            "(Application::compute_mse's region), 256 spp per frame, 5 bounces",
                "grid": "64^3 cells x 8 vMF lobes, FP64 EM statistics, decay 0.9, alpha 0.5",
                "mlp": "80-64x4-48 BF16 tcgen05 MLP, Adam lr 1e-2, 2^18 samples per frame, alpha 0.5", **r}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
                "config": config_dict(args),
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "ms_per_step": e2e_ms},
                "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu, "parity": parity, "clocks": clk,
                "stages_ms": {**{k: round(v, 4) for k, v in stage.items()},
                              "pt_" + "raygen": round(pt_stage["raygen"], 4),
                              "pt_extend": round(pt_stage["extend"], 4), "pt_shade": round(pt_stage["shade"], 4),
                              "pt_shadow": round(pt_stage["shadow"], 4),
                              "scope": "each stage timed alone on one stream, same frames; the timed frames run "
                                       "each bounce's shadow launch beside the next bounce's extend launch"},
                "rays_per_step": rays, "mrays_per_s": rays / (ms_step * 1e-3) / 1e6,
                "stage_mrays_per_s": {
                    "extend": counted["extension_rays"] / (pt_stage["extend"] * 1e-3) / 1e6 if pt_stage["extend"] else 0,
                    "shadow": counted["shadow_rays"] / (pt_stage["shadow"] * 1e-3) / 1e6 if pt_stage["shadow"] else 0},
                "scene": {"triangles": sst.triangle_count, "bvh_nodes": sst.bvh_node_count,
                          "bvh_depth": sst.bvh_max_depth, "bvh_build_ms": round(sst.build_ms, 1),
                          "lights": sst.light_count},
                "traversal_per_step": counted, "autotune": tuned, "emitter_mode": emitter_mode, "time_to_rmse": rmse}
        print(json.dumps(line), flush=True)
    scene.close()
    ctx.close()


def main():
    args = parse()
    ws, rank, local = dist_init(args)
    if args.impl == "reference":
        run_reference(args, ws, rank)
    else:
        from research_b200 import build
        if not (ROOT / "research_b200" / "lib" / "librr_cuda.so").exists():
            build.build_cuda()
        run_ours(args, ws, rank, local)
    from research_b200 import replicas
    replicas.finish(ws)


if __name__ == "__main__":
    main()
