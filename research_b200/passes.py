"""Python mirror of the reference's pass classes and headless Application.

Same names, public tuning fields and frame bookkeeping as the reference's
C++ passes (src/passes/*) and rr::app::Application (src/app/Application.h),
driving librr_cuda.so through its C ABI. Images are CUDA torch tensors
(H x W x 4 float32), the equivalent of the reference's RGBA32F storage images.
Windowing, ImGui, swapchain and the raster G-buffer are not part of this
build: the G-buffer comes from ReSTIR DI's primary rays (restir_di.slang:
208-223), as in the reference.
"""
from __future__ import annotations

import ctypes as C
import struct
import zlib
from pathlib import Path

from . import rr


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


class PathTracerPass:
    """PathTracerPass (PathTracerPass.h:22-67): one path per pixel per frame."""
    name = "PathTracerPass"

    def __init__(self, ctx, extent):
        import torch
        self.ctx, self.torch = ctx, torch
        self.width, self.height = extent
        self.max_bounces = 5            # PathTracerPass.h:46
        self.frame_count = 0            # frame_seed = frame_count_++ (PathTracerPass.cpp:215)
        self.enabled = True
        self.radiance = torch.zeros((1, self.height, self.width, 4), device="cuda")

    def execute(self, scene, camera):
        p = rr.PtParams(self.frame_count, self.max_bounces, 1, 0)
        self.frame_count += 1
        self.ctx.check(rr.lib().rr_pathtracer_execute(self.ctx.handle, scene.handle, C.byref(camera), C.byref(p),
                                                      self.radiance.data_ptr(), _stream(self.torch)))


class AccumulatePass:
    """AccumulatePass (AccumulatePass.h): FP32 running mean, reset on camera move."""
    name = "AccumulatePass"

    def __init__(self, ctx, extent):
        import torch
        self.ctx, self.torch = ctx, torch
        self.width, self.height = extent
        self.camera_moved = False
        self.accumulated_spp = 0
        self.enabled = True
        self.accumulated = torch.zeros((self.height, self.width, 4), device="cuda")

    def execute(self, radiance):
        p = rr.AccParams(self.width, self.height, 1 if self.camera_moved else 0, self.accumulated_spp)
        self.ctx.check(rr.lib().rr_accumulate_execute(self.ctx.handle, radiance.data_ptr(), 1,
                                                      self.accumulated.data_ptr(), None, C.byref(p),
                                                      _stream(self.torch)))
        # AccumulatePass.cpp:211-217
        self.accumulated_spp = 1 if self.camera_moved else self.accumulated_spp + 1
        self.camera_moved = False


class ReSTIRDIPass:
    """ReSTIRDIPass (ReSTIRDIPass.h): initial / temporal / spatial+shade."""
    name = "ReSTIRDIPass"

    def __init__(self, ctx, extent):
        import torch
        self.ctx, self.torch = ctx, torch
        self.width, self.height = extent
        self.temporal_enable = True      # ReSTIRDIPass.h:89-93
        self.spatial_enable = True
        self.num_initial_candidates = 16
        self.spatial_num_neighbors = 4
        self.spatial_radius = 15
        self.m_cap_factor = 20           # restir_di.slang:300
        self.enabled = False
        z = lambda: torch.zeros((self.height, self.width, 4), device="cuda")
        self.gbuf_pos, self.gbuf_norm, self.output = z(), z(), z()
        self.reservoirs = [z(), z()]
        self.reset_history()

    def reset_history(self):
        """ReSTIRDIPass.h:80-85"""
        self.reservoir_flip = 0
        self.frame_count = 0
        for r in self.reservoirs:
            r.zero_()

    def execute(self, scene, camera):
        p = rr.DIParams(self.frame_count, self.num_initial_candidates, int(self.temporal_enable),
                        int(self.spatial_enable), self.spatial_num_neighbors, self.spatial_radius,
                        self.m_cap_factor, 0)
        self.frame_count += 1
        cur = self.reservoirs[self.reservoir_flip]
        prev = self.reservoirs[1 - self.reservoir_flip]
        self.ctx.check(rr.lib().rr_restir_di_execute(self.ctx.handle, scene.handle, C.byref(camera), C.byref(p),
                                                     self.gbuf_pos.data_ptr(), self.gbuf_norm.data_ptr(),
                                                     cur.data_ptr(), prev.data_ptr(), self.output.data_ptr(),
                                                     _stream(self.torch)))
        self.reservoir_flip ^= 1


class ReSTIRGIPass:
    """ReSTIRGIPass (ReSTIRGIPass.h:67-74 defaults): initial / temporal /
    spatial+shade over the G-buffer, with ReSTIR DI's output as direct light."""
    name = "ReSTIRGIPass"

    def __init__(self, ctx, extent):
        import torch
        self.ctx, self.torch = ctx, torch
        self.width, self.height = extent
        self.include_direct_lighting = True
        self.temporal_enable = True
        self.spatial_enable = True
        self.indirect_strength = 1.0
        self.ray_bias = 1.0e-3
        self.num_initial_candidates = 8
        self.spatial_num_neighbors = 4
        self.spatial_radius = 12
        self.enabled = False
        z = lambda: torch.zeros((self.height, self.width, 4), device="cuda")
        self.reservoirs = [[z() for _ in range(3)] for _ in range(2)]
        self.history = [[z() for _ in range(2)] for _ in range(2)]
        self.output = z()
        for h in self.history:   # pre_transition_to_general's first clear (ReSTIRGIPass.cpp:383-399)
            h[0][..., 3] = -1.0
        self.reset_history()

    def reset_history(self):
        """ReSTIRGIPass.h:54-59"""
        self.reservoir_flip = 0
        self.frame_count = 0
        self.history_dirty = True

    def execute(self, scene, camera, gbuf_pos, gbuf_norm, direct):
        p = rr.gi_reuse_params(self.frame_count, self.num_initial_candidates, int(self.temporal_enable),
                               int(self.spatial_enable), self.spatial_num_neighbors, self.spatial_radius,
                               int(self.include_direct_lighting), self.indirect_strength, self.ray_bias)
        self.frame_count += 1
        c, v = self.reservoir_flip, 1 - self.reservoir_flip
        im = rr.GiReuseImages()
        im.gbuf_pos, im.gbuf_norm = gbuf_pos.data_ptr(), gbuf_norm.data_ptr()
        im.direct = direct.data_ptr() if (self.include_direct_lighting and direct is not None) else None
        for k in range(3):
            im.reservoir_curr[k], im.reservoir_prev[k] = self.reservoirs[c][k].data_ptr(), self.reservoirs[v][k].data_ptr()
        for k in range(2):
            im.history_curr[k], im.history_prev[k] = self.history[c][k].data_ptr(), self.history[v][k].data_ptr()
        im.output = self.output.data_ptr()
        L, st = rr.lib(), _stream(self.torch)
        if self.history_dirty:   # consume_history_dirty (ReSTIRGIPass.cpp:484-530)
            self.history_dirty = False
            self.ctx.check(L.rr_restir_gi_reset_history(self.ctx.handle, C.byref(im), self.width, self.height, st))
        self.ctx.check(L.rr_restir_gi_execute(self.ctx.handle, scene.handle, C.byref(camera), C.byref(p),
                                              C.byref(im), st))
        self.reservoir_flip ^= 1


class ReSTIRPTPass:
    """ReSTIRPTPass (ReSTIRPTPass.h:82-99 defaults): initial / temporal /
    spatial+shade with the reconnection shift, and the vMF guiding grid."""
    name = "ReSTIRPTPass"
    kGridCellCount = 1 << 20

    def __init__(self, ctx, extent):
        import torch
        self.ctx, self.torch = ctx, torch
        self.width, self.height = extent
        self.include_direct_lighting = True
        self.temporal_enable = True
        self.spatial_enable = True
        self.indirect_strength = 1.0
        self.ray_bias = 1.0e-3
        self.num_initial_candidates = 8
        self.max_bounces = 4
        self.spatial_num_neighbors = 4
        self.spatial_radius = 12
        self.guiding_enable = True
        self.guiding_alpha = 0.5
        self.grid_base_cell_size = 0.10
        self.grid_distance_slope = 0.02
        self.grid_min_samples = 8
        self.grid_kappa_max = 512.0
        self.enabled = False
        z = lambda: torch.zeros((self.height, self.width, 4), device="cuda")
        self.reservoirs = [[z() for _ in range(4)] for _ in range(2)]
        self.history = [[z() for _ in range(2)] for _ in range(2)]
        self.output = z()
        for h in self.history:
            h[0][..., 3] = -1.0
        self.guiding_accum = torch.zeros((self.kGridCellCount, 4), dtype=torch.int32, device="cuda")
        self.guiding_fitted = torch.zeros((self.kGridCellCount, 4), device="cuda")
        self.reset_history()

    def reset_history(self):
        """ReSTIRPTPass.h:63-69"""
        self.reservoir_flip = 0
        self.frame_count = 0
        self.history_dirty = True
        self.grid_dirty = True

    def execute(self, scene, camera, gbuf_pos, gbuf_norm, direct):
        p = rr.pt_reuse_params(self.frame_count, self.num_initial_candidates, self.max_bounces,
                               int(self.temporal_enable), int(self.spatial_enable), self.spatial_num_neighbors,
                               self.spatial_radius, int(self.include_direct_lighting), self.indirect_strength,
                               self.ray_bias, int(self.guiding_enable), self.guiding_alpha, self.kGridCellCount,
                               self.grid_min_samples, self.grid_kappa_max)
        p.guiding.base_cell_size, p.guiding.distance_slope = self.grid_base_cell_size, self.grid_distance_slope
        self.frame_count += 1
        c, v = self.reservoir_flip, 1 - self.reservoir_flip
        im = rr.PtReuseImages()
        im.gbuf_pos, im.gbuf_norm = gbuf_pos.data_ptr(), gbuf_norm.data_ptr()
        im.direct = direct.data_ptr() if (self.include_direct_lighting and direct is not None) else None
        for k in range(4):
            im.reservoir_curr[k], im.reservoir_prev[k] = self.reservoirs[c][k].data_ptr(), self.reservoirs[v][k].data_ptr()
        for k in range(2):
            im.history_curr[k], im.history_prev[k] = self.history[c][k].data_ptr(), self.history[v][k].data_ptr()
        im.output = self.output.data_ptr()
        im.guiding_accum, im.guiding_fitted = self.guiding_accum.data_ptr(), self.guiding_fitted.data_ptr()
        L, st = rr.lib(), _stream(self.torch)
        if self.grid_dirty:      # consume_grid_dirty (ReSTIRPTPass.cpp:596-611)
            self.grid_dirty = False
            self.ctx.check(L.rr_guiding_reset(self.ctx.handle, im.guiding_accum, im.guiding_fitted,
                                              C.byref(p.guiding), st))
        if self.history_dirty:   # consume_history_dirty (ReSTIRPTPass.cpp:613-652)
            self.history_dirty = False
            self.ctx.check(L.rr_restir_pt_reset_history(self.ctx.handle, C.byref(im), self.width, self.height, st))
        self.ctx.check(L.rr_restir_pt_execute(self.ctx.handle, scene.handle, C.byref(camera), C.byref(p),
                                              C.byref(im), st))
        self.reservoir_flip ^= 1


class AtrousPass:
    """AtrousPass (AtrousPass.h:55-58 defaults)."""
    name = "AtrousPass"

    def __init__(self, ctx, extent):
        import torch
        self.ctx, self.torch = ctx, torch
        self.width, self.height = extent
        self.iterations = 5
        self.sigma_position = 0.25
        self.sigma_normal = 0.20
        self.sigma_luminance = 1.00
        self.enabled = False
        self.ping = [torch.zeros((self.height, self.width, 4), device="cuda") for _ in range(2)]
        self.output_slot = 0

    def execute(self, inp, gbuf_pos, gbuf_norm):
        p = rr.AtrousParams(self.width, self.height, self.iterations, 0, self.sigma_position, self.sigma_normal,
                            self.sigma_luminance, 0)
        slot = C.c_uint32()
        self.ctx.check(rr.lib().rr_atrous_execute(self.ctx.handle, inp.data_ptr(), gbuf_pos.data_ptr(),
                                                  gbuf_norm.data_ptr(), self.ping[0].data_ptr(),
                                                  self.ping[1].data_ptr(), C.byref(p), C.byref(slot),
                                                  _stream(self.torch)))
        self.output_slot = slot.value

    def output(self):
        return self.ping[self.output_slot]


def write_png(path, rgba8) -> None:
    """8-bit RGBA (H x W x 4 numpy uint8) to PNG."""
    h, w, _ = rgba8.shape
    raw = b"".join(b"\x00" + rgba8[y].tobytes() for y in range(h))

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)

    p = Path(path)
    if p.parent and not p.parent.exists():
        p.parent.mkdir(parents=True, exist_ok=True)
    p.write_bytes(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)) +
                  chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))


class Application:
    """Headless counterpart of rr::app::Application (Application.h:50-96):
    the same control surface (load_cornell, set_camera_look_at,
    set_pass_enabled, set_exposure, step, capture_screenshot, compute_mse)
    over the CUDA passes, without a window."""

    def __init__(self):
        self.ctx = None
        self.width, self.height = 1280, 720
        self.exposure = 1.0
        self.scene_name = ""
        self._host = None
        self.scene = None
        self.use_di = self.use_gi = self.use_pt = self.use_denoise = False
        self.input_enabled = False
        self.mse_latest = None

    # ── lifecycle ──────────────────────────────────────────────────────────
    def initialize(self, width: int = 1280, height: int = 720, device: int = 0):
        import torch
        self.torch = torch
        torch.cuda.set_device(device)
        self.width, self.height = width, height
        self.ctx = rr.Context(device)
        ext = (width, height)
        self.pathtracer = PathTracerPass(self.ctx, ext)
        self.accumulate = AccumulatePass(self.ctx, ext)
        self.restir_di = ReSTIRDIPass(self.ctx, ext)
        self.restir_gi = ReSTIRGIPass(self.ctx, ext)
        self.restir_pt = ReSTIRPTPass(self.ctx, ext)
        self.atrous = AtrousPass(self.ctx, ext)
        self.camera_desc = rr.camera_desc(width, height)
        self._prev_desc = None
        self.load_cornell()

    def shutdown(self):
        if self.scene is not None:
            self.scene.close()
            self.scene = None
        if self.ctx is not None:
            self.ctx.close()
            self.ctx = None

    # ── scene ──────────────────────────────────────────────────────────────
    def _set_scene(self, host, name):
        if self.scene is not None:
            self.scene.close()
        self._host = host
        self.scene = rr.Scene(self.ctx, host.arrays)
        self.scene_name = name
        self.camera_desc = rr.camera_desc(self.width, self.height)   # scene load resets the camera
        self._reset_accumulation()

    def load_cornell(self):
        self._set_scene(rr.HostScene.cornell(0), "Cornell Box")

    def load_procedural(self, seed=0x5EED0002, triangles=1_000_000, emitters=4096):
        self._set_scene(rr.HostScene.procedural(seed, triangles, emitters), "Procedural room")
        self.set_camera_look_at((0.0, 4.0, 34.0), (0.0, -3.0, 0.0))

    def load_gltf(self, path):
        """Application::reload_scene_gltf (Application.cpp:761-794): on a load
        failure the Cornell box is loaded instead and the error is reported."""
        try:
            host = rr.HostScene.gltf(path)
        except rr.RRError as e:
            print(f"[Scene] glTF load failed for '{path}', falling back to Cornell Box: {e}")
            self.load_cornell()
            return False
        self._set_scene(host, Path(str(path)).name)
        return True

    # ── camera / passes / tonemap ─────────────────────────────────────────
    def set_camera_look_at(self, eye, center, up=(0.0, 1.0, 0.0)):
        self.camera_desc = rr.camera_desc(self.width, self.height, eye=eye, center=center)
        self._reset_accumulation()

    def set_pass_enabled(self, name: str, enabled: bool):
        """Application::set_pass_enabled (Application.cpp:993-1003)."""
        if name == "restir_di":
            self.use_di = enabled
        elif name == "restir_gi":
            self.use_gi = enabled
        elif name == "restir_pt":
            self.use_pt = enabled
        elif name == "denoise":
            self.use_denoise = enabled
        else:
            raise ValueError(f"set_pass_enabled: unknown pass '{name}' (restir_di | restir_gi | restir_pt | denoise)")
        self._reset_accumulation()

    def set_exposure(self, exposure: float):
        self.exposure = float(exposure)

    def _reset_accumulation(self):
        if hasattr(self, "accumulate"):
            self.accumulate.camera_moved = True
            self.accumulate.accumulated_spp = 0
            self.restir_di.reset_history()
            self.restir_gi.reset_history()
            self.restir_pt.reset_history()

    # ── frame ──────────────────────────────────────────────────────────────
    def _modes(self):
        """ReSTIR PT and GI are exclusive indirect modes, PT wins (Application.cpp:417-421)."""
        use_gi_eff = self.use_gi and not self.use_pt
        realtime = self.use_di or use_gi_eff or self.use_pt
        return use_gi_eff, realtime, self.use_denoise and realtime

    def _realtime_image(self):
        """The atrous input and the realtime image (Application.cpp:516-535)."""
        if self.use_pt:
            return self.restir_pt.output
        if self.use_gi:
            return self.restir_gi.output
        if self.use_di:
            return self.restir_di.output
        return None

    def step(self):
        """Application::render_frame pass scheduling (Application.cpp:388-443).
        The G-buffer is ReSTIR DI's primary-ray G-buffer, so DI runs whenever a
        realtime pass does; its output is added as direct light only when DI is
        enabled (include_direct_lighting = use_di_)."""
        if not (self.use_di or self.use_gi):
            self.use_denoise = False
        use_gi_eff, realtime, use_denoise = self._modes()
        cam = rr.camera_data(self.camera_desc, self._prev_desc)
        self._prev_desc = self.camera_desc
        if not realtime:
            self.pathtracer.execute(self.scene, cam)
            self.accumulate.execute(self.pathtracer.radiance[0])
            return
        di = self.restir_di
        di.execute(self.scene, cam)
        if use_gi_eff:
            self.restir_gi.include_direct_lighting = self.use_di
            self.restir_gi.execute(self.scene, cam, di.gbuf_pos, di.gbuf_norm, di.output)
        if self.use_pt:
            self.restir_pt.include_direct_lighting = self.use_di
            self.restir_pt.execute(self.scene, cam, di.gbuf_pos, di.gbuf_norm, di.output)
        if use_denoise:
            self.atrous.execute(self._realtime_image(), di.gbuf_pos, di.gbuf_norm)

    def displayed_image(self):
        """Application::current_display_image (Application.cpp:795-813)."""
        use_gi_eff, realtime, use_denoise = self._modes()
        if use_denoise:
            return self.atrous.output()
        if self.use_pt:
            return self.restir_pt.output
        if use_gi_eff:
            return self.restir_gi.output
        if self.use_di:
            return self.restir_di.output
        return self.accumulate.accumulated

    def capture_screenshot(self, path: str):
        torch = self.torch
        img = self.displayed_image()
        ldr = torch.empty((self.height, self.width, 4), dtype=torch.uint8, device="cuda")
        self.ctx.check(rr.lib().rr_tonemap_execute(self.ctx.handle, img.data_ptr(), self.width, self.height,
                                                   self.exposure, ldr.data_ptr(), _stream(torch)))
        write_png(path, ldr.cpu().numpy())

    def compute_mse(self, crop: int = 64):
        """MSE of the realtime image against the accumulated image over a
        centre crop (Application.cpp:892-949)."""
        torch = self.torch
        if not (self.use_di or self.use_gi or self.use_pt) or self.width < crop or self.height < crop:
            return None
        out = torch.zeros(1, dtype=torch.float64, device="cuda")
        x0, y0 = (self.width - crop) // 2, (self.height - crop) // 2
        self.ctx.check(rr.lib().rr_image_mse(self.ctx.handle, self.accumulate.accumulated.data_ptr(),
                                             self.displayed_image().data_ptr(), self.width, self.height, x0, y0,
                                             crop, crop, out.data_ptr(), _stream(torch)))
        self.mse_latest = float(out.item())
        return self.mse_latest

    @property
    def window_size(self):
        return (self.width, self.height)
