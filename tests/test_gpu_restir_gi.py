"""ReSTIR GI (restir_gi.slang, ReSTIRGIPass::execute) on the GPU against the
oracle, bit-exact after every dispatch.

Each frame takes its G-buffer and direct lighting from the GPU ReSTIR DI pass
(itself bit-exact against the oracle in test_gpu_parity.py) and feeds the same
inputs to both sides; the camera moves a little between frames so that the
temporal pass reprojects. Compared: the three reservoir images after each of
initial, temporal and spatial shade, the primary history and the shaded
output.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _assert_same(gpu, ref, what):
    g, r = _bits(gpu), _bits(ref)
    bad = np.argwhere(g != r)
    assert bad.size == 0, f"{what}: {len(bad)} words differ, first at {tuple(bad[0])}: gpu {gpu[tuple(bad[0])]} " \
                          f"oracle {ref[tuple(bad[0])]}"


def _run(rr, O, ctx, torch, arrays, W, H, frames, eye0, center, move, **kw):
    scene = rr.Scene(ctx, arrays)
    S = O.OracleScene(arrays)
    L = rr.lib()
    st = _stream(torch)
    dev = lambda: torch.zeros((H, W, 4), device="cuda")
    gpos, gnrm, dres, direct = dev(), dev(), dev(), dev()
    res = [[dev() for _ in range(3)] for _ in range(2)]
    hist = [[dev() for _ in range(2)] for _ in range(2)]
    out = dev()
    p = rr.gi_reuse_params(**kw)
    o_p = O.gi_reuse_params(**kw)
    imgs = rr.GiReuseImages()
    o_res = [[np.zeros((H, W, 4), np.float32) for _ in range(3)] for _ in range(2)]
    o_hist = [[np.zeros((H, W, 4), np.float32) for _ in range(2)] for _ in range(2)]
    o_out = np.zeros((H, W, 4), np.float32)
    # the reference clears the history before the first frame (ReSTIRGIPass.cpp:383-399)
    for h in hist:
        h[0][..., 3] = -1.0
    for h in o_hist:
        h[0][..., 3] = -1.0
    prev_desc = None
    di = rr.DIParams(0, 8, 0, 0, 4, 15, 20, 0)
    for f in range(frames):
        desc = rr.camera_desc(W, H, eye=tuple(e + d * f for e, d in zip(eye0, move)), center=center)
        cam = rr.camera_data(desc, prev_desc)
        di.frame_seed = f
        ctx.check(L.rr_restir_di_initial(ctx.handle, scene.handle, C.byref(cam), C.byref(di), gpos.data_ptr(),
                                         gnrm.data_ptr(), dres.data_ptr(), st))
        ctx.check(L.rr_restir_di_spatial_shade(ctx.handle, scene.handle, C.byref(cam), C.byref(di),
                                               gpos.data_ptr(), gnrm.data_ptr(), dres.data_ptr(), direct.data_ptr(), st))
        c, pv = f & 1, 1 - (f & 1)
        imgs.gbuf_pos, imgs.gbuf_norm, imgs.direct = gpos.data_ptr(), gnrm.data_ptr(), direct.data_ptr()
        for k in range(3):
            imgs.reservoir_curr[k], imgs.reservoir_prev[k] = res[c][k].data_ptr(), res[pv][k].data_ptr()
        for k in range(2):
            imgs.history_curr[k], imgs.history_prev[k] = hist[c][k].data_ptr(), hist[pv][k].data_ptr()
        imgs.output = out.data_ptr()
        p.frame_seed = f
        o_p.frame_seed = f
        torch.cuda.synchronize()
        o_img = dict(gbuf_pos=gpos.cpu().numpy(), gbuf_norm=gnrm.cpu().numpy(), direct=direct.cpu().numpy(),
                     res_curr=o_res[c], res_prev=o_res[pv], hist_curr=o_hist[c], hist_prev=o_hist[pv], output=o_out)
        stages = [("initial", L.rr_restir_gi_initial, O.restir_gi_initial),
                  ("temporal", L.rr_restir_gi_temporal, O.restir_gi_temporal),
                  ("spatial_shade", L.rr_restir_gi_spatial_shade, O.restir_gi_spatial_shade)]
        for name, gfn, ofn in stages:
            ctx.check(gfn(ctx.handle, scene.handle, C.byref(cam), C.byref(p), C.byref(imgs), st))
            ofn(S, cam, o_p, o_img)
            torch.cuda.synchronize()
            for k in range(3):
                _assert_same(res[c][k].cpu().numpy(), o_res[c][k], f"frame {f} {name} reservoir[{k}]")
        for k in range(2):
            _assert_same(hist[c][k].cpu().numpy(), o_hist[c][k], f"frame {f} history[{k}]")
        _assert_same(out.cpu().numpy(), o_out, f"frame {f} output")
        prev_desc = desc
    last = o_res[(frames - 1) & 1]
    M = last[2][..., 3].view(np.uint32)
    stats = dict(filled=float((M > 0).mean()), M=float(M.mean()), out_mean=float(o_out[..., :3].mean()),
                 direct_mean=float(o_img["direct"][..., :3].mean()))
    scene.close()
    return stats


@pytest.fixture(params=[1, 0], ids=["wavefront", "per_pixel"])
def initial_form(request, rr, ctx):
    """cs_initial as the wavefront (default) and as one thread per pixel."""
    ctx.check(rr.lib().rr_reuse_set_wavefront(ctx.handle, request.param))
    yield request.param
    ctx.check(rr.lib().rr_reuse_set_wavefront(ctx.handle, 1))


def test_restir_gi_cornell_bit_exact(rr, O, ctx, torch_cuda, initial_form):
    torch = torch_cuda
    hs = rr.HostScene.cornell(0)
    s = _run(rr, O, ctx, torch, hs.arrays, 48, 40, 4, (0.0, 0.0, 3.0), (0.0, 0.0, 0.0), (0.004, 0.0, -0.01))
    # the reuse passes act: temporal M grows past one frame's candidates, indirect light is added
    assert s["filled"] > 0.9 and s["M"] > 16 and s["out_mean"] > s["direct_mean"]


def test_restir_gi_procedural_bit_exact(rr, O, ctx, torch_cuda, initial_form):
    torch = torch_cuda
    hs = rr.HostScene.procedural(target_triangles=20_000, emissive_triangles=64, box_half=20.0)
    s = _run(rr, O, ctx, torch, hs.arrays, 40, 32, 3, (0.0, 4.0, 34.0), (0.0, -3.0, 0.0), (0.05, 0.0, -0.1))
    assert s["filled"] > 0.5


def test_restir_gi_options_bit_exact(rr, O, ctx, torch_cuda):
    """Temporal and spatial off, no direct input term, three candidates, a larger bias."""
    torch = torch_cuda
    hs = rr.HostScene.cornell(1)
    _run(rr, O, ctx, torch, hs.arrays, 32, 24, 2, (0.0, 0.0, 3.0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0),
         temporal=0, spatial=0, include_direct=0, candidates=3, ray_bias=2e-3, indirect_strength=0.5)


@pytest.mark.parametrize("candidates", [0, 1])
def test_restir_gi_few_candidates_bit_exact(rr, O, ctx, torch_cuda, initial_form, candidates):
    """No candidate at all (zero wavefront steps) and a single one."""
    torch = torch_cuda
    hs = rr.HostScene.cornell(0)
    _run(rr, O, ctx, torch, hs.arrays, 24, 16, 2, (0.0, 0.0, 3.0), (0.0, 0.0, 0.0), (0.002, 0.0, -0.01),
         candidates=candidates)


def test_restir_gi_execute_matches_dispatches(rr, ctx, torch_cuda):
    """rr_restir_gi_execute is the three dispatches in order."""
    torch = torch_cuda
    hs = rr.HostScene.cornell(0)
    scene = rr.Scene(ctx, hs.arrays)
    L = rr.lib()
    st = _stream(torch)
    W, H = 32, 24
    dev = lambda: torch.zeros((H, W, 4), device="cuda")
    gpos, gnrm, dres, direct = dev(), dev(), dev(), dev()
    cam = rr.camera_data(rr.camera_desc(W, H, eye=(0.0, 0.0, 3.0), center=(0.0, 0.0, 0.0)))
    di = rr.DIParams(0, 8, 0, 0, 4, 15, 20, 0)
    ctx.check(L.rr_restir_di_initial(ctx.handle, scene.handle, C.byref(cam), C.byref(di), gpos.data_ptr(),
                                     gnrm.data_ptr(), dres.data_ptr(), st))
    ctx.check(L.rr_restir_di_spatial_shade(ctx.handle, scene.handle, C.byref(cam), C.byref(di), gpos.data_ptr(),
                                           gnrm.data_ptr(), dres.data_ptr(), direct.data_ptr(), st))
    outs = []
    for split in (False, True):
        res = [[dev() for _ in range(3)] for _ in range(2)]
        hist = [[dev() for _ in range(2)] for _ in range(2)]
        out = dev()
        imgs = rr.GiReuseImages()
        imgs.gbuf_pos, imgs.gbuf_norm, imgs.direct, imgs.output = (gpos.data_ptr(), gnrm.data_ptr(),
                                                                   direct.data_ptr(), out.data_ptr())
        for k in range(3):
            imgs.reservoir_curr[k], imgs.reservoir_prev[k] = res[0][k].data_ptr(), res[1][k].data_ptr()
        for k in range(2):
            imgs.history_curr[k], imgs.history_prev[k] = hist[0][k].data_ptr(), hist[1][k].data_ptr()
        ctx.check(L.rr_restir_gi_reset_history(ctx.handle, C.byref(imgs), W, H, st))
        p = rr.gi_reuse_params(frame_seed=5)
        if split:
            for fn in (L.rr_restir_gi_initial, L.rr_restir_gi_temporal, L.rr_restir_gi_spatial_shade):
                ctx.check(fn(ctx.handle, scene.handle, C.byref(cam), C.byref(p), C.byref(imgs), st))
        else:
            ctx.check(L.rr_restir_gi_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), C.byref(imgs), st))
        torch.cuda.synchronize()
        outs.append([out.cpu().numpy()] + [r.cpu().numpy() for r in res[0]])
    for a, b in zip(*outs):
        _assert_same(a, b, "execute vs dispatches")
    scene.close()


def test_restir_gi_reset_history(rr, ctx, torch_cuda):
    torch = torch_cuda
    W, H = 8, 4
    imgs = rr.GiReuseImages()
    bufs = [torch.full((H, W, 4), 7.0, device="cuda") for _ in range(5)]
    for k in range(3):
        imgs.reservoir_prev[k] = bufs[k].data_ptr()
    imgs.history_prev[0], imgs.history_prev[1] = bufs[3].data_ptr(), bufs[4].data_ptr()
    ctx.check(rr.lib().rr_restir_gi_reset_history(ctx.handle, C.byref(imgs), W, H, _stream(torch)))
    torch.cuda.synchronize()
    for k in range(3):
        assert (bufs[k] == 0).all()
    assert (bufs[3][..., :3] == 0).all() and (bufs[3][..., 3] == -1).all() and (bufs[4] == 0).all()


def test_restir_gi_rejects_null_images(rr, ctx, torch_cuda):
    torch = torch_cuda
    hs = rr.HostScene.cornell(0)
    scene = rr.Scene(ctx, hs.arrays)
    cam = rr.camera_data(rr.camera_desc(16, 8, eye=(0.0, 0.0, 3.0), center=(0.0, 0.0, 0.0)))
    p = rr.gi_reuse_params()
    imgs = rr.GiReuseImages()
    with pytest.raises(rr.RRError, match="ReSTIR GI"):
        ctx.check(rr.lib().rr_restir_gi_initial(ctx.handle, scene.handle, C.byref(cam), C.byref(p), C.byref(imgs),
                                                _stream(torch)))
    scene.close()


@pytest.mark.parametrize("name", ["directional", "no_lights", "no_geometry"])
def test_restir_gi_light_edge_cases_bit_exact(rr, O, ctx, torch_cuda, name):
    """The light sample's directional (MIS) branch, a scene without lights, and
    a view without geometry (no pixel has a surface: the wavefront's first
    launch finishes every pixel and its steps find empty queues)."""
    import test_gpu_parity
    arrays = test_gpu_parity._edge_scenes(rr)[name]
    _run(rr, O, ctx, torch_cuda, arrays, 32, 24, 2, (0.0, 0.0, 3.0), (0.0, 0.0, 0.0), (0.003, 0.0, -0.01))
