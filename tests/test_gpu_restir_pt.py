"""ReSTIR PT (restir_pt.slang, ReSTIRPTPass::execute) on the GPU against the
oracle, bit-exact after every dispatch.

Each frame takes its G-buffer and direct lighting from the GPU ReSTIR DI pass
(itself bit-exact against the oracle in test_gpu_parity.py) and feeds the same
inputs to both sides; the camera moves a little between frames so that the
temporal pass reprojects, and guiding is on with a small grid so that later
frames sample fitted lobes. Compared: the four reservoir images, the primary
history, the shaded output, the guiding accumulators after the splats and the
fitted lobes after cs_fit_guiding.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CELLS = 1 << 12


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
    res = [[dev() for _ in range(4)] for _ in range(2)]
    hist = [[dev() for _ in range(2)] for _ in range(2)]
    out = dev()
    accum = torch.zeros((CELLS, 4), dtype=torch.int32, device="cuda")
    fitted = torch.zeros((CELLS, 4), device="cuda")
    guiding_on = kw.pop("guiding", 1)
    gp = rr.GuidingParams(0.10, 0.02, CELLS, 1, 2, 512.0, 0.5, 0)
    p = rr.pt_reuse_params(cell_count=CELLS, min_samples=2, guiding=guiding_on, **kw)
    imgs = rr.PtReuseImages()
    # oracle state
    o_res = [[np.zeros((H, W, 4), np.float32) for _ in range(4)] for _ in range(2)]
    o_hist = [[np.zeros((H, W, 4), np.float32) for _ in range(2)] for _ in range(2)]
    o_out = np.zeros((H, W, 4), np.float32)
    o_accum = np.zeros((CELLS, 4), np.int32)
    o_fitted = np.zeros((CELLS, 4), np.float32)
    o_gp = O.guiding_params(cell_count=CELLS, min_samples=2)
    o_p = O.pt_reuse_params(gp=O.guiding_params(cell_count=CELLS, min_samples=2, enabled=guiding_on), **kw)
    # the reference clears the history before the first frame (ReSTIRPTPass.cpp:480-502)
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
        for k in range(4):
            imgs.reservoir_curr[k], imgs.reservoir_prev[k] = res[c][k].data_ptr(), res[pv][k].data_ptr()
        for k in range(2):
            imgs.history_curr[k], imgs.history_prev[k] = hist[c][k].data_ptr(), hist[pv][k].data_ptr()
        imgs.output, imgs.guiding_accum, imgs.guiding_fitted = out.data_ptr(), accum.data_ptr(), fitted.data_ptr()
        p.frame_seed = f
        o_p.frame_seed = f
        torch.cuda.synchronize()
        o_img = dict(gbuf_pos=gpos.cpu().numpy(), gbuf_norm=gnrm.cpu().numpy(), direct=direct.cpu().numpy(),
                     res_curr=o_res[c], res_prev=o_res[pv], hist_curr=o_hist[c], hist_prev=o_hist[pv],
                     output=o_out, accum=o_accum, fitted=o_fitted)
        stages = [("initial", L.rr_restir_pt_initial, O.restir_pt_initial),
                  ("temporal", L.rr_restir_pt_temporal, O.restir_pt_temporal),
                  ("spatial_shade", L.rr_restir_pt_spatial_shade, O.restir_pt_spatial_shade)]
        for name, gfn, ofn in stages:
            ctx.check(gfn(ctx.handle, scene.handle, C.byref(cam), C.byref(p), C.byref(imgs), st))
            ofn(S, cam, o_p, o_img)
            torch.cuda.synchronize()
            for k in range(4):
                _assert_same(res[c][k].cpu().numpy(), o_res[c][k], f"frame {f} {name} reservoir[{k}]")
        for k in range(2):
            _assert_same(hist[c][k].cpu().numpy(), o_hist[c][k], f"frame {f} history[{k}]")
        _assert_same(out.cpu().numpy(), o_out, f"frame {f} output")
        _assert_same(accum.cpu().numpy(), o_accum, f"frame {f} guiding accumulators")
        ctx.check(L.rr_guiding_fit(ctx.handle, accum.data_ptr(), fitted.data_ptr(), C.byref(gp), st))
        O.guiding_fit(o_accum, o_fitted, o_gp)
        torch.cuda.synchronize()
        _assert_same(fitted.cpu().numpy(), o_fitted, f"frame {f} fitted lobes")
        prev_desc = desc
    stats = dict(valid=float((o_res[(frames - 1) & 1][3][..., 3] > 0.5).mean()),
                 M=float(o_res[(frames - 1) & 1][1][..., 3].view(np.uint32).mean()),
                 lobes=int((o_fitted[:, 3] > 0).sum()), out_mean=float(o_out[..., :3].mean()),
                 direct_mean=float(o_img["direct"][..., :3].mean()))
    scene.close()
    return stats


@pytest.fixture(params=[1, 0], ids=["wavefront", "per_pixel"])
def initial_form(request, rr, ctx):
    """cs_initial as the wavefront (default) and as one thread per pixel."""
    ctx.check(rr.lib().rr_reuse_set_wavefront(ctx.handle, request.param))
    yield request.param
    ctx.check(rr.lib().rr_reuse_set_wavefront(ctx.handle, 1))


def test_restir_pt_cornell_bit_exact(rr, O, ctx, torch_cuda, initial_form):
    torch = torch_cuda
    hs = rr.HostScene.cornell(0)
    s = _run(rr, O, ctx, torch, hs.arrays, 48, 40, 4, (0.0, 0.0, 3.0), (0.0, 0.0, 0.0), (0.004, 0.0, -0.01))
    # the reuse passes act: temporal M grows, the grid fills, indirect light is added
    assert s["valid"] > 0.9 and s["M"] > 16 and s["lobes"] > 50 and s["out_mean"] > s["direct_mean"]


def test_restir_pt_procedural_bit_exact(rr, O, ctx, torch_cuda, initial_form):
    torch = torch_cuda
    hs = rr.HostScene.procedural(target_triangles=20_000, emissive_triangles=64, box_half=20.0)
    s = _run(rr, O, ctx, torch, hs.arrays, 40, 32, 3, (0.0, 4.0, 34.0), (0.0, -3.0, 0.0), (0.05, 0.0, -0.1))
    assert s["valid"] > 0.5


def test_restir_pt_options_bit_exact(rr, O, ctx, torch_cuda):
    """Temporal and spatial off, no direct input term, one bounce, no guiding."""
    torch = torch_cuda
    hs = rr.HostScene.cornell(1)
    _run(rr, O, ctx, torch, hs.arrays, 32, 24, 2, (0.0, 0.0, 3.0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0),
         temporal=0, spatial=0, include_direct=0, max_bounces=1, guiding=0, candidates=3)


def test_restir_pt_deep_paths_bit_exact(rr, O, ctx, torch_cuda):
    """More candidates and bounces than the defaults (the wavefront runs
    candidates x bounces steps), on the procedural room."""
    torch = torch_cuda
    hs = rr.HostScene.procedural(seed=5, target_triangles=20_000, emissive_triangles=32, box_half=20.0)
    s = _run(rr, O, ctx, torch, hs.arrays, 24, 20, 2, (0.0, 4.0, 34.0), (0.0, -3.0, 0.0), (0.05, 0.0, -0.1),
             candidates=5, max_bounces=7)
    assert s["valid"] > 0.5


@pytest.mark.parametrize("candidates,bounces", [(0, 4), (1, 0), (2, 1)])
def test_restir_pt_few_candidates_bit_exact(rr, O, ctx, torch_cuda, initial_form, candidates, bounces):
    """No candidate at all (zero wavefront steps), max_bounces 0 (treated as
    one segment), one bounce."""
    torch = torch_cuda
    hs = rr.HostScene.cornell(0)
    _run(rr, O, ctx, torch, hs.arrays, 24, 16, 2, (0.0, 0.0, 3.0), (0.0, 0.0, 0.0), (0.002, 0.0, -0.01),
         candidates=candidates, max_bounces=bounces)


def test_restir_pt_reset_history(rr, ctx, torch_cuda):
    torch = torch_cuda
    W, H = 8, 4
    imgs = rr.PtReuseImages()
    bufs = [torch.full((H, W, 4), 7.0, device="cuda") for _ in range(6)]
    for k in range(4):
        imgs.reservoir_prev[k] = bufs[k].data_ptr()
    imgs.history_prev[0], imgs.history_prev[1] = bufs[4].data_ptr(), bufs[5].data_ptr()
    ctx.check(rr.lib().rr_restir_pt_reset_history(ctx.handle, C.byref(imgs), W, H, _stream(torch)))
    torch.cuda.synchronize()
    for k in range(4):
        assert (bufs[k] == 0).all()
    assert (bufs[4][..., :3] == 0).all() and (bufs[4][..., 3] == -1).all() and (bufs[5] == 0).all()


@pytest.mark.parametrize("name", ["directional", "no_lights", "no_geometry"])
def test_restir_pt_light_edge_cases_bit_exact(rr, O, ctx, torch_cuda, name):
    """The light sample's directional (MIS) branch, a scene without lights, and
    a view without geometry (no pixel has a surface: the wavefront's first
    launch finishes every pixel and its steps find empty queues)."""
    import test_gpu_parity
    arrays = test_gpu_parity._edge_scenes(rr)[name]
    _run(rr, O, ctx, torch_cuda, arrays, 32, 24, 2, (0.0, 0.0, 3.0), (0.0, 0.0, 0.0), (0.003, 0.0, -0.01))
