"""Batches of scenes (rr_batch_*): one set of wavefront launches for many
scenes with their own cameras and image sizes. Every scene's images must be
bit-identical to rr_pathtracer_execute of that scene alone (the single-scene
path is itself bit-exact against the oracle), in plain and in CUDA-graph
mode, across graph replays with new frame seeds and cameras, and after the
batch autotuner has switched traversal variants."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


def _single(rr, ctx, torch, scene, cam, p):
    out = torch.empty((p.spp, cam.screen_height, cam.screen_width, 4), device="cuda")
    ctx.check(rr.lib().rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), out.data_ptr(),
                                             _stream(torch)))
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.fixture(scope="module")
def scenes(rr, ctx):
    hs = [rr.HostScene.cornell(0), rr.HostScene.procedural(target_triangles=30_000, emissive_triangles=64),
          rr.HostScene.cornell(1), rr.HostScene.procedural(seed=7, target_triangles=60_000, emissive_triangles=32)]
    sc = [rr.Scene(ctx, h.arrays) for h in hs]
    yield sc
    for s in sc:
        s.close()


def _cams(rr, shift=0.0):
    sizes = [(40, 24), (33, 17), (64, 48), (24, 40)]
    eyes = [(0.0, 0.0, 3.0), (0.0, 4.0, 34.0), (0.2, 0.1, 3.0), (3.0, 6.0, 30.0)]
    centers = [(0.0, 0.0, 0.0), (0.0, -3.0, 0.0), (0.0, 0.0, 0.0), (0.0, -2.0, 0.0)]
    return [rr.camera_data(rr.camera_desc(w, h, eye=(e[0] + shift, e[1], e[2]), center=c))
            for (w, h), e, c in zip(sizes, eyes, centers)]


@pytest.mark.parametrize("mode", ["wavefront", "per_scene"])
@pytest.mark.parametrize("graph", [False, True])
def test_batch_matches_single_scene_renders(rr, ctx, torch_cuda, scenes, graph, mode):
    torch = torch_cuda
    b = rr.Batch(ctx, scenes)
    b.set_mode(rr.BATCH_WAVEFRONT if mode == "wavefront" else rr.BATCH_PER_SCENE)
    assert b.mode == (rr.BATCH_WAVEFRONT if mode == "wavefront" else rr.BATCH_PER_SCENE)
    flags = rr.PT_FLAG_GRAPH if graph else 0
    for frame, shift in ((0, 0.0), (16, 0.05), (32, -0.1)):   # graph replays with new seeds and cameras
        cams = _cams(rr, shift)
        p = rr.PtParams(frame, 5, 3, flags)
        outs = [torch.full((3, c.screen_height, c.screen_width, 4), -1.0, device="cuda") for c in cams]
        b.execute(cams, p, [o.data_ptr() for o in outs], _stream(torch))
        torch.cuda.synchronize()
        for k, (sc, cam, o) in enumerate(zip(scenes, cams, outs)):
            ref = _single(rr, ctx, torch, sc, cam, rr.PtParams(frame, 5, 3, 0))
            got = o.cpu().numpy()
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (graph, mode, frame, k)
    b.close()


def test_batch_tuner_and_counts(rr, ctx, torch_cuda, scenes):
    torch = torch_cuda
    b = rr.Batch(ctx, scenes)
    cams = _cams(rr)
    outs = [torch.empty((2, c.screen_height, c.screen_width, 4), device="cuda") for c in cams]
    ptrs = [o.data_ptr() for o in outs]
    res = b.tune(cams, rr.PtParams(3, 5, 2, 0), ptrs, _stream(torch))
    assert 0 <= res.best_extend < rr.PT_VARIANT_COUNT and 0 <= res.best_shadow < rr.PT_VARIANT_COUNT
    assert all(t > 0 for t in res.extend_ms) and all(t > 0 for t in res.shadow_ms)
    assert b.mode in (rr.BATCH_WAVEFRONT, rr.BATCH_PER_SCENE)
    # after tuning, graph and plain runs still match the single-scene renders
    b.execute(cams, rr.PtParams(3, 5, 2, rr.PT_FLAG_GRAPH), ptrs, _stream(torch))
    torch.cuda.synchronize()
    for sc, cam, o in zip(scenes, cams, outs):
        ref = _single(rr, ctx, torch, sc, cam, rr.PtParams(3, 5, 2, 0))
        assert np.array_equal(o.cpu().numpy().view(np.uint32), ref.view(np.uint32))
    # ray counts of a batch are the sums of the scenes' counts
    b.execute(cams, rr.PtParams(3, 5, 2, rr.PT_FLAG_COUNT_TRAVERSAL), ptrs, _stream(torch))
    st = rr.PtStats()
    ctx.check(rr.lib().rr_pathtracer_stats(ctx.handle, C.byref(st), 1))
    total = 0
    for sc, cam in zip(scenes, cams):
        _single(rr, ctx, torch, sc, cam, rr.PtParams(3, 5, 2, 0))
        s1 = rr.PtStats()
        ctx.check(rr.lib().rr_pathtracer_stats(ctx.handle, C.byref(s1), 1))
        total += s1.extension_rays
    assert st.extension_rays == total
    ctx.check(rr.lib().rr_pathtracer_set_variants(ctx.handle, 0, 0))
    b.close()


def test_batch_rejects_bad_arguments(rr, ctx, torch_cuda, scenes):
    b = rr.Batch(ctx, scenes[:1])
    cams = _cams(rr)[:1]
    with pytest.raises(rr.RRError):
        b.execute(cams, rr.PtParams(0, 5, 1, rr.PT_FLAG_GRAPH | rr.PT_FLAG_TIME_STAGES), [0], 0)
    with pytest.raises(rr.RRError):
        b.execute(cams, rr.PtParams(0, 5, 1, 0), [0], 0)   # null output
    with pytest.raises(rr.RRError):
        b.set_mode(2)
    assert b.mode == rr.BATCH_WAVEFRONT
    b.close()
