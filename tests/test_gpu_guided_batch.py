"""Guided batches (rr_batch_execute_guided, rr_guides_update): many scenes,
each with its own guide, in one set of wavefront launches; MLP guides run
through one grouped tensor-core launch per bounce, each scene's queries
through its own network. Every scene's image must be bit-identical to
rr_guided_pathtracer_execute of that scene alone with an identical guide,
in plain and CUDA-graph mode, across replays with new seeds and cameras; the
training samples each guide receives must be the same set (grid guides
updated from them stay bit-identical)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


BOUNDS = [((-1.05,) * 3, (1.05,) * 3), ((-52.0,) * 3, (52.0,) * 3), ((-1.05,) * 3, (1.05,) * 3),
          ((-52.0,) * 3, (52.0,) * 3)]


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


def _guide(rr, ctx, kind, k):
    bmin, bmax = BOUNDS[k]
    d = rr.GuideDesc(kind, 8, 0.5, 0.8, (C.c_float * 3)(*bmin), (C.c_float * 3)(*bmax), 1 << 17, 1 << 12, 1e-2,
                     11 + k)
    h = C.c_void_p()
    ctx.check(rr.lib().rr_guide_create(ctx.handle, C.byref(d), C.byref(h)))
    return h


def _single(rr, ctx, torch, scene, cam, p, guide):
    out = torch.empty((p.spp, cam.screen_height, cam.screen_width, 4), device="cuda")
    ctx.check(rr.lib().rr_guided_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), guide,
                                                    out.data_ptr(), _stream(torch)))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _stats(rr, ctx, g):
    st = rr.GuideStats()
    ctx.check(rr.lib().rr_guide_get_stats(ctx.handle, g, C.byref(st)))
    return st


def _eval(rr, ctx, torch, g, k):
    rng = np.random.default_rng(k)
    bmin, bmax = BOUNDS[k]
    N = 512
    surf = np.zeros((N, 3, 4), np.float32)
    surf[:, 0, :3] = rng.uniform(bmin[0], bmax[0], (N, 3)); surf[:, 0, 3] = 1
    n = rng.normal(size=(N, 3)); n /= np.linalg.norm(n, axis=1, keepdims=True)
    surf[:, 1, :3] = n; surf[:, 1, 3] = 1
    surf[:, 2, :3] = n
    ts = torch.from_numpy(surf).cuda()
    mix = torch.zeros((N, 10, 4), device="cuda")
    ctx.check(rr.lib().rr_guide_eval(ctx.handle, g, ts.data_ptr(), N, mix.data_ptr(), _stream(torch)))
    torch.cuda.synchronize()
    return mix.cpu().numpy()


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("kind", ["grid", "mlp"])
def test_guided_batch_matches_single_scene_renders(rr, ctx, torch_cuda, scenes, kind, graph):
    torch = torch_cuda
    L = rr.lib()
    st = _stream(torch)
    gk = rr.GUIDE_GRID if kind == "grid" else rr.GUIDE_MLP
    ga = [_guide(rr, ctx, gk, k) for k in range(len(scenes))]     # the batch's
    gb = [_guide(rr, ctx, gk, k) for k in range(len(scenes))]     # the single-scene renders'
    b = rr.Batch(ctx, scenes)
    if kind == "grid":
        # give the grids lobes: one identical, deterministic training frame on both sets
        for sc, cam, a, g in zip(scenes, _cams(rr), ga, gb):
            p = rr.PtParams(900, 5, 2, 0)
            for h in (a, g):
                _single(rr, ctx, torch, sc, cam, p, h)
                ctx.check(L.rr_guide_update(ctx.handle, h, st))
        for k, (a, g) in enumerate(zip(ga, gb)):
            ea, eb = _eval(rr, ctx, torch, a, k), _eval(rr, ctx, torch, g, k)
            assert np.array_equal(ea.view(np.uint32), eb.view(np.uint32))
            assert _stats(rr, ctx, a).cells_valid > 0
    else:
        # the networks differ per scene (initialised from different seeds)
        assert not np.array_equal(_eval(rr, ctx, torch, ga[0], 1), _eval(rr, ctx, torch, ga[1], 1))
    flags = rr.PT_FLAG_GRAPH if graph else 0
    for frame, shift in ((0, 0.0), (16, 0.05), (32, -0.1)):
        cams = _cams(rr, shift)
        p = rr.PtParams(frame, 5, 2, flags)
        outs = [torch.full((2, c.screen_height, c.screen_width, 4), -1.0, device="cuda") for c in cams]
        b.execute_guided(cams, p, [g.value for g in ga], [o.data_ptr() for o in outs], st)
        torch.cuda.synchronize()
        for k, (sc, cam, o, g) in enumerate(zip(scenes, cams, outs, gb)):
            ref = _single(rr, ctx, torch, sc, cam, rr.PtParams(frame, 5, 2, 0), g)
            got = o.cpu().numpy()
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (kind, graph, frame, k)
        if kind == "grid":
            # the same sample sets -> the same grids after one update (batched vs one by one)
            arr = (C.c_void_p * len(ga))(*[g.value for g in ga])
            ctx.check(L.rr_guides_update(ctx.handle, arr, len(ga), st))
            for g in gb:
                ctx.check(L.rr_guide_update(ctx.handle, g, st))
            for k, (a, g) in enumerate(zip(ga, gb)):
                sa, sb = _stats(rr, ctx, a), _stats(rr, ctx, g)
                assert sa.samples_recorded == sb.samples_recorded > 0, (frame, k)
                ea, eb = _eval(rr, ctx, torch, a, k), _eval(rr, ctx, torch, g, k)
                assert np.array_equal(ea.view(np.uint32), eb.view(np.uint32)), (frame, k)
    if kind == "mlp":
        # the recorded sample counts agree, and the batched update trains every network
        arr = (C.c_void_p * len(ga))(*[g.value for g in ga])
        ctx.check(L.rr_guides_update(ctx.handle, arr, len(ga), st))
        for g in gb:
            ctx.check(L.rr_guide_update(ctx.handle, g, st))
        for k, (a, g) in enumerate(zip(ga, gb)):
            sa, sb = _stats(rr, ctx, a), _stats(rr, ctx, g)
            assert sa.samples_recorded == sb.samples_recorded > 0, k
            assert sa.updates == 1 and np.isfinite(sa.last_loss)
        err = C.c_int(0)
        for g in ga:
            ctx.check(L.rr_guide_mlp_params(ctx.handle, g, None, None, None, rr.MLP_PARAM_COUNT, C.byref(err)))
            assert err.value == 0        # no tensor-core wait gave up
    b.close()
    for g in ga + gb:
        L.rr_guide_destroy(g)


def test_guided_batch_rejects_bad_arguments(rr, ctx, torch_cuda, scenes):
    torch = torch_cuda
    L = rr.lib()
    st = _stream(torch)
    b = rr.Batch(ctx, scenes[:2])
    cams = _cams(rr)[:2]
    outs = [torch.empty((1, c.screen_height, c.screen_width, 4), device="cuda") for c in cams]
    ptrs = [o.data_ptr() for o in outs]
    grid0, grid1 = _guide(rr, ctx, rr.GUIDE_GRID, 0), _guide(rr, ctx, rr.GUIDE_GRID, 1)
    mlp1 = _guide(rr, ctx, rr.GUIDE_MLP, 1)
    p = rr.PtParams(0, 5, 1, 0)
    with pytest.raises(rr.RRError, match="null"):
        b.execute_guided(cams, p, [grid0.value, None], ptrs, st)
    with pytest.raises(rr.RRError, match="twice"):
        b.execute_guided(cams, p, [grid0.value, grid0.value], ptrs, st)
    with pytest.raises(rr.RRError, match="different kinds"):
        b.execute_guided(cams, p, [grid0.value, mlp1.value], ptrs, st)
    with pytest.raises(rr.RRError, match="max_bounces"):
        b.execute_guided(cams, rr.PtParams(0, 0, 1, 0), [grid0.value, grid1.value], ptrs, st)
    b.execute_guided(cams, p, [grid0.value, grid1.value], ptrs, st)      # and a valid call still works
    with pytest.raises(rr.RRError, match="null"):
        ctx.check(L.rr_guides_update(ctx.handle, None, 2, st))
    ctx.check(L.rr_guides_update(ctx.handle, (C.c_void_p * 0)(), 0, st))
    torch.cuda.synchronize()
    b.close()
    for g in (grid0, grid1, mlp1):
        L.rr_guide_destroy(g)
