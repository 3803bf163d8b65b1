"""GPU parity: every kernel against the CPU oracle on the same seeded inputs.

The kernels and the oracle evaluate the same binary32 operations in the same
order (no FMA contraction, IEEE division/sqrt, the rr_detmath.h elementary
functions), so the stated tolerance is ZERO: images, G-buffers, reservoirs,
hits and guiding state must be bit-identical. Calls go through the C ABI.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


@pytest.fixture(scope="module")
def cornell(rr, O, ctx):
    hs = rr.HostScene.cornell(0)
    return hs.arrays, rr.Scene(ctx, hs.arrays), O.OracleScene(hs.arrays, use_bvh=False)


@pytest.fixture(scope="module")
def procedural(rr, O, ctx):
    hs = rr.HostScene.procedural(seed=0x5EED0002, target_triangles=120_000, emissive_triangles=128, box_half=20.0)
    return hs.arrays, rr.Scene(ctx, hs.arrays), O.OracleScene(hs.arrays, use_bvh=True)


def cam_for(rr, kind, w, h):
    if kind == "cornell":
        return rr.camera_data(rr.camera_desc(w, h))
    return rr.camera_data(rr.camera_desc(w, h, eye=(0.0, 8.0, 45.0), center=(0.0, -2.0, 0.0)))


def gpu_pathtrace(rr, ctx, scene, cam, torch, frame_seed, max_bounces, spp):
    out = torch.empty((spp, cam.screen_height, cam.screen_width, 4), device="cuda", dtype=torch.float32)
    p = rr.PtParams(frame_seed, max_bounces, spp, 0)
    ctx.check(rr.lib().rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), out.data_ptr(),
                                             _stream(torch)))
    torch.cuda.synchronize()
    return _np(out)


def test_trace_closest_matches_oracle(rr, O, ctx, torch_cuda, cornell, procedural):
    torch = torch_cuda
    rng = np.random.default_rng(11)
    for arrays, scene, oscene, span in (cornell + (1.0,), procedural + (25.0,)):
        n = 20000
        o = np.zeros((n, 4), np.float32)
        o[:, :3] = rng.uniform(-span, span, (n, 3))
        d = np.zeros((n, 4), np.float32)
        v = rng.normal(size=(n, 3))
        d[:, :3] = v / np.linalg.norm(v, axis=1, keepdims=True)
        ho, po = oscene.trace(o, d)
        to, td = torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()
        hits = torch.empty((n, 4), device="cuda")
        prims = torch.empty(n, device="cuda", dtype=torch.int32)
        ctx.check(rr.lib().rr_trace_closest(ctx.handle, scene.handle, to.data_ptr(), td.data_ptr(), 0.001, 1e9, n,
                                            hits.data_ptr(), prims.data_ptr(), _stream(torch)))
        torch.cuda.synchronize()
        hg, pg = _np(hits), _np(prims).view(np.uint32)
        assert (ho[:, 3].view(np.uint32) != 0xFFFFFFFF).mean() > 0.3
        np.testing.assert_array_equal(hg.view(np.uint32), ho.view(np.uint32))
        np.testing.assert_array_equal(pg, po)


def test_traversal_work_matches_cpu_restatement(rr, O, ctx, torch_cuda, cornell, procedural):
    """The traversal's node / triangle counters (the algorithmic work behind the
    roofline bytes) equal a CPU restatement walking the library's own BVH in the
    same child order (front to back for closest hit, back to front for any
    hit), ray by ray, for closest-hit and any-hit rays;
    the hits agree bit for bit too."""
    torch = torch_cuda
    rng = np.random.default_rng(23)
    L = rr.lib()
    for arrays, scene, _, span in (cornell + (1.0,), procedural + (25.0,)):
        stats = rr.SceneStats()
        ctx.check(L.rr_scene_get_stats(scene.handle, C.byref(stats)))
        nodes = np.zeros((stats.bvh_node_count, 16), np.float32)
        tris = np.zeros((max(stats.triangle_count, 1), 12), np.float32)
        ctx.check(L.rr_scene_copy_bvh(ctx.handle, scene.handle, nodes.ctypes.data, tris.ctypes.data))
        n = 8192
        o = np.zeros((n, 4), np.float32)
        o[:, :3] = rng.uniform(-span, span, (n, 3))
        d = np.zeros((n, 4), np.float32)
        v = rng.normal(size=(n, 3))
        d[:, :3] = v / np.linalg.norm(v, axis=1, keepdims=True)
        d[:64, :3] = [1.0, 0.0, 0.0]        # axis-parallel rays: zero direction components
        nodes4 = np.zeros((stats.bvh4_node_count, 32), np.float32)
        ctx.check(L.rr_scene_copy_bvh4(ctx.handle, scene.handle, nodes4.ctypes.data))
        for any_hit, tmax in ((0, 1e9), (1, 0.7 * span)):
            to, td = torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()
            results = []
            for wide in (0, rr.TRACE_WIDE):
                hits = torch.empty((n, 4), device="cuda")
                prims = torch.empty(n, device="cuda", dtype=torch.int32)
                work = torch.empty((n, 2), device="cuda", dtype=torch.int32)
                ctx.check(L.rr_trace_counted(ctx.handle, scene.handle, to.data_ptr(), td.data_ptr(), 0.001, tmax, n,
                                             any_hit | wide, hits.data_ptr(), prims.data_ptr(), work.data_ptr(),
                                             _stream(torch)))
                torch.cuda.synchronize()
                if wide:
                    oh, op, ow = O.bvh4_trace(nodes4, tris, o, d, 0.001, tmax, any_hit)
                else:
                    oh, op, ow = O.bvh2_trace(nodes, tris, o, d, 0.001, tmax, any_hit)
                np.testing.assert_array_equal(_np(hits).view(np.uint32), oh.view(np.uint32))
                np.testing.assert_array_equal(_np(prims).view(np.uint32), op)
                np.testing.assert_array_equal(_np(work).view(np.uint32), ow)
                assert ow[:, 0].mean() > 2 and (oh[:, 3].view(np.uint32) != 0xFFFFFFFF).mean() > 0.1
                results.append((oh, op, ow))
            # both trees give the same closest hits (an any-hit ray reports the first
            # triangle it meets, which depends on the visiting order: compare hit / miss);
            # the 4-wide tree in fewer node visits
            if any_hit:
                np.testing.assert_array_equal(results[0][0][:, 0] >= 0, results[1][0][:, 0] >= 0)
            else:
                np.testing.assert_array_equal(results[0][0].view(np.uint32), results[1][0].view(np.uint32))
                np.testing.assert_array_equal(results[0][1], results[1][1])
            assert results[1][2][:, 0].sum() < results[0][2][:, 0].sum()


@pytest.mark.parametrize("seed", [0, 7])
def test_pathtracer_cornell_bit_exact(rr, O, ctx, torch_cuda, cornell, seed):
    _, scene, oscene = cornell
    cam = cam_for(rr, "cornell", 64, 48)
    g = gpu_pathtrace(rr, ctx, scene, cam, torch_cuda, seed, 8, 2)
    o, _ = O.pathtrace(oscene, cam, seed, 8, 2)
    assert g[..., :3].mean() > 0.1
    np.testing.assert_array_equal(g.view(np.uint32), o.view(np.uint32))


def test_pathtracer_counts_match_oracle(rr, O, ctx, torch_cuda, cornell):
    _, scene, oscene = cornell
    cam = cam_for(rr, "cornell", 40, 40)
    gpu_pathtrace(rr, ctx, scene, cam, torch_cuda, 3, 5, 1)
    st = rr.PtStats()
    ctx.check(rr.lib().rr_pathtracer_stats(ctx.handle, C.byref(st), 1))
    _, (oe, os_) = O.pathtrace(oscene, cam, 3, 5, 1)
    assert (st.extension_rays, st.shadow_rays) == (oe, os_)


def test_pathtracer_count_and_timing_flags_keep_results(rr, O, ctx, torch_cuda, procedural):
    torch = torch_cuda
    _, scene, _ = procedural
    cam = cam_for(rr, "procedural", 64, 40)
    ref = gpu_pathtrace(rr, ctx, scene, cam, torch, 2, 5, 1)
    out = torch.empty((1, 40, 64, 4), device="cuda")
    p = rr.PtParams(2, 5, 1, rr.PT_FLAG_COUNT_TRAVERSAL | rr.PT_FLAG_TIME_STAGES)
    ctx.check(rr.lib().rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), out.data_ptr(),
                                             _stream(torch)))
    st = rr.PtStats()
    ctx.check(rr.lib().rr_pathtracer_stats(ctx.handle, C.byref(st), 1))
    np.testing.assert_array_equal(_np(out), ref)
    assert st.extension_nodes >= st.extension_rays and st.extension_tris > 0
    assert st.launches_extend == 5 and st.ms_extend > 0


def test_pathtracer_procedural_bit_exact(rr, O, ctx, torch_cuda, procedural):
    _, scene, oscene = procedural
    cam = cam_for(rr, "procedural", 96, 64)
    g = gpu_pathtrace(rr, ctx, scene, cam, torch_cuda, 5, 5, 1)
    o, _ = O.pathtrace(oscene, cam, 5, 5, 1)
    np.testing.assert_array_equal(g.view(np.uint32), o.view(np.uint32))


def test_pathtracer_region_odd_size(rr, O, ctx, torch_cuda, cornell):
    # non-multiple-of-tile image sizes exercise the raygen compaction
    _, scene, oscene = cornell
    cam = cam_for(rr, "cornell", 37, 19)
    g = gpu_pathtrace(rr, ctx, scene, cam, torch_cuda, 1, 4, 3)
    o, _ = O.pathtrace(oscene, cam, 1, 4, 3)
    np.testing.assert_array_equal(g.view(np.uint32), o.view(np.uint32))


@pytest.mark.parametrize("W,H", [(33, 17), (640, 480)])
def test_accumulate_bit_exact_and_fp64(rr, O, ctx, torch_cuda, W, H):
    """33 x 17: one thread per channel (small images); 640 x 480 (307,200
    pixels): one thread per pixel."""
    torch = torch_cuda
    rng = np.random.default_rng(5)
    frames = rng.random((43, H, W, 4)).astype(np.float32) * 3
    acc_o = np.zeros((H, W, 4), np.float32)
    acc_g = torch.zeros((H, W, 4), device="cuda")
    sum64 = torch.zeros((H, W, 4), device="cuda", dtype=torch.float64)
    fr = torch.from_numpy(frames).cuda()
    spp = 0
    # one frame with camera_moved, then batches of 2, 3 and 37 frames (the
    # kernel reads 16 images at a time: 37 crosses two of those boundaries)
    for start, count, moved in ((0, 1, 1), (1, 2, 0), (3, 3, 0), (6, 37, 0)):
        for k in range(count):
            O.accumulate(np.ascontiguousarray(frames[start + k]), acc_o, moved if k == 0 else 0, spp + k)
        p = rr.AccParams(W, H, moved, spp)
        ctx.check(rr.lib().rr_accumulate_execute(ctx.handle, fr[start].data_ptr(), count, acc_g.data_ptr(),
                                                 sum64.data_ptr(), C.byref(p), _stream(torch)))
        spp = (0 if moved else spp) + count
    torch.cuda.synchronize()
    np.testing.assert_array_equal(_np(acc_g).view(np.uint32), acc_o.view(np.uint32))
    np.testing.assert_allclose(_np(sum64), frames.astype(np.float64).sum(0), rtol=1e-12)


def _di_run_gpu(rr, ctx, torch, scene, cam, params_list):
    W, H = cam.screen_width, cam.screen_height
    t = lambda: torch.zeros((H, W, 4), device="cuda")
    gpos, gnrm, out = t(), t(), t()
    res = [t(), t()]
    outs = []
    for f, p in enumerate(params_list):
        cur, prev = res[f & 1], res[(f & 1) ^ 1]
        ctx.check(rr.lib().rr_restir_di_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), gpos.data_ptr(),
                                                gnrm.data_ptr(), cur.data_ptr(), prev.data_ptr(), out.data_ptr(),
                                                _stream(torch)))
        torch.cuda.synchronize()
        outs.append((_np(gpos).copy(), _np(gnrm).copy(), _np(cur).copy(), _np(out).copy()))
    return outs


def _di_run_oracle(O, oscene, cam, params_list):
    W, H = cam.screen_width, cam.screen_height
    z = lambda: np.zeros((H, W, 4), np.float32)
    gpos, gnrm, out = z(), z(), z()
    res = [z(), z()]
    outs = []
    for f, p in enumerate(params_list):
        cur, prev = res[f & 1], res[(f & 1) ^ 1]
        O.restir_di_initial(oscene, cam, p, gpos, gnrm, cur)
        O.restir_di_temporal(oscene, cam, p, gpos, gnrm, cur, prev)
        O.restir_di_spatial_shade(oscene, cam, p, gpos, gnrm, cur, out)
        outs.append((gpos.copy(), gnrm.copy(), cur.copy(), out.copy()))
    return outs


@pytest.mark.parametrize("kind", ["cornell", "procedural"])
def test_restir_di_three_frames_bit_exact(rr, O, ctx, torch_cuda, cornell, procedural, kind):
    arrays, scene, oscene = cornell if kind == "cornell" else procedural
    cam = cam_for(rr, kind, 80, 56)
    # config-2 settings: M=32, K=5, R=30, cap 20*M; frames 0..2 exercise temporal reuse
    plist_g = [rr.DIParams(f, 32, 1, 1, 5, 30, 20, 0) for f in range(3)]
    plist_o = [O.di_params(f, 32, 1, 1, 5, 30, 20) for f in range(3)]
    g = _di_run_gpu(rr, ctx, torch_cuda, scene, cam, plist_g)
    o = _di_run_oracle(O, oscene, cam, plist_o)
    for (gg, go) in zip(g, o):
        for a, b in zip(gg, go):
            np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    assert (o[-1][2][..., 3].view(np.uint32) > 32).any()  # temporal history was merged


def test_restir_di_disabled_paths(rr, O, ctx, torch_cuda, cornell):
    _, scene, oscene = cornell
    cam = cam_for(rr, "cornell", 24, 24)
    plist_g = [rr.DIParams(f, 4, 0, 0, 0, 10, 20, 0) for f in range(2)]
    plist_o = [O.di_params(f, 4, 0, 0, 0, 10, 20) for f in range(2)]
    g = _di_run_gpu(rr, ctx, torch_cuda, scene, cam, plist_g)
    o = _di_run_oracle(O, oscene, cam, plist_o)
    for a, b in zip(g[-1], o[-1]):
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.fixture(scope="module")
def room_1m(rr, O, ctx):
    """The benchmarked scene: the seeded 1M-triangle procedural room."""
    hs = rr.HostScene.procedural(seed=0x5EED0002, target_triangles=1_000_000, emissive_triangles=4096, box_half=20.0)
    return hs.arrays, rr.Scene(ctx, hs.arrays), O.OracleScene(hs.arrays, use_bvh=True)


def test_room_1m_frame_bit_exact(rr, O, ctx, torch_cuda, room_1m):
    """The benchmarked configuration (1M-triangle room, its view, 4 spp at
    depth 5, ReSTIR DI M=32 / cap 20 M / K=5 / R=30 over three frames,
    A-trous 5 iterations) at a small full image, against the oracle."""
    torch = torch_cuda
    _, scene, oscene = room_1m
    W, H = 240, 136
    cam = rr.camera_data(rr.camera_desc(W, H, eye=(0.0, 4.0, 34.0), center=(0.0, -3.0, 0.0)))
    g_img = gpu_pathtrace(rr, ctx, scene, cam, torch, 8, 5, 4)
    o_img, _ = O.pathtrace(oscene, cam, 8, 5, 4)
    np.testing.assert_array_equal(g_img.view(np.uint32), o_img.view(np.uint32))
    plist_g = [rr.DIParams(f, 32, 1, 1, 5, 30, 20, 0) for f in range(3)]
    plist_o = [O.di_params(f, 32, 1, 1, 5, 30, 20) for f in range(3)]
    g = _di_run_gpu(rr, ctx, torch, scene, cam, plist_g)
    o = _di_run_oracle(O, oscene, cam, plist_o)
    for (gg, go) in zip(g, o):
        for a, b in zip(gg, go):
            np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    gpos, gnrm, _, out = o[-1]
    ref = O.atrous(out, gpos, gnrm, 5)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    tin, tp, tn = t(g[-1][3]), t(g[-1][0]), t(g[-1][1])
    ping = [torch.empty_like(tin), torch.empty_like(tin)]
    slot = C.c_uint32()
    for tma in (1, 0):
        ctx.check(rr.lib().rr_atrous_set_tma(ctx.handle, tma))
        ctx.check(rr.lib().rr_atrous_execute(ctx.handle, tin.data_ptr(), tp.data_ptr(), tn.data_ptr(),
                                             ping[0].data_ptr(), ping[1].data_ptr(),
                                             C.byref(rr.AtrousParams(W, H, 5, 0, 0.25, 0.20, 1.0, 0)),
                                             C.byref(slot), _stream(torch)))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(_np(ping[slot.value]).view(np.uint32), ref.view(np.uint32))
    ctx.check(rr.lib().rr_atrous_set_tma(ctx.handle, 1))
    assert (o[-1][2][..., 3].view(np.uint32) > 32).any()   # temporal history was merged


@pytest.mark.parametrize("tma", [1, 0])
@pytest.mark.parametrize("iterations", [1, 5, 7])
def test_atrous_bit_exact(rr, O, ctx, torch_cuda, procedural, iterations, tma):
    """tma 1: TMA tiles for strides 1, 2, 4, the pair-weight kernels beyond;
    tma 0: the pair-weight kernels at every stride (up to 64 on a 72 x 40
    image: taps clamped on every side)."""
    torch = torch_cuda
    _, scene, oscene = procedural
    cam = cam_for(rr, "procedural", 72, 40)
    p = O.di_params(0, 8, 1, 1, 4, 15, 20)
    W, H = 72, 40
    z = lambda: np.zeros((H, W, 4), np.float32)
    gpos, gnrm, res, prev, out = z(), z(), z(), z(), z()
    O.restir_di_initial(oscene, cam, p, gpos, gnrm, res)
    O.restir_di_spatial_shade(oscene, cam, p, gpos, gnrm, res, out)
    ref = O.atrous(out, gpos, gnrm, iterations)
    t = lambda a: torch.from_numpy(a).cuda()
    tin, tp, tn = t(out), t(gpos), t(gnrm)
    ping = [torch.empty_like(tin), torch.empty_like(tin)]
    ap = rr.AtrousParams(W, H, iterations, 0, 0.25, 0.20, 1.0, 0)
    slot = C.c_uint32()
    ctx.check(rr.lib().rr_atrous_set_tma(ctx.handle, tma))
    try:
        ctx.check(rr.lib().rr_atrous_execute(ctx.handle, tin.data_ptr(), tp.data_ptr(), tn.data_ptr(),
                                             ping[0].data_ptr(), ping[1].data_ptr(), C.byref(ap), C.byref(slot),
                                             _stream(torch)))
        torch.cuda.synchronize()
    finally:
        ctx.check(rr.lib().rr_atrous_set_tma(ctx.handle, 1))
    assert slot.value == (min(iterations, 7) - 1) & 1
    np.testing.assert_array_equal(_np(ping[slot.value]).view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("W,H", [(72, 40), (333, 197)])
def test_atrous_tma_tiles_bit_identical(rr, O, ctx, torch_cuda, procedural, W, H):
    """The TMA-staged kernel (strides 1, 2, 4; halo tiles loaded from
    negative and past-the-edge coordinates at the borders) against the
    direct-load kernel and the oracle, one iteration per stride and the
    full 7-iteration run; no tile's copies gave up."""
    torch = torch_cuda
    L = rr.lib()
    _, scene, oscene = procedural
    cam = cam_for(rr, "procedural", W, H)
    p = O.di_params(1, 8, 1, 1, 4, 15, 20)
    z = lambda: np.zeros((H, W, 4), np.float32)
    gpos, gnrm, res, out = z(), z(), z(), z()
    O.restir_di_initial(oscene, cam, p, gpos, gnrm, res)
    O.restir_di_spatial_shade(oscene, cam, p, gpos, gnrm, res, out)
    t = lambda a: torch.from_numpy(a).cuda()
    tin, tp, tn = t(out), t(gpos), t(gnrm)
    st = _stream(torch)
    for stride in (1, 2, 4, 8):
        ap = rr.AtrousParams(W, H, 1, stride, 0.25, 0.20, 1.0, 0)
        got = {}
        for tma in (1, 0):
            ctx.check(L.rr_atrous_set_tma(ctx.handle, tma))
            o = torch.full_like(tin, -7.0)
            ctx.check(L.rr_atrous_iteration(ctx.handle, tin.data_ptr(), tp.data_ptr(), tn.data_ptr(), o.data_ptr(),
                                            C.byref(ap), st))
            torch.cuda.synchronize()
            got[tma] = _np(o)
        np.testing.assert_array_equal(got[1].view(np.uint32), got[0].view(np.uint32), err_msg=f"stride {stride}")
    ctx.check(L.rr_atrous_set_tma(ctx.handle, 1))
    ref = O.atrous(out, gpos, gnrm, 7)
    ping = [torch.empty_like(tin), torch.empty_like(tin)]
    ap = rr.AtrousParams(W, H, 7, 0, 0.25, 0.20, 1.0, 0)
    slot = C.c_uint32()
    ctx.check(L.rr_atrous_execute(ctx.handle, tin.data_ptr(), tp.data_ptr(), tn.data_ptr(), ping[0].data_ptr(),
                                  ping[1].data_ptr(), C.byref(ap), C.byref(slot), st))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(_np(ping[slot.value]).view(np.uint32), ref.view(np.uint32))
    err = C.c_int(-1)
    ctx.check(L.rr_atrous_tma_error(ctx.handle, C.byref(err)))
    assert err.value == 0


def test_atrous_tma_give_up_is_reported_and_output_complete(rr, O, ctx, torch_cuda, procedural):
    """A tile whose copies miss the bounded wait (here: a wait of zero tries,
    so every block gives up at once while its copies still land) filters its
    pixels from global memory: the output stays bit-identical to the oracle.
    The next A-trous call then returns RR_ERR_TIMEOUT without doing work, and
    the call after it proceeds."""
    torch = torch_cuda
    L = rr.lib()
    _, scene, oscene = procedural
    W, H = 131, 77
    cam = cam_for(rr, "procedural", W, H)
    p = O.di_params(2, 8, 1, 1, 4, 15, 20)
    z = lambda: np.zeros((H, W, 4), np.float32)
    gpos, gnrm, res, out = z(), z(), z(), z()
    O.restir_di_initial(oscene, cam, p, gpos, gnrm, res)
    O.restir_di_spatial_shade(oscene, cam, p, gpos, gnrm, res, out)
    ref = O.atrous(out, gpos, gnrm, 5)
    t = lambda a: torch.from_numpy(a).cuda()
    tin, tp, tn = t(out), t(gpos), t(gnrm)
    st = _stream(torch)
    ap = rr.AtrousParams(W, H, 5, 0, 0.25, 0.20, 1.0, 0)
    ping = [torch.empty_like(tin), torch.empty_like(tin)]
    slot = C.c_uint32()
    run = lambda: L.rr_atrous_execute(ctx.handle, tin.data_ptr(), tp.data_ptr(), tn.data_ptr(), ping[0].data_ptr(),
                                      ping[1].data_ptr(), C.byref(ap), C.byref(slot), st)
    ctx.check(L.rr_atrous_set_tma(ctx.handle, 1))
    try:
        ctx.check(L.rr_atrous_set_tma_wait_tries(ctx.handle, 0))
        for p_ in ping:
            p_.fill_(-7.0)
        ctx.check(run())
        torch.cuda.synchronize()
        np.testing.assert_array_equal(_np(ping[slot.value]).view(np.uint32), ref.view(np.uint32))
        assert run() == 6                                  # RR_ERR_TIMEOUT, reported once
        assert "bounded wait" in ctx.last_error()
        ctx.check(L.rr_atrous_set_tma_wait_tries(ctx.handle, 1 << 22))
        ctx.check(run())                                   # flag cleared: this call works
        torch.cuda.synchronize()
        np.testing.assert_array_equal(_np(ping[slot.value]).view(np.uint32), ref.view(np.uint32))
        err = C.c_int(-1)
        ctx.check(L.rr_atrous_tma_error(ctx.handle, C.byref(err)))
        assert err.value == 0
    finally:
        L.rr_atrous_set_tma_wait_tries(ctx.handle, 1 << 22)


def test_queue_limit_returns_queue_overflow(rr, ctx, torch_cuda, cornell):
    """A context capped below a call's paths in flight refuses the call with
    RR_ERR_QUEUE_OVERFLOW before launching anything; lifting the cap lets the
    same call run."""
    torch = torch_cuda
    L = rr.lib()
    _, scene, _ = cornell
    W, H, spp = 32, 16, 2
    cam = cam_for(rr, "cornell", W, H)
    out = torch.full((spp, H, W, 4), -3.0, device="cuda")
    p = rr.PtParams(0, 4, spp, 0)
    try:
        ctx.check(L.rr_ctx_set_queue_limit(ctx.handle, W * H * spp - 1))
        st = L.rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), out.data_ptr(), _stream(torch))
        assert st == 5, rr.RR_STATUS.get(st, st)           # RR_ERR_QUEUE_OVERFLOW
        torch.cuda.synchronize()
        assert bool((out == -3.0).all())                    # nothing ran
        ctx.check(L.rr_ctx_set_queue_limit(ctx.handle, W * H * spp))
        ctx.check(L.rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), out.data_ptr(),
                                          _stream(torch)))
        torch.cuda.synchronize()
        assert bool((out[..., 3] == 1.0).all())
    finally:
        ctx.check(L.rr_ctx_set_queue_limit(ctx.handle, 0))


def test_guiding_splat_fit_sample_bit_exact(rr, O, ctx, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(9)
    cells = 1 << 12
    n = 50000
    pos = np.zeros((n, 4), np.float32); pos[:, :3] = rng.uniform(-2, 2, (n, 3))
    dirs = np.zeros((n, 4), np.float32)
    v = rng.normal(size=(n, 3)) + np.array([0.0, 2.0, 0.0])
    dirs[:, :3] = v / np.linalg.norm(v, axis=1, keepdims=True)
    bsdf = rng.integers(0, 3, n).astype(np.uint32)
    cam = np.array([0.0, 0.5, 4.0], np.float32)
    gp_o = O.guiding_params(cell_count=cells, min_samples=4, base_cell_size=0.5, distance_slope=0.05)
    gp_g = rr.GuidingParams(0.5, 0.05, cells, 1, 4, 512.0, 0.5, 0)
    acc_o = np.zeros((cells, 4), np.int32); fit_o = np.zeros((cells, 4), np.float32)
    O.guiding_splat(acc_o, pos, dirs, bsdf, cam, gp_o)
    acc_before = acc_o.copy()
    O.guiding_fit(acc_o, fit_o, gp_o)
    acc_g = torch.zeros((cells, 4), device="cuda", dtype=torch.int32)
    fit_g = torch.zeros((cells, 4), device="cuda")
    t = lambda a: torch.from_numpy(a).cuda()
    cp = (C.c_float * 3)(*cam.tolist())
    # keep every input tensor referenced until the kernels have run
    tpos, tdirs, tbsdf = t(pos), t(dirs), t(bsdf.view(np.int32))
    ctx.check(rr.lib().rr_guiding_splat(ctx.handle, acc_g.data_ptr(), tpos.data_ptr(), tdirs.data_ptr(),
                                        tbsdf.data_ptr(), n, cp, C.byref(gp_g), _stream(torch)))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(_np(acc_g), acc_before)
    ctx.check(rr.lib().rr_guiding_fit(ctx.handle, acc_g.data_ptr(), fit_g.data_ptr(), C.byref(gp_g), _stream(torch)))
    torch.cuda.synchronize()
    assert not _np(acc_g).any()
    np.testing.assert_array_equal(_np(fit_g).view(np.uint32), fit_o.view(np.uint32))
    assert (fit_o[:, 3] > 0).sum() > 50
    # one-sample MIS sampling at new points, guided where a lobe exists
    m = 20000
    sp = np.zeros((m, 4), np.float32); sp[:, :3] = rng.uniform(-2, 2, (m, 3))
    sn = np.zeros((m, 4), np.float32)
    vv = rng.normal(size=(m, 3)); sn[:, :3] = vv / np.linalg.norm(vv, axis=1, keepdims=True)
    sb = rng.integers(0, 3, m).astype(np.uint32)
    seeds = rng.integers(0, 2 ** 32, m, dtype=np.uint64).astype(np.uint32)
    so = seeds.copy()
    wi_o, pdf_o = O.guiding_sample(fit_o, sp, sn, sb, so, cam, gp_o)
    sg = t(seeds.view(np.int32))
    wi_g = torch.empty((m, 4), device="cuda"); pdf_g = torch.empty(m, device="cuda")
    tsp, tsn, tsb = t(sp), t(sn), t(sb.view(np.int32))
    ctx.check(rr.lib().rr_guiding_sample(ctx.handle, fit_g.data_ptr(), tsp.data_ptr(), tsn.data_ptr(),
                                         tsb.data_ptr(), sg.data_ptr(), m, cp, C.byref(gp_g),
                                         wi_g.data_ptr(), pdf_g.data_ptr(), _stream(torch)))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(_np(wi_g).view(np.uint32), wi_o.view(np.uint32))
    np.testing.assert_array_equal(_np(pdf_g).view(np.uint32), pdf_o.view(np.uint32))
    np.testing.assert_array_equal(_np(sg).view(np.uint32), so)


def test_detmath_against_cuda_libm(rr, O, ctx, torch_cuda):
    """rr_detmath.h through the oracle stays within 2 ulp of CUDA's own
    sinf/cosf/expf/logf (accurate mode) on the argument ranges of the path."""
    torch = torch_cuda
    x = np.linspace(0, 2 * np.pi, 200001, dtype=np.float32)
    xs = torch.from_numpy(x).cuda()
    for name, fn in (("sin", torch.sin), ("cos", torch.cos)):
        ref = _np(fn(xs)).astype(np.float64)
        ours = O.detmath(name, x).astype(np.float64)
        ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
        assert (np.abs(ours - ref) / ulp).max() <= 3.0
    e = np.linspace(-80, 0, 200001, dtype=np.float32)
    ref = _np(torch.exp(torch.from_numpy(e).cuda())).astype(np.float64)
    ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    assert (np.abs(O.detmath("exp", e) - ref) / ulp).max() <= 3.0


def test_traversal_variants_identical_and_tuner(rr, O, ctx, torch_cuda, procedural):
    """Every traversal schedule/occupancy variant renders the same bits; the
    autotuner keeps the fastest and reports a time for each variant."""
    torch = torch_cuda
    _, scene, oscene = procedural
    cam = cam_for(rr, "procedural", 80, 48)
    ref, _ = O.pathtrace(oscene, cam, 9, 5, 1)
    for v in range(rr.PT_VARIANT_COUNT):
        ctx.check(rr.lib().rr_pathtracer_set_variants(ctx.handle, v, v))
        g = gpu_pathtrace(rr, ctx, scene, cam, torch, 9, 5, 1)
        np.testing.assert_array_equal(g.view(np.uint32), ref.view(np.uint32))
    out = torch.empty((1, 48, 80, 4), device="cuda")
    res = rr.PtTuneResult()
    ctx.check(rr.lib().rr_pathtracer_tune(ctx.handle, scene.handle, C.byref(cam), C.byref(rr.PtParams(9, 5, 1, 0)),
                                          out.data_ptr(), _stream(torch), C.byref(res)))
    assert all(t > 0 for t in res.extend_ms) and all(t > 0 for t in res.shadow_ms)
    assert res.extend_ms[res.best_extend] == min(res.extend_ms)
    g = gpu_pathtrace(rr, ctx, scene, cam, torch, 9, 5, 1)
    np.testing.assert_array_equal(g.view(np.uint32), ref.view(np.uint32))
    assert rr.lib().rr_pathtracer_set_variants(ctx.handle, rr.PT_VARIANT_COUNT, 0) == 1
    ctx.check(rr.lib().rr_pathtracer_set_variants(ctx.handle, 0, 0))


def test_shadow_overlap_is_bit_identical(rr, O, ctx, torch_cuda, procedural):
    """Bounce b's shadow rays on the context's second stream next to bounce
    b+1's extension rays (the default) render the same bits as one stream, as
    the stage-timed form, and as the oracle; repeated frames at a size where
    the two launches do overlap."""
    torch = torch_cuda
    _, scene, oscene = procedural
    L = rr.lib()
    cam = cam_for(rr, "procedural", 80, 48)
    ref, _ = O.pathtrace(oscene, cam, 21, 6, 1)
    ctx.check(L.rr_pathtracer_set_overlap(ctx.handle, 1))
    g = gpu_pathtrace(rr, ctx, scene, cam, torch, 21, 6, 1)
    np.testing.assert_array_equal(g.view(np.uint32), ref.view(np.uint32))
    big = cam_for(rr, "procedural", 640, 360)
    outs = {}
    for name, overlap, flags in (("overlap", 1, 0), ("serial", 0, 0), ("timed", 1, rr.PT_FLAG_TIME_STAGES)):
        ctx.check(L.rr_pathtracer_set_overlap(ctx.handle, overlap))
        frames = []
        for f in range(3):
            out = torch.empty((4, 360, 640, 4), device="cuda")
            p = rr.PtParams(100 + 4 * f, 6, 4, flags)
            ctx.check(L.rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(big), C.byref(p), out.data_ptr(),
                                              _stream(torch)))
            frames.append(out)
        torch.cuda.synchronize()
        outs[name] = np.stack([_np(o) for o in frames])
    ctx.check(L.rr_pathtracer_set_overlap(ctx.handle, 1))
    assert np.isfinite(outs["serial"]).all() and outs["serial"][..., :3].mean() > 0
    for name in ("overlap", "timed"):
        np.testing.assert_array_equal(outs[name].view(np.uint32), outs["serial"].view(np.uint32), err_msg=name)


def test_pathtracer_in_a_captured_cuda_graph(rr, O, ctx, torch_cuda, procedural):
    """rr_pathtracer_execute captured into a CUDA graph on the caller's stream
    (the shadow overlap forks to the context's second stream and joins back
    inside the capture) replays to the same bits as a direct call."""
    torch = torch_cuda
    L = rr.lib()
    _, scene, _ = procedural
    cam = cam_for(rr, "procedural", 160, 96)
    ctx.check(L.rr_pathtracer_set_overlap(ctx.handle, 1))
    direct = gpu_pathtrace(rr, ctx, scene, cam, torch, 31, 5, 2)       # also sizes the queues
    out = torch.full((2, 96, 160, 4), -1.0, device="cuda")
    p = rr.PtParams(31, 5, 2, 0)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            ctx.check(L.rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), out.data_ptr(),
                                              side.cuda_stream))
    torch.cuda.current_stream().wait_stream(side)
    for _ in range(2):
        out.fill_(-1.0)
        graph.replay()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(_np(out).view(np.uint32), direct.view(np.uint32))
    del graph


def _edge_scenes(rr):
    """Cornell variants: a directional plus a point light (the MIS branch of
    the light sample and of ReSTIR DI's target), no lights at all, and all
    geometry moved out of view (every ray misses)."""
    base = rr.HostScene.cornell(0).arrays
    two = np.zeros(2, rr.LIGHT)
    two[0]["position"] = (0.0, 0.0, 0.0)
    two[0]["type"] = 1
    two[0]["direction"] = (0.3, -1.0, -0.2)
    two[0]["emission"] = (1.0, 0.9, 0.8)
    two[0]["intensity"] = 2.5
    two[1] = base["lights"][0]
    out = {"directional": dict(base, lights=two),
           "no_lights": dict(base, lights=np.zeros(0, rr.LIGHT))}
    away = base["instances"].copy()
    away["transform"][:, 3] += 1000.0      # every instance far off to the side: no ray hits
    out["no_geometry"] = dict(base, instances=away)
    return out


@pytest.mark.parametrize("name", ["cornell", "cornell_emitters_only", "procedural", "procedural_emitters_only",
                                  "no_lights"])
def test_restir_di_emitters_bit_exact(rr, O, ctx, torch_cuda, procedural, name):
    """RR_DI_FLAG_EMITTERS (candidates from the GpuLights and the emissive
    triangles, each a 32-bit state decoded wherever it is reused) against the
    oracle over three frames at the benchmarked M=32 / K=5 / R=30."""
    torch = torch_cuda
    cornell = rr.HostScene.cornell(0).arrays
    scenes = {"cornell": (cornell, "cornell"), "procedural": (procedural[0], "procedural"),
              "cornell_emitters_only": (dict(cornell, lights=np.zeros(0, rr.LIGHT)), "cornell"),
              "procedural_emitters_only": (dict(procedural[0], lights=np.zeros(0, rr.LIGHT)), "procedural"),
              "no_lights": (_edge_scenes(rr)["no_lights"], "cornell")}
    arrays, view = scenes[name]
    scene = rr.Scene(ctx, arrays)
    osc = O.OracleScene(arrays)
    cam = cam_for(rr, view, 64, 48)
    plist_g = [rr.DIParams(f, 32, 1, 1, 5, 30, 20, rr.DI_FLAG_EMITTERS) for f in range(3)]
    plist_o = [O.di_params(f, 32, 1, 1, 5, 30, 20, flags=O.DI_EMITTERS) for f in range(3)]
    g = _di_run_gpu(rr, ctx, torch_cuda, scene, cam, plist_g)
    o = _di_run_oracle(O, osc, cam, plist_o)
    for (gg, go) in zip(g, o):
        for a, b in zip(gg, go):
            np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    if name != "no_lights":
        assert float(o[-1][3][..., :3].mean()) > 0.0
    scene.close()


@pytest.mark.parametrize("name", ["cornell", "cornell_emitters_only", "procedural", "procedural_emitters_only",
                                  "directional", "no_lights", "no_geometry"])
def test_pathtracer_emitters_bit_exact(rr, O, ctx, torch_cuda, procedural, name):
    """RR_PT_FLAG_EMITTERS (next-event estimation over the GpuLights and the
    emissive triangles, MIS with bounces weighted by brdf_sample's actual
    density) against the oracle: both light groups, emissive triangles
    only, GpuLights only (directional MIS branch), nothing to sample, nothing
    in view."""
    torch = torch_cuda
    cornell = rr.HostScene.cornell(0).arrays
    scenes = {"cornell": (cornell, "cornell", 8), "procedural": (procedural[0], "procedural", 5),
              "cornell_emitters_only": (dict(cornell, lights=np.zeros(0, rr.LIGHT)), "cornell", 8),
              "procedural_emitters_only": (dict(procedural[0], lights=np.zeros(0, rr.LIGHT)), "procedural", 5)}
    edge = _edge_scenes(rr)
    arrays, view, depth = scenes[name] if name in scenes else (edge[name], "cornell", 6)
    scene = rr.Scene(ctx, arrays)
    osc = O.OracleScene(arrays)
    W, H = 56, 40
    cam = cam_for(rr, view, W, H)
    out = torch.empty((3, H, W, 4), device="cuda")
    ctx.check(rr.lib().rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam),
                                             C.byref(rr.PtParams(7, depth, 3, rr.PT_FLAG_EMITTERS)), out.data_ptr(),
                                             _stream(torch)))
    torch.cuda.synchronize()
    want, _ = O.pathtrace(osc, cam, 7, depth, 3, flags=O.PT_EMITTERS)
    np.testing.assert_array_equal(_np(out).view(np.uint32), want.view(np.uint32))
    if name in ("cornell", "procedural"):
        assert float(want[..., :3].mean()) > 0.0
    scene.close()


@pytest.mark.parametrize("name", ["directional", "no_lights", "no_geometry"])
def test_edge_scenes_bit_exact(rr, O, ctx, torch_cuda, name):
    torch = torch_cuda
    arrays = _edge_scenes(rr)[name]
    scene = rr.Scene(ctx, arrays)
    osc = O.OracleScene(arrays, use_bvh=False)
    cam = cam_for(rr, "cornell", 40, 32)
    g = gpu_pathtrace(rr, ctx, scene, cam, torch, 4, 6, 2)
    o, _ = O.pathtrace(osc, cam, 4, 6, 2)
    np.testing.assert_array_equal(g.view(np.uint32), o.view(np.uint32))
    plist_g = [rr.DIParams(f, 8, 1, 1, 4, 10, 20, 0) for f in range(2)]
    plist_o = [O.di_params(f, 8, 1, 1, 4, 10, 20) for f in range(2)]
    for a, b in zip(_di_run_gpu(rr, ctx, torch, scene, cam, plist_g)[-1], _di_run_oracle(O, osc, cam, plist_o)[-1]):
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    if name == "no_geometry":
        assert np.isfinite(g).all() and g[..., :3].min() > 0.05      # sky everywhere
        # a scene without instances is refused, as Scene::upload throws (Scene.cpp:261-262)
        with pytest.raises(rr.RRError):
            rr.Scene(ctx, dict(arrays, instances=np.zeros(0, arrays["instances"].dtype)))
    else:
        assert g[..., :3].mean() > 0.01
    scene.close()
