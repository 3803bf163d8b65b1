"""GPU tests of the path guides (dense vMF grid with FP64 EM, tensor-core
MLP) and of the guided path tracer."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


def make_guide(rr, ctx, kind, bmin=(-1, -1, -1), bmax=(1, 1, 1), max_samples=1 << 20, batch=1 << 18, res=16,
               lr=1e-2, decay=0.8, alpha=0.5):
    d = rr.GuideDesc(kind, res, alpha, decay, (C.c_float * 3)(*bmin), (C.c_float * 3)(*bmax), max_samples, batch,
                     lr, 7)
    h = C.c_void_p()
    ctx.check(rr.lib().rr_guide_create(ctx.handle, C.byref(d), C.byref(h)))
    return h


def set_samples(rr, ctx, torch, guide, pos, om, w, n_, wo):
    N = len(pos)
    s = np.zeros((N, 16), np.float32)
    s[:, 0:3] = pos; s[:, 3] = w
    s[:, 4:7] = om; s[:, 7] = np.arange(N, dtype=np.uint32).view(np.float32)
    s[:, 8:11] = n_
    s[:, 12:15] = wo
    t = torch.from_numpy(s).cuda()
    ctx.check(rr.lib().rr_guide_set_samples(ctx.handle, guide, t.data_ptr(), N, _stream(torch)))
    torch.cuda.synchronize()
    return t


def unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def eval_guide(rr, ctx, torch, guide, pos, n_, wo):
    N = len(pos)
    surf = np.zeros((N, 3, 4), np.float32)
    surf[:, 0, :3] = pos; surf[:, 0, 3] = 1
    surf[:, 1, :3] = n_; surf[:, 1, 3] = 1
    surf[:, 2, :3] = wo
    ts = torch.from_numpy(surf).cuda()
    mix = torch.zeros((N, 10, 4), device="cuda")
    ctx.check(rr.lib().rr_guide_eval(ctx.handle, guide, ts.data_ptr(), N, mix.data_ptr(), _stream(torch)))
    torch.cuda.synchronize()
    m = mix.cpu().numpy()
    return m[:, :8, :3], m[:, :8, 3], m[:, 8:, :].reshape(N, 8)


def test_mlp_forward_matches_fp64(rr, ctx, torch_cuda):
    import mlp_ref
    torch = torch_cuda
    g = make_guide(rr, ctx, rr.GUIDE_MLP)
    rng = np.random.default_rng(3)
    params = (rng.normal(size=mlp_ref.PARAM_COUNT) * 0.15).astype(np.float32)
    flag = C.c_int()
    ctx.check(rr.lib().rr_guide_mlp_params(ctx.handle, g, None, None, params.ctypes.data, rr.MLP_PARAM_COUNT,
                                           C.byref(flag)))
    N = 1000
    pos = rng.uniform(-1, 1, (N, 3)).astype(np.float32)
    nrm = unit(rng.normal(size=(N, 3))).astype(np.float32)
    wo = unit(rng.normal(size=(N, 3))).astype(np.float32)
    mu, kappa, pi = eval_guide(rr, ctx, torch, g, pos, nrm, wo)
    # reference on the BF16-rounded weights the tensor cores see
    p16 = torch.from_numpy(params).bfloat16().float().numpy().astype(np.float64)
    k = 0
    for i, o in mlp_ref.LAYERS:   # biases stay FP32
        p16[k + o * i:k + o * i + o] = params[k + o * i:k + o * i + o]
        k += o * i + o
    F = mlp_ref.encode(pos.astype(np.float64), nrm, wo, np.array([-1.0] * 3), np.array([1.0] * 3))
    raw, _ = mlp_ref.forward(p16, F)
    rmu, rk, rpi, _ = mlp_ref.mixture(raw)
    assert np.abs(pi - rpi).max() < 0.03
    assert np.abs(np.einsum("bjk,bjk->bj", mu, rmu)).min() > 0.97
    assert np.abs(kappa - rk).max() / rk.max() < 0.05
    ctx.check(rr.lib().rr_guide_mlp_params(ctx.handle, g, None, None, None, rr.MLP_PARAM_COUNT, C.byref(flag)))
    assert flag.value == 0
    rr.lib().rr_guide_destroy(g)


def _direction_samples(rng, N, axis):
    pos = rng.uniform(-1, 1, (N, 3)).astype(np.float32)
    om = unit(axis + 0.35 * rng.normal(size=(N, 3))).astype(np.float32)
    nrm = np.tile(np.array([0, 1, 0], np.float32), (N, 1))
    wo = unit(rng.normal(size=(N, 3)) + np.array([0, 2, 0])).astype(np.float32)
    w = rng.uniform(0.1, 2.0, N).astype(np.float32)
    return pos, om, nrm, wo, w


@pytest.mark.parametrize("N", [100, 2000, 148 * 32 * 9 + 17])
def test_mlp_gradient_matches_fp64(rr, ctx, torch_cuda, N):
    """N = 100: less than one 128-sample tile (the backward's copies map a
    zeroed tail); 2000: a ragged last tile, one or two tiles per
    warpgroup; 42,641: several tiles per warpgroup, so the dW products of
    the CTA's warpgroups are chained over many tiles, and a ragged last
    tile."""
    import mlp_ref
    torch = torch_cuda
    rng = np.random.default_rng(5)
    g = make_guide(rr, ctx, rr.GUIDE_MLP, batch=N, max_samples=N)
    params = (rng.normal(size=mlp_ref.PARAM_COUNT) * 0.1).astype(np.float32)
    ctx.check(rr.lib().rr_guide_mlp_params(ctx.handle, g, None, None, params.ctypes.data, rr.MLP_PARAM_COUNT, None))
    pos, om, nrm, wo, w = _direction_samples(rng, N, np.array([0.3, 1.0, 0.2]))
    keep = set_samples(rr, ctx, torch, g, pos, om, w, nrm, wo)
    ctx.check(rr.lib().rr_guide_update(ctx.handle, g, _stream(torch)))
    grad = np.zeros(mlp_ref.PARAM_COUNT, np.float32)
    flag = C.c_int()
    ctx.check(rr.lib().rr_guide_mlp_params(ctx.handle, g, None, grad.ctypes.data, None, rr.MLP_PARAM_COUNT,
                                           C.byref(flag)))
    assert flag.value == 0
    p16 = torch.from_numpy(params).bfloat16().float().numpy().astype(np.float64)
    k = 0
    for i, o in mlp_ref.LAYERS:
        p16[k + o * i:k + o * i + o] = params[k + o * i:k + o * i + o]
        k += o * i + o
    F = mlp_ref.encode(pos.astype(np.float64), nrm, wo, np.array([-1.0] * 3), np.array([1.0] * 3))
    loss, ref = mlp_ref.loss_and_grad(p16, F, om.astype(np.float64), w.astype(np.float64))
    cos = float(grad @ ref / (np.linalg.norm(grad) * np.linalg.norm(ref)))
    rel = float(np.linalg.norm(grad - ref) / np.linalg.norm(ref))
    assert cos > 0.99, (cos, rel)
    assert rel < 0.1, (cos, rel)
    # every layer's weights and biases on their own: one wrong block (a bias
    # column, a transposed layer) cannot hide under the global norm
    per_block = {}
    k = 0
    for li, (i, o) in enumerate(mlp_ref.LAYERS):
        for name, sl in (("W", slice(k, k + o * i)), ("b", slice(k + o * i, k + o * i + o))):
            a, b = grad[sl].astype(np.float64), ref[sl]
            nb = np.linalg.norm(b)
            per_block[f"layer{li}.{name}"] = (float(a @ b / (np.linalg.norm(a) * nb)), float(np.linalg.norm(a - b) / nb))
        k += o * i + o
    bad = {n: e for n, e in per_block.items() if not (e[0] > 0.99 and e[1] < 0.1)}
    assert not bad, per_block
    st = rr.GuideStats()
    ctx.check(rr.lib().rr_guide_get_stats(ctx.handle, g, C.byref(st)))
    assert st.last_loss == pytest.approx(loss, rel=0.05)
    # a second guide with the same parameters and samples gets the same
    # gradient bits: the warpgroups' shared weight-gradient sums run in a
    # fixed order
    g2 = make_guide(rr, ctx, rr.GUIDE_MLP, batch=N, max_samples=N)
    ctx.check(rr.lib().rr_guide_mlp_params(ctx.handle, g2, None, None, params.ctypes.data, rr.MLP_PARAM_COUNT, None))
    keep2 = set_samples(rr, ctx, torch, g2, pos, om, w, nrm, wo)
    ctx.check(rr.lib().rr_guide_update(ctx.handle, g2, _stream(torch)))
    grad2 = np.zeros(mlp_ref.PARAM_COUNT, np.float32)
    ctx.check(rr.lib().rr_guide_mlp_params(ctx.handle, g2, None, grad2.ctypes.data, None, rr.MLP_PARAM_COUNT, None))
    assert np.array_equal(grad.view(np.uint32), grad2.view(np.uint32))
    del keep, keep2
    rr.lib().rr_guide_destroy(g)
    rr.lib().rr_guide_destroy(g2)


def test_mlp_training_lowers_loss(rr, ctx, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(6)
    N = 1 << 16
    g = make_guide(rr, ctx, rr.GUIDE_MLP, batch=1 << 14, max_samples=N, lr=5e-3)
    pos, om, nrm, wo, w = _direction_samples(rng, N, np.array([0.0, 1.0, 0.0]))
    # direction depends on position: two half-spaces, two lobes
    om[pos[:, 0] > 0] = unit(np.array([1.0, 0.3, 0.0]) + 0.2 * rng.normal(size=((pos[:, 0] > 0).sum(), 3)))
    keep = set_samples(rr, ctx, torch, g, pos, om, w, nrm, wo)
    losses = []
    for it in range(60):
        ctx.check(rr.lib().rr_guide_update(ctx.handle, g, _stream(torch)))
        st = rr.GuideStats()
        ctx.check(rr.lib().rr_guide_get_stats(ctx.handle, g, C.byref(st)))
        losses.append(st.last_loss)
    assert losses[-1] < losses[0] - 1.0, losses[::10]
    # the learned mixture points where the data points
    mu, kappa, pi = eval_guide(rr, ctx, torch, g, np.array([[0.5, 0, 0], [-0.5, 0, 0]], np.float32),
                               np.array([[0, 1, 0]] * 2, np.float32), np.array([[0, 1, 0]] * 2, np.float32))
    mean_dir = [unit((pi[i][:, None] * mu[i]).sum(0)) for i in range(2)]
    assert mean_dir[0] @ unit(np.array([1.0, 0.3, 0.0])) > 0.8
    assert mean_dir[1] @ np.array([0.0, 1.0, 0.0]) > 0.8
    del keep
    rr.lib().rr_guide_destroy(g)


def test_grid_em_fits_and_is_deterministic(rr, ctx, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(8)
    N = 1 << 16
    pos, om, nrm, wo, w = _direction_samples(rng, N, np.array([0.0, 0.0, 1.0]))
    out = []
    for rep in range(2):
        g = make_guide(rr, ctx, rr.GUIDE_GRID, res=4)
        keep = set_samples(rr, ctx, torch, g, pos, om, w, nrm, wo)
        for it in range(3):
            ctx.check(rr.lib().rr_guide_update(ctx.handle, g, _stream(torch)))
        st = rr.GuideStats()
        ctx.check(rr.lib().rr_guide_get_stats(ctx.handle, g, C.byref(st)))
        assert st.cells_valid == 64
        mu, kappa, pi = eval_guide(rr, ctx, torch, g, pos[:200], nrm[:200], wo[:200])
        out.append((mu, kappa, pi))
        del keep
        rr.lib().rr_guide_destroy(g)
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
    mu, kappa, pi = out[0]
    mean_dir = unit((pi[:, :, None] * mu).sum(1))
    assert (mean_dir @ np.array([0, 0, 1.0])).min() > 0.9


def _em_step_fp64(om, w):
    """One EM update of a never-fitted cell in FP64: responsibilities under 8
    kappa-2 lobes on the cube diagonals, then Banerjee's kappa and the
    normalised lobe masses (the grid guide's update, restated)."""
    k = 1 / np.sqrt(3.0)
    mu0 = np.array([[k if j & 1 else -k, k if j & 2 else -k, k if j & 4 else -k] for j in range(8)])
    kap0 = 2.0
    pdf = kap0 * np.exp(kap0 * (om @ mu0.T - 1)) / (2 * np.pi * (1 - np.exp(-2 * kap0)))
    gam = pdf / pdf.sum(1, keepdims=True)
    r = w[:, None] * gam
    s0 = r.sum(0)
    s1 = r.T @ om
    ln = np.linalg.norm(s1, axis=1)
    rb = np.clip(ln / s0, 1e-4, 0.9999)
    kappa = np.clip(rb * (3 - rb * rb) / (1 - rb * rb), 0.5, 512.0)
    return s1 / ln[:, None], kappa, s0 / s0.sum()


def test_grid_em_update_matches_fp64_restatement(rr, ctx, torch_cuda):
    """One update of a 2^3 grid against the FP64 restatement, with cells of
    very uneven sample counts (a few samples to 40k) so that the chunked
    reduction runs with one and with many chunks per cell."""
    torch = torch_cuda
    rng = np.random.default_rng(21)
    counts = [3, 17, 1000, 1025, 4096, 40000, 0, 250]
    pos, om, w = [], [], []
    for c, n in enumerate(counts):
        lo = np.array([(c & 1) - 1.0, ((c >> 1) & 1) - 1.0, ((c >> 2) & 1) - 1.0])
        pos.append(lo + rng.uniform(0.05, 0.95, (n, 3)))
        axis = unit(rng.normal(size=3))
        om.append(unit(axis + 0.6 * rng.normal(size=(n, 3))))
        w.append(rng.uniform(0.1, 2.0, n))
    pos, om, w = (np.concatenate(a) for a in (pos, om, w))
    N = len(pos)
    nrm = np.tile([0.0, 0.0, 1.0], (N, 1)); wo = nrm
    g = make_guide(rr, ctx, rr.GUIDE_GRID, res=2, max_samples=1 << 16)
    keep = set_samples(rr, ctx, torch, g, pos.astype(np.float32), om.astype(np.float32), w.astype(np.float32),
                       nrm.astype(np.float32), wo.astype(np.float32))
    ctx.check(rr.lib().rr_guide_update(ctx.handle, g, _stream(torch)))
    st = rr.GuideStats()
    ctx.check(rr.lib().rr_guide_get_stats(ctx.handle, g, C.byref(st)))
    assert st.cells_valid == sum(1 for n in counts if n > 0)
    start = 0
    for c, n in enumerate(counts):
        centre = np.array([[(c & 1) - 0.5, ((c >> 1) & 1) - 0.5, ((c >> 2) & 1) - 0.5]], np.float32)
        mu, kappa, pi = eval_guide(rr, ctx, torch, g, centre, nrm[:1].astype(np.float32), wo[:1].astype(np.float32))
        if n == 0:
            assert pi.sum() == 0.0
            continue
        f32 = slice(start, start + n)
        rmu, rk, rpi = _em_step_fp64(om[f32].astype(np.float32).astype(np.float64),
                                     w[f32].astype(np.float32).astype(np.float64))
        np.testing.assert_allclose(pi[0], rpi, rtol=2e-5, atol=1e-6)
        np.testing.assert_allclose(mu[0], rmu, rtol=0, atol=2e-5)
        np.testing.assert_allclose(kappa[0], rk, rtol=2e-4)
        start += n
    del keep
    rr.lib().rr_guide_destroy(g)


def _render(rr, ctx, torch, scene, cam, frames, guide=None, train=True, spp=1, bounces=5, flags=0):
    W, H = cam.screen_width, cam.screen_height
    acc = np.zeros((H, W, 3))
    rad = torch.empty((spp, H, W, 4), device="cuda")
    for f in range(frames):
        p = rr.PtParams(1000 + f * spp, bounces, spp, flags)
        if guide is None:
            ctx.check(rr.lib().rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p),
                                                     rad.data_ptr(), _stream(torch)))
        else:
            ctx.check(rr.lib().rr_guided_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p),
                                                            guide, rad.data_ptr(), _stream(torch)))
            if train:
                ctx.check(rr.lib().rr_guide_update(ctx.handle, guide, _stream(torch)))
        acc += rad[..., :3].mean(0).cpu().numpy()
    return acc / frames


def metal_floor_arrays(rr, roughness=0.6):
    """A 100 x 100 rough-metal floor under the sky, no lights: every path is
    one GGX bounce seen at grazing angles, where the VNDF density brdf_sample
    draws from differs most from the density the reference divides by."""
    v = np.zeros(4, rr.VERTEX)
    v["pos"] = [(-50, 0, -50), (50, 0, -50), (50, 0, 50), (-50, 0, 50)]
    v["normal"] = (0, 1, 0)
    v["tangent"] = (1, 0, 0, 1)
    idx = np.array([0, 2, 1, 0, 3, 2], np.uint32)
    mesh = np.zeros(1, rr.MESH)
    mesh["vertex_count"], mesh["index_count"] = 4, 6
    mat = np.zeros(1, rr.MATERIAL)
    mat["base_color"] = (0.9, 0.9, 0.9, 1.0)
    mat["metallic"], mat["roughness"], mat["ior"] = 1.0, roughness, 1.5
    inst = np.zeros(1, rr.INSTANCE)
    inst["transform"] = np.eye(4, dtype=np.float32).ravel()
    return {"vertices": v, "indices": idx, "meshes": mesh, "materials": mat, "instances": inst,
            "lights": np.zeros(0, rr.LIGHT)}


@pytest.mark.parametrize("kind", ["grid", "mlp"])
def test_guided_matches_reference_expectation_on_ggx(rr, ctx, torch_cuda, kind):
    """On GGX the guided estimator converges to the reference tracer's own
    expectation (its weight carries the VNDF/reference density ratio and a
    rejected VNDF sample ends the path)."""
    torch = torch_cuda
    scene = rr.Scene(ctx, metal_floor_arrays(rr))
    cam = rr.camera_data(rr.camera_desc(64, 64, eye=(0.0, 1.0, 8.0), center=(0.0, 0.0, 0.0)))
    g = make_guide(rr, ctx, rr.GUIDE_GRID if kind == "grid" else rr.GUIDE_MLP, bmin=(-50.5, -1.0, -50.5),
                   bmax=(50.5, 1.0, 50.5), res=16, batch=1 << 14, max_samples=1 << 18)
    _render(rr, ctx, torch, scene, cam, 16, guide=g, train=True, spp=4)
    guided = _render(rr, ctx, torch, scene, cam, 64, guide=g, train=False, spp=4, bounces=2)
    plain = _render(rr, ctx, torch, scene, cam, 64, spp=4, bounces=2)
    floor = plain.sum(-1) != guided.sum(-1)             # pixels whose path reached the floor
    assert floor.mean() > 0.3
    mg, mp = guided[floor].mean(), plain[floor].mean()
    assert abs(mg - mp) / mp < 0.01, (mg, mp)
    rr.lib().rr_guide_destroy(g)
    scene.close()


@pytest.mark.parametrize("kind", ["grid", "mlp"])
def test_guided_training_is_deterministic(rr, ctx, torch_cuda, kind):
    """Two guides trained from the same guided frames end with the same
    mixtures bit for bit: the samples are compacted in record order, the
    grid's EM sums run in a fixed order and the MLP's gradients too."""
    torch = torch_cuda
    hs = rr.HostScene.cornell(1)
    scene = rr.Scene(ctx, hs.arrays)
    cam = rr.camera_data(rr.camera_desc(48, 48))
    guides = [make_guide(rr, ctx, rr.GUIDE_GRID if kind == "grid" else rr.GUIDE_MLP, bmin=(-1.01,) * 3,
                         bmax=(1.01,) * 3, res=16, batch=1 << 14, max_samples=1 << 18) for _ in range(2)]
    imgs = [_render(rr, ctx, torch, scene, cam, 3, guide=g, train=True, spp=4) for g in guides]
    assert np.array_equal(imgs[0], imgs[1])
    rng = np.random.default_rng(2)
    pos = rng.uniform(-0.9, 0.9, (512, 3)).astype(np.float32)
    nrm = unit(rng.normal(size=(512, 3))).astype(np.float32)
    wo = unit(rng.normal(size=(512, 3))).astype(np.float32)
    evs = [eval_guide(rr, ctx, torch, g, pos, nrm, wo) for g in guides]
    for a, b in zip(evs[0], evs[1]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert (evs[0][2] > 0).any()   # the guides hold mixtures
    for g in guides:
        rr.lib().rr_guide_destroy(g)
    scene.close()


@pytest.mark.parametrize("kind", ["grid", "mlp"])
def test_guided_pathtracer_is_unbiased(rr, ctx, torch_cuda, kind):
    torch = torch_cuda
    hs = rr.HostScene.cornell(1)
    scene = rr.Scene(ctx, hs.arrays)
    cam = rr.camera_data(rr.camera_desc(64, 64))
    g = make_guide(rr, ctx, rr.GUIDE_GRID if kind == "grid" else rr.GUIDE_MLP, bmin=(-1.01,) * 3,
                   bmax=(1.01,) * 3, res=16, batch=1 << 14, max_samples=1 << 18)
    _render(rr, ctx, torch, scene, cam, 16, guide=g, train=True, spp=4)          # learn
    guided = _render(rr, ctx, torch, scene, cam, 64, guide=g, train=False, spp=4)
    plain = _render(rr, ctx, torch, scene, cam, 64, spp=4)
    st = rr.GuideStats()
    ctx.check(rr.lib().rr_guide_get_stats(ctx.handle, g, C.byref(st)))
    assert st.samples_recorded > 1000
    # image means agree (MIS keeps the estimator unbiased for any guide)
    mg, mp = guided.mean(), plain.mean()
    assert abs(mg - mp) / mp < 0.03, (mg, mp)
    rr.lib().rr_guide_destroy(g)
    scene.close()


@pytest.mark.parametrize("kind", ["grid", "mlp"])
def test_guided_emitter_mode_is_unbiased(rr, ctx, torch_cuda, kind):
    """RR_PT_FLAG_EMITTERS in the guided tracer (emitter samples weighted
    against the guided mixture's density) converges to the unguided
    emitter-mode image: same mean on the Cornell box with its point light and
    emissive quad, and on the quad alone."""
    torch = torch_cuda
    base = rr.HostScene.cornell(1).arrays
    for arrays in (base, dict(base, lights=np.zeros(0, rr.LIGHT))):
        scene = rr.Scene(ctx, arrays)
        cam = rr.camera_data(rr.camera_desc(48, 48))
        g = make_guide(rr, ctx, rr.GUIDE_GRID if kind == "grid" else rr.GUIDE_MLP, bmin=(-1.01,) * 3,
                       bmax=(1.01,) * 3, res=16, batch=1 << 14, max_samples=1 << 18)
        E = rr.PT_FLAG_EMITTERS
        _render(rr, ctx, torch, scene, cam, 16, guide=g, train=True, spp=4, flags=E)
        guided = _render(rr, ctx, torch, scene, cam, 96, guide=g, train=False, spp=4, flags=E)
        plain = _render(rr, ctx, torch, scene, cam, 96, spp=4, flags=E)
        mg, mp = guided.mean(), plain.mean()
        assert abs(mg - mp) / mp < 0.02, (len(arrays["lights"]), mg, mp)
        rr.lib().rr_guide_destroy(g)
        scene.close()


@pytest.mark.parametrize("kind", ["grid", "mlp"])
def test_guided_shadow_overlap_is_bit_identical(rr, ctx, torch_cuda, kind):
    """The guided tracer with each bounce's shadow rays beside the next
    bounce's extension rays (the default) renders the same bits as with one
    stream, for a trained grid and a (fixed) MLP guide."""
    torch = torch_cuda
    L = rr.lib()
    hs = rr.HostScene.procedural(target_triangles=40_000, emissive_triangles=64, box_half=20.0)
    scene = rr.Scene(ctx, hs.arrays)
    cam = rr.camera_data(rr.camera_desc(160, 96, eye=(0.0, 4.0, 34.0), center=(0.0, -3.0, 0.0)))
    g = make_guide(rr, ctx, rr.GUIDE_GRID if kind == "grid" else rr.GUIDE_MLP, bmin=(-21.0,) * 3, bmax=(21.0,) * 3,
                   res=16, batch=1 << 14, max_samples=1 << 18)
    _render(rr, ctx, torch, scene, cam, 2, guide=g, train=True, spp=2)
    imgs = []
    for overlap in (1, 0):
        ctx.check(L.rr_pathtracer_set_overlap(ctx.handle, overlap))
        out = torch.empty((4, 96, 160, 4), device="cuda")
        p = rr.PtParams(77, 5, 4, 0)
        ctx.check(L.rr_guided_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), g,
                                                 out.data_ptr(), _stream(torch)))
        torch.cuda.synchronize()
        imgs.append(out.cpu().numpy())
    ctx.check(L.rr_pathtracer_set_overlap(ctx.handle, 1))
    assert np.array_equal(imgs[0].view(np.uint32), imgs[1].view(np.uint32))
    assert imgs[0][..., :3].mean() > 0
    L.rr_guide_destroy(g)
    scene.close()


def _frame_variance(rr, ctx, torch, scene, cam, frames, spp, guide=None, seed0=5000):
    """Mean over pixels of the variance between frame images (spp each), and
    the mean image."""
    W, H = cam.screen_width, cam.screen_height
    rad = torch.empty((spp, H, W, 4), device="cuda")
    imgs = []
    for f in range(frames):
        p = rr.PtParams(seed0 + f * spp, 5, spp, 0)
        if guide is None:
            ctx.check(rr.lib().rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p),
                                                     rad.data_ptr(), _stream(torch)))
        else:
            ctx.check(rr.lib().rr_guided_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p),
                                                            guide, rad.data_ptr(), _stream(torch)))
        imgs.append(rad[..., :3].mean(0).mean(-1).cpu().numpy().astype(np.float64))
    a = np.stack(imgs)
    return float(a.var(axis=0, ddof=1).mean()), a.mean(0)


def test_trained_mlp_guide_lowers_variance(rr, ctx, torch_cuda):
    """What the trained network gains over the method without it: on the
    Cornell box (config-1 light), after online training the MLP-guided
    tracer's per-pixel variance at equal spp (48 frames of 4 spp) is below
    that of the same network untrained and of the unguided tracer; all three
    agree in mean (the estimator is unbiased for any guide)."""
    torch = torch_cuda
    hs = rr.HostScene.cornell(1)
    scene = rr.Scene(ctx, hs.arrays)
    cam = rr.camera_data(rr.camera_desc(64, 64))
    kw = dict(bmin=(-1.01,) * 3, bmax=(1.01,) * 3, res=16, batch=1 << 14, max_samples=1 << 18)
    trained = make_guide(rr, ctx, rr.GUIDE_MLP, **kw)
    _render(rr, ctx, torch, scene, cam, 24, guide=trained, train=True, spp=4)
    untrained = make_guide(rr, ctx, rr.GUIDE_MLP, **kw)
    v_plain, m_plain = _frame_variance(rr, ctx, torch, scene, cam, 48, 4)
    v_untrained, m_untrained = _frame_variance(rr, ctx, torch, scene, cam, 48, 4, untrained)
    v_trained, m_trained = _frame_variance(rr, ctx, torch, scene, cam, 48, 4, trained)
    gain_plain, gain_untrained = v_plain / v_trained, v_untrained / v_trained
    print(f"variance: unguided {v_plain:.5g}, untrained MLP {v_untrained:.5g}, trained MLP {v_trained:.5g}; "
          f"gain {gain_plain:.3f}x over unguided, {gain_untrained:.3f}x over untrained")
    # measured 1.23x and 2.16x; the bounds leave room for the run-to-run
    # spread of online training and of the variance estimate
    assert gain_plain > 1.1 and gain_untrained > 1.5
    for m in (m_untrained, m_trained):
        assert abs(m.mean() - m_plain.mean()) / m_plain.mean() < 0.03
    for g in (trained, untrained):
        rr.lib().rr_guide_destroy(g)
    scene.close()


def test_bounded_mbarrier_wait_gives_up_and_reports(rr, ctx, torch_cuda):
    """A tensor-core wait on a barrier that nothing completes returns after its
    bound with the outcome recorded (no hang, no trap); the context stays usable."""
    import ctypes as C
    torch = torch_cuda
    out = (C.c_int * 2)(7, 7)
    ctx.check(rr.lib().rr_tc_wait_selftest(ctx.handle, 2000, out))
    assert list(out) == [0, 1]
    # the device still runs work afterwards
    a = torch.ones(1024, device="cuda")
    assert float((a * 2).sum()) == 2048.0
    with pytest.raises(rr.RRError):
        ctx.check(rr.lib().rr_tc_wait_selftest(ctx.handle, 0, out))

