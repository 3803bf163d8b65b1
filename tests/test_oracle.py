"""CPU checks of the oracle itself: known-answer vectors and analytic properties.

The reference ships no tests or golden vectors; the RNG known answers below
were computed from the formula of Common.slang:18-28 / Sampling.slang:11-30
(pcg_hash, make_seed, rand_float) in 32-bit unsigned arithmetic, and are also
re-derived here by an independent pure-Python restatement.
"""
import math

import numpy as np
import pytest

# (input, pcg_hash(input))
PCG_KAT = [(0, 0x07BB2FE2), (1, 0xA8BEEA3C), (2, 0x7A7ECC88), (0xFFFFFFFF, 0xE62A4902), (12345, 0xF45EAD0E)]
# ((px, py, frame), make_seed, first two rand_float)
SEED_KAT = [((0, 0, 0), 0x07BB2FE2, 0.190399349, 0.499476671),
            ((1, 0, 0), 0xA8BEEA3C, 0.910801947, 0.138429046),
            ((0, 1, 0), 0x9734F28B, 0.268874466, 0.641497195),
            ((128, 128, 0), 0x3D67FDC9, 0.935119748, 0.568711281),
            ((0, 0, 1), 0x703CC78A, 0.98334682, 0.724128723)]


def py_pcg(x):
    s = (x * 747796405 + 2891336453) & 0xFFFFFFFF
    w = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & 0xFFFFFFFF
    return ((w >> 22) ^ w) & 0xFFFFFFFF


@pytest.mark.parametrize("x,h", PCG_KAT)
def test_pcg_hash_kat(O, x, h):
    assert O.pcg_hash(x) == h
    assert py_pcg(x) == h


@pytest.mark.parametrize("pix,seed,r0,r1", SEED_KAT)
def test_make_seed_and_rand_kat(O, pix, seed, r0, r1):
    assert O.make_seed(*pix) == seed
    h = (pix[0] ^ ((pix[1] * 1000003) & 0xFFFFFFFF) ^ ((pix[2] * 2654435761) & 0xFFFFFFFF)) & 0xFFFFFFFF
    assert py_pcg(h) == seed
    (a, b), _ = O.rand_floats(seed, 2)
    assert a == pytest.approx(r0, abs=5e-9) and b == pytest.approx(r1, abs=5e-9)
    # rand_float = (pcg(seed) >> 8) * 2^-24 exactly
    assert a == np.float32((py_pcg(seed) >> 8) * 2.0 ** -24)


def _ulp_err(y, ref):
    ref32 = ref.astype(np.float32)
    ulp = np.spacing(np.abs(ref32)).astype(np.float64)
    return np.abs(y.astype(np.float64) - ref) / ulp


def test_detmath_accuracy(O):
    x = np.linspace(0, 8 * math.pi, 400001, dtype=np.float32)
    assert _ulp_err(O.detmath("sin", x), np.sin(x.astype(np.float64))).max() <= 2.0
    assert _ulp_err(O.detmath("cos", x), np.cos(x.astype(np.float64))).max() <= 2.0
    e = np.linspace(-87, 88, 400001, dtype=np.float32)
    assert _ulp_err(O.detmath("exp", e), np.exp(e.astype(np.float64))).max() <= 2.0
    lg = (np.linspace(1e-3, 1, 400001) ** 3 * 1e3).astype(np.float32)
    lg = lg[lg != 1.0]
    assert _ulp_err(O.detmath("log", lg), np.log(lg.astype(np.float64))).max() <= 2.0
    # edge values
    assert O.detmath("log", np.array([0.0], np.float32))[0] == -np.inf
    assert O.detmath("exp", np.array([-200.0], np.float32))[0] == 0.0
    assert O.detmath("exp", np.array([0.0], np.float32))[0] == 1.0
    assert O.detmath("log", np.array([1.0], np.float32))[0] == 0.0


def _sphere_dirs(n, seed=0):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


@pytest.mark.parametrize("kappa", [0.5, 2.0, 10.0, 100.0])
def test_vmf_pdf_normalised(O, kappa):
    # integrate vMF pdf over the sphere by quadrature in cos(theta)
    mu = np.array([0.0, 0.0, 1.0], np.float32)
    ws = np.linspace(-1, 1, 20001)
    vals = [O.vmf_pdf(mu, kappa, np.array([math.sqrt(max(0, 1 - w * w)), 0.0, w], np.float32)) for w in ws]
    integral = 2 * math.pi * np.trapezoid(vals, ws)
    assert integral == pytest.approx(1.0, rel=2e-3)


def test_brdf_sample_pdf_and_value_consistent(O):
    # brdf_sample returns brdf_eval at the sampled direction (BRDF.slang:171)
    rng = np.random.default_rng(1)
    n = np.array([0, 0, 1], np.float32)
    for _ in range(200):
        wo = _sphere_dirs(1, rng.integers(1 << 30))[0]
        wo[2] = abs(wo[2]) + 0.05
        wo /= np.linalg.norm(wo)
        base = rng.uniform(0.05, 0.95, 3).astype(np.float32)
        m, r = float(rng.integers(0, 2)), float(rng.uniform(0.05, 1))
        wi, pdf, f = O.brdf_sample(wo, n, base, m, r, float(rng.random()), float(rng.random()))
        assert pdf >= 1e-6
        if np.any(f != 0):
            np.testing.assert_array_equal(f, O.brdf_eval(n, wo, wi, base, m, r))


def test_banerjee_fit_kappa(O):
    gp = O.guiding_params(cell_count=4, min_samples=1)
    accum = np.zeros((4, 4), np.int32)
    fitted = np.zeros((4, 4), np.float32)
    # cell 0: 10 identical +z splats -> r clamps to 0.9999 -> kappa clamps to kappa_max
    # cell 1: +x and -x -> r = 1e-4 -> kappa = 0.5 (clamp)
    accum[0] = [0, 0, 10 * (1 << 20), 10]
    accum[1] = [0, 0, 0, 2]
    accum[2] = [0, 0, 0, 0]
    O.guiding_fit(accum, fitted, gp)
    assert fitted[0, 3] == 512.0 and tuple(fitted[0, :3]) == (0.0, 0.0, 1.0)
    assert fitted[1, 3] == 0.5 and tuple(fitted[1, :3]) == (0.0, 0.0, 1.0)
    assert fitted[2, 3] == -1.0
    assert not accum.any()  # accumulators reset by the fit
    # closed form on a generic r
    r = np.float32(0.6)
    k = r * (np.float32(3) - r * r) / (np.float32(1) - r * r)
    accum[3] = [int(0.6 * (1 << 20)) * 100, 0, 0, 100]
    O.guiding_fit(accum, fitted, gp)
    assert fitted[3, 3] == pytest.approx(float(k), rel=1e-5)


def test_atrous_flat_image_is_fixed_point(O):
    # flat radiance + flat G-buffer: every tap weighs the same colour -> identity
    H, W = 32, 40
    inp = np.full((H, W, 4), 0.5, np.float32)
    gpos = np.zeros((H, W, 4), np.float32); gpos[..., 3] = 1.0
    gnrm = np.zeros((H, W, 4), np.float32); gnrm[..., 2] = 1.0
    out = O.atrous(inp, gpos, gnrm, 5)
    np.testing.assert_allclose(out, inp, rtol=1e-6)


def test_atrous_tap_weight_is_symmetric(O):
    """A pixel's tap on a neighbour weighs the same, bit for bit, as the
    neighbour's opposite tap on the pixel (what the pair-weight A-trous
    kernels rely on): random positions (small and far apart), unit normals,
    radiances over six decades, every offset, the library's default and
    extreme sigmas."""
    import ctypes as C
    lib = O.lib()
    rng = np.random.default_rng(17)
    fp = lambda a: np.ascontiguousarray(a, np.float32).ctypes.data_as(C.c_void_p)
    lum = lambda c: np.float32(np.float32(np.float32(c[0] * np.float32(0.299)) + np.float32(c[1] * np.float32(0.587)))
                               + np.float32(c[2] * np.float32(0.114)))
    n = 0
    for sig in ((0.25, 0.20, 1.0), (1e-3, 1e-3, 1e-3), (40.0, 3.0, 50.0)):
        sp2, sn2, sl2 = (max(np.float32(v) * np.float32(v), np.float32(1e-6)) for v in sig)
        for _ in range(400):
            scale = 10.0 ** rng.uniform(-3, 3)
            p, q = (rng.normal(size=3) * scale).astype(np.float32), (rng.normal(size=3) * scale).astype(np.float32)
            np_, nq = rng.normal(size=3), rng.normal(size=3)
            np_ = (np_ / np.linalg.norm(np_)).astype(np.float32)
            nq = (nq / np.linalg.norm(nq)).astype(np.float32)
            rp = (10.0 ** rng.uniform(-3, 3, 3)).astype(np.float32)
            rq = (10.0 ** rng.uniform(-3, 3, 3)).astype(np.float32)
            lp, lq = lum(rp), lum(rq)
            for ty in range(-2, 3):
                for tx in range(-2, 3):
                    a = lib.oracle_atrous_tap_weight(fp(p), fp(np_), lp, fp(q), fp(nq), fp(rq), tx, ty, sp2, sn2, sl2)
                    b = lib.oracle_atrous_tap_weight(fp(q), fp(nq), lq, fp(p), fp(np_), fp(rp), -tx, -ty, sp2, sn2, sl2)
                    assert np.float32(a).view(np.uint32) == np.float32(b).view(np.uint32), (a, b, tx, ty)
                    n += 1
    assert n == 3 * 400 * 25


def test_atrous_kernel_weights_sum_to_one():
    k = np.array([1, 4, 6, 4, 1], np.float32)
    assert (np.outer(k, k) / 256.0).sum() == 1.0


def test_accumulate_running_mean(O):
    rng = np.random.default_rng(3)
    frames = rng.random((5, 8, 8, 4)).astype(np.float32)
    acc = np.zeros((8, 8, 4), np.float32)
    for k in range(5):
        O.accumulate(np.ascontiguousarray(frames[k]), acc, 1 if k == 0 else 0, k)
    np.testing.assert_allclose(acc, frames.mean(0), rtol=1e-5)


def test_mlp_reference_gradient_finite_differences():
    """The FP64 reference gradient of the learned guide's loss agrees with
    central finite differences (it is the checker of the GPU backward pass)."""
    import mlp_ref
    rng = np.random.default_rng(0)
    params = rng.normal(size=mlp_ref.PARAM_COUNT) * 0.2
    N = 16
    pos = rng.uniform(-1, 1, (N, 3))
    nrm = rng.normal(size=(N, 3)); nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    wo = rng.normal(size=(N, 3)); wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    om = rng.normal(size=(N, 3)); om /= np.linalg.norm(om, axis=1, keepdims=True)
    w = rng.uniform(0.1, 1.0, N)
    F = mlp_ref.encode(pos, nrm, wo, np.array([-1.0] * 3), np.array([1.0] * 3))
    loss, g = mlp_ref.loss_and_grad(params, F, om, w)
    idx = rng.choice(mlp_ref.PARAM_COUNT, 40, replace=False)
    idx = np.concatenate([idx, [mlp_ref.PARAM_COUNT - 1, mlp_ref.PARAM_COUNT - 60]])
    for i in idx:
        h = 1e-6
        p1 = params.copy(); p1[i] += h
        p2 = params.copy(); p2[i] -= h
        fd = (mlp_ref.loss_and_grad(p1, F, om, w)[0] - mlp_ref.loss_and_grad(p2, F, om, w)[0]) / (2 * h)
        assert g[i] / mlp_ref.LOSS_SCALE == pytest.approx(fd, rel=1e-4, abs=1e-7)


@pytest.mark.parametrize("keep_point_light", [False, True])
def test_restir_di_emitter_candidates_are_unbiased(rr, O, keep_point_light):
    """Without reuse, ReSTIR DI's emitter candidates (ORACLE_DI_EMITTERS, M
    candidates, RIS) estimate the same direct light as the emitter-sampling
    path tracer at one bounce (light sample only, same primary rays for the
    same frame seed): the frame-averaged images agree."""
    hs = rr.HostScene.cornell(0)
    arrays = hs.arrays if keep_point_light else dict(hs.arrays, lights=hs.arrays["lights"][:0])
    osc = O.OracleScene(arrays, use_bvh=False)
    W = H = 16
    cam = rr.camera_data(rr.camera_desc(W, H))
    frames = 384
    z = lambda: np.zeros((H, W, 4), np.float32)
    di = np.zeros((H, W, 3))
    for f in range(frames):
        g, n, res, out = z(), z(), z(), z()
        p = O.di_params(f, 4, 0, 0, 0, 15, 20, flags=O.DI_EMITTERS)
        O.restir_di_initial(osc, cam, p, g, n, res)
        O.restir_di_spatial_shade(osc, cam, p, g, n, res, out)
        di += out[..., :3]
    di /= frames
    pt, _ = O.pathtrace(osc, cam, 0, 1, frames, flags=O.PT_EMITTERS)
    pt = pt[..., :3].mean(0)
    # the DI pass shades a missed pixel with the sky at the pixel centre and
    # the path tracer at the jittered ray: compare surface pixels
    surf = g[..., 3] >= 0
    md, mp = di[surf].mean(), pt[surf].mean()
    assert abs(md - mp) / mp < 0.02, (md, mp)


def test_emitter_alias_table_reproduces_the_power_distribution(rr, O):
    """The alias table the emitter sampling draws from picks emitter k with
    probability power_k / total (power = luminance(Le) * area), summed from the
    table's columns: (prob_k + sum over columns aliasing to k of 1 - prob_j) / n.
    On the procedural room's 4096 emitters of radiance log-uniform in
    [0.1, 100]."""
    hs = rr.HostScene.procedural(seed=0x5EED0002, target_triangles=20_000, emissive_triangles=4096,
                                 box_half=20.0, L=O.inputs_lib())
    osc = O.OracleScene(hs.arrays, use_bvh=False)
    rec, prob, alias, total = O.emitters(osc)
    n = len(prob)
    assert n >= 1000 and np.all((prob >= 0) & (prob <= 1)) and np.all(alias < n)
    e1, e2 = rec[:, 4:7].astype(np.float64), rec[:, 8:11].astype(np.float64)
    area = 0.5 * np.linalg.norm(np.cross(e1, e2), axis=1)
    le = rec[:, [3, 7, 11]].astype(np.float64)
    power = (0.2126 * le[:, 0] + 0.7152 * le[:, 1] + 0.0722 * le[:, 2]) * area
    implied = prob.astype(np.float64).copy()
    np.add.at(implied, alias, 1.0 - prob.astype(np.float64))
    implied -= np.where(alias == np.arange(n), 1.0 - prob, 0.0)   # a column's own alias adds nothing
    implied /= n
    np.testing.assert_allclose(implied, power / power.sum(), rtol=2e-5, atol=1e-9)
    assert abs(power.sum() - total) / total < 1e-5
    osc.close()
    hs.close()
