"""The oracle pinned to the reference's own shader text (CPU only).

oracle/make_ref.py rewrites the reference's .slang files (Common, Sampling,
BRDF, GuidingGrid, GpuScene, the path tracer, accumulate, ReSTIR DI, A-trous,
ReSTIR PT and ReSTIR GI) mechanically into C++; oracle/slang_ref_harness.cpp
runs their compute entry points over the same inputs as the hand-written
oracle (rr_oracle.cpp), with the same intersector standing in for the
reference's ray-tracing hardware. The hand-written oracle is the checker of
every GPU test, so these tests tie the GPU kernels, through it, to the
reference's source text. Tolerance zero: the same bits everywhere.

The rewrite needs the reference checkout; without it (and without a library
built earlier) the tests skip.
"""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def S(built):
    import slang_ref
    try:
        ok = slang_ref.available()
    except RuntimeError as e:
        pytest.fail(str(e))
    if not ok:
        pytest.skip("the reference checkout is not present: the reference-text checker cannot be built")
    slang_ref.lib()
    return slang_ref


def _same(a, b, what):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    ia, ib = a.view(np.uint32), b.view(np.uint32)
    bad = np.argwhere(ia != ib)
    assert bad.size == 0, f"{what}: {len(bad)} words differ, first at {tuple(bad[0])}: reference text " \
                          f"{a[tuple(bad[0])]} oracle {b[tuple(bad[0])]}"


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def test_rng_matches_reference_text(S, O):
    rng = np.random.default_rng(1)
    xs = rng.integers(0, 2**32, 4000, dtype=np.uint64)
    for x in xs:
        assert S.pcg_hash(int(x)) == O.pcg_hash(int(x))
    for px, py, f in rng.integers(0, 5000, (1000, 3)):
        assert S.make_seed(int(px), int(py), int(f)) == O.make_seed(int(px), int(py), int(f))
    s_ref, s_or = 12345, 12345
    for _ in range(500):
        r_ref, s_ref = S.rand_float(s_ref)
        (r_or,), s_or = O.rand_floats(s_or, 1)
        assert np.float32(r_ref).view(np.uint32) == np.float32(r_or).view(np.uint32) and s_ref == s_or


def test_brdf_matches_reference_text(S, O):
    """brdf_eval / brdf_sample / brdf_pdf (BRDF.slang) over random surfaces,
    directions, materials (rough and near-mirror, metallic and not) and
    random numbers, both sampling lobes included."""
    rng = np.random.default_rng(2)
    L = O.lib()
    f3 = lambda: np.zeros(3, np.float32)
    for k in range(3000):
        n = _unit(rng.normal(size=3)).astype(np.float32)
        wo = _unit(n + rng.normal(size=3) * 0.8).astype(np.float32)
        wi = _unit(rng.normal(size=3)).astype(np.float32)
        base = rng.uniform(0.0, 1.0, 3).astype(np.float32)
        metallic = float(np.float32(rng.choice([0.0, 1.0, rng.uniform()])))
        rough = float(np.float32(rng.choice([0.0, 0.02, rng.uniform(), 1.0])))
        u0, u1 = (float(np.float32(x)) for x in rng.uniform(0.0, 1.0, 2))
        o = f3()
        L.oracle_brdf_eval(n.ctypes.data, wo.ctypes.data, wi.ctypes.data, base.ctypes.data, metallic, rough,
                           o.ctypes.data)
        _same(S.brdf_eval(n, wo, wi, base, metallic, rough), o, f"brdf_eval case {k}")
        wi_o, f_o, pdf_o = f3(), f3(), np.zeros(1, np.float32)
        L.oracle_brdf_sample(wo.ctypes.data, n.ctypes.data, base.ctypes.data, metallic, rough, u0, u1,
                             wi_o.ctypes.data, pdf_o.ctypes.data, f_o.ctypes.data)
        wi_r, pdf_r, f_r = S.brdf_sample(wo, n, base, metallic, rough, u0, u1)
        _same(wi_r, wi_o, f"brdf_sample wi case {k}")
        _same(np.float32(pdf_r), pdf_o[0], f"brdf_sample pdf case {k}")
        _same(f_r, f_o, f"brdf_sample f case {k}")
        p_o = L.oracle_brdf_pdf(wo.ctypes.data, wi.ctypes.data, n.ctypes.data, rough)
        _same(np.float32(S.brdf_pdf(wo, wi, n, rough)), np.float32(p_o), f"brdf_pdf case {k}")


def test_guiding_grid_matches_reference_text(S, O):
    """guiding_cell_index, the fixed-point splat and the Banerjee fit
    (GuidingGrid.slang:54-137), and vmf_pdf (:182-189)."""
    rng = np.random.default_rng(3)
    cells = 1 << 10
    gp = O.guiding_params(cell_count=cells, min_samples=4)
    cam = np.array([0.3, 1.0, 4.0], np.float32)
    n = 30000
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(-3, 3, (n, 3))
    dirs = np.zeros((n, 4), np.float32)
    dirs[:, :3] = _unit(rng.normal(size=(n, 3)) + np.array([0.0, 1.5, 0.3]))
    bsdf = rng.integers(0, 5, n).astype(np.uint32)
    for i in range(0, n, 97):
        assert S.guiding_cell_index(pos[i, :3], int(bsdf[i]), cam, gp) == \
            O.guiding_cell_index(pos[i, :3], int(bsdf[i]), cam, gp)
    acc_r, acc_o = np.zeros((cells, 4), np.int32), np.zeros((cells, 4), np.int32)
    S.guiding_splat(acc_r, pos, dirs, bsdf, cam, gp)
    O.guiding_splat(acc_o, pos, dirs, bsdf, cam, gp)
    _same(acc_r, acc_o, "splat accumulators")
    fit_r, fit_o = np.zeros((cells, 4), np.float32), np.zeros((cells, 4), np.float32)
    S.guiding_fit(acc_r, fit_r, gp)
    O.guiding_fit(acc_o, fit_o, gp)
    _same(fit_r, fit_o, "fitted lobes")
    _same(acc_r, acc_o, "accumulators after the fit's reset")
    for k in range(2000):
        mu = _unit(rng.normal(size=3)).astype(np.float32)
        d = _unit(rng.normal(size=3)).astype(np.float32)
        kappa = float(np.float32(rng.choice([0.0, 1e-4, rng.uniform(0.5, 600.0)])))
        _same(np.float32(S.vmf_pdf(mu, kappa, d)), np.float32(O.vmf_pdf(mu, kappa, d)), f"vmf_pdf case {k}")


@pytest.fixture(scope="module")
def scenes(rr, O, S):
    out = {}
    for name, hs in (("cornell", rr.HostScene.cornell(0)),
                     ("procedural", rr.HostScene.procedural(seed=0x5EED0002, target_triangles=20_000,
                                                            emissive_triangles=64, box_half=20.0))):
        tracer = O.OracleScene(hs.arrays)
        out[name] = (hs.arrays, tracer, S.RefScene(hs.arrays, tracer))
    return out


def _cam(rr, name, W, H, move=0.0, prev=None):
    if name == "cornell":
        d = rr.camera_desc(W, H, eye=(0.0 + move, 0.0, 3.0 - 2.5 * move), center=(0.0, 0.0, 0.0))
    else:
        d = rr.camera_desc(W, H, eye=(0.0 + move, 4.0, 34.0 - 2.0 * move), center=(0.0, -3.0, 0.0))
    return d, rr.camera_data(d, prev)


@pytest.mark.parametrize("name", ["cornell", "procedural"])
def test_pathtracer_matches_reference_text(rr, O, S, scenes, name):
    """pathtracer.slang:cs_main (trace, sample_lights, the bounce loop with
    Russian roulette) for several frame seeds, full image and a region."""
    _, tracer, ref = scenes[name]
    W, H = 40, 28
    _, cam = _cam(rr, name, W, H)
    depth = 8 if name == "cornell" else 5
    got = S.pathtrace(ref, cam, 3, depth, 3)
    want, _ = O.pathtrace(tracer, cam, 3, depth, 3)
    _same(got, want, f"{name} path tracer")
    got = S.pathtrace(ref, cam, 11, depth, 1, region=(7, 5, 16, 9))
    want, _ = O.pathtrace(tracer, cam, 11, depth, 1, region=(7, 5, 16, 9))
    _same(got, want, f"{name} path tracer region")
    assert float(want[..., :3].mean()) > 0.0


def test_accumulate_matches_reference_text(S, O):
    rng = np.random.default_rng(4)
    H, W = 13, 17
    acc_r, acc_o = np.zeros((H, W, 4), np.float32), np.zeros((H, W, 4), np.float32)
    for f, moved in enumerate((1, 0, 0, 1, 0, 0, 0)):
        rad = rng.uniform(0, 3, (H, W, 4)).astype(np.float32)
        S.accumulate(rad, acc_r, moved, f)
        O.accumulate(rad, acc_o, moved, f)
        _same(acc_r, acc_o, f"accumulate frame {f}")


@pytest.mark.parametrize("name", ["cornell", "procedural"])
def test_restir_di_and_atrous_match_reference_text(rr, O, S, scenes, name):
    """cs_initial / cs_temporal / cs_spatial_shade (restir_di.slang) over
    three frames with M=32, K=5, R=30 (the benchmarked settings), then
    A-trous 5 iterations (atrous.slang) on the result."""
    _, tracer, ref = scenes[name]
    W, H = 36, 30
    _, cam = _cam(rr, name, W, H)
    z = lambda: np.zeros((H, W, 4), np.float32)
    R = dict(g=z(), n=z(), res=[z(), z()], out=z())
    Q = dict(g=z(), n=z(), res=[z(), z()], out=z())
    for f in range(3):
        p = O.di_params(f, 32, 1, 1, 5, 30, 20)
        c, pv = f & 1, (f & 1) ^ 1
        for stage in range(3):
            S.restir_di(stage, ref, cam, p, R["g"], R["n"], R["res"][c], R["res"][pv], R["out"])
        O.restir_di_initial(tracer, cam, p, Q["g"], Q["n"], Q["res"][c])
        O.restir_di_temporal(tracer, cam, p, Q["g"], Q["n"], Q["res"][c], Q["res"][pv])
        O.restir_di_spatial_shade(tracer, cam, p, Q["g"], Q["n"], Q["res"][c], Q["out"])
        for k in ("g", "n", "out"):
            _same(R[k], Q[k], f"{name} DI frame {f} {k}")
        _same(R["res"][c], Q["res"][c], f"{name} DI frame {f} reservoir")
    _same(S.atrous(R["out"], R["g"], R["n"], 5), O.atrous(Q["out"], Q["g"], Q["n"], 5), f"{name} A-trous")
    assert (Q["res"][0][..., 3].view(np.uint32) > 32).any()   # temporal history was merged


def _reuse_inputs(rr, O, tracer, cam, W, H, f):
    """G-buffer and direct light of the oracle's ReSTIR DI (the reuse passes' inputs)."""
    z = lambda: np.zeros((H, W, 4), np.float32)
    g, n, res, direct = z(), z(), z(), z()
    p = O.di_params(f, 8, 0, 0, 4, 15, 20)
    O.restir_di_initial(tracer, cam, p, g, n, res)
    O.restir_di_spatial_shade(tracer, cam, p, g, n, res, direct)
    return g, n, direct


@pytest.mark.parametrize("name", ["cornell", "procedural"])
def test_restir_pt_matches_reference_text(rr, O, S, scenes, name):
    """restir_pt.slang: cs_initial (guided first bounce, reconnection vertex,
    NEE), cs_temporal (reprojection, Jacobian), cs_spatial_shade (neighbour
    reconnection, guiding splat) and cs_fit_guiding, over three frames with a
    moving camera."""
    _, tracer, ref = scenes[name]
    W, H = 24, 20
    cells = 1 << 10
    z = lambda: np.zeros((H, W, 4), np.float32)
    sides = []
    for _ in range(2):
        st = dict(res=[[z() for _ in range(4)] for _ in range(2)], hist=[[z() for _ in range(2)] for _ in range(2)],
                  output=z(), accum=np.zeros((cells, 4), np.int32), fitted=np.zeros((cells, 4), np.float32))
        for h in st["hist"]:
            h[0][..., 3] = -1.0
        sides.append(st)
    gp = O.guiding_params(cell_count=cells, min_samples=2)
    p = O.pt_reuse_params(gp=gp)
    prev = None
    for f in range(3):
        desc, cam = _cam(rr, name, W, H, move=0.01 * f, prev=prev)
        g, n, direct = _reuse_inputs(rr, O, tracer, cam, W, H, f)
        p.frame_seed = f
        c, pv = f & 1, 1 - (f & 1)
        imgs = []
        for st in sides:
            imgs.append(dict(gbuf_pos=g, gbuf_norm=n, direct=direct, res_curr=st["res"][c], res_prev=st["res"][pv],
                             hist_curr=st["hist"][c], hist_prev=st["hist"][pv], output=st["output"],
                             accum=st["accum"], fitted=st["fitted"]))
        for stage, ofn in enumerate((O.restir_pt_initial, O.restir_pt_temporal, O.restir_pt_spatial_shade)):
            S.restir_pt(stage, ref, cam, p, O.pt_reuse_images(imgs[0]))
            ofn(tracer, cam, p, imgs[1])
            for k in range(4):
                _same(sides[0]["res"][c][k], sides[1]["res"][c][k], f"{name} PT frame {f} stage {stage} res[{k}]")
        for k in range(2):
            _same(sides[0]["hist"][c][k], sides[1]["hist"][c][k], f"{name} PT frame {f} history[{k}]")
        _same(sides[0]["output"], sides[1]["output"], f"{name} PT frame {f} output")
        _same(sides[0]["accum"], sides[1]["accum"], f"{name} PT frame {f} guiding accumulators")
        S.restir_pt(3, ref, cam, p, O.pt_reuse_images(imgs[0]))
        O.guiding_fit(sides[1]["accum"], sides[1]["fitted"], gp)
        _same(sides[0]["fitted"], sides[1]["fitted"], f"{name} PT frame {f} fitted lobes")
        prev = desc
    assert (sides[1]["fitted"][:, 3] > 0).any()


@pytest.mark.parametrize("name", ["cornell", "procedural"])
def test_restir_gi_matches_reference_text(rr, O, S, scenes, name):
    """restir_gi.slang: cs_initial (cosine candidates, light sample at the
    secondary hit), cs_temporal and cs_spatial_shade, over three frames with a
    moving camera."""
    _, tracer, ref = scenes[name]
    W, H = 24, 20
    z = lambda: np.zeros((H, W, 4), np.float32)
    sides = []
    for _ in range(2):
        st = dict(res=[[z() for _ in range(3)] for _ in range(2)], hist=[[z() for _ in range(2)] for _ in range(2)],
                  output=z())
        for h in st["hist"]:
            h[0][..., 3] = -1.0
        sides.append(st)
    p = O.gi_reuse_params()
    prev = None
    for f in range(3):
        desc, cam = _cam(rr, name, W, H, move=0.01 * f, prev=prev)
        g, n, direct = _reuse_inputs(rr, O, tracer, cam, W, H, f)
        p.frame_seed = f
        c, pv = f & 1, 1 - (f & 1)
        imgs = []
        for st in sides:
            imgs.append(dict(gbuf_pos=g, gbuf_norm=n, direct=direct, res_curr=st["res"][c], res_prev=st["res"][pv],
                             hist_curr=st["hist"][c], hist_prev=st["hist"][pv], output=st["output"]))
        for stage, ofn in enumerate((O.restir_gi_initial, O.restir_gi_temporal, O.restir_gi_spatial_shade)):
            S.restir_gi(stage, ref, cam, p, O.gi_reuse_images(imgs[0]))
            ofn(tracer, cam, p, imgs[1])
            for k in range(3):
                _same(sides[0]["res"][c][k], sides[1]["res"][c][k], f"{name} GI frame {f} stage {stage} res[{k}]")
        for k in range(2):
            _same(sides[0]["hist"][c][k], sides[1]["hist"][c][k], f"{name} GI frame {f} history[{k}]")
        _same(sides[0]["output"], sides[1]["output"], f"{name} GI frame {f} output")
        prev = desc
