"""The RenderPass adapters (research_b200/adapters/rr_passes.h) driven through
the reference renderer's own RenderGraph (src/render/RenderGraph.cpp,
compiled unmodified from the reference checkout into oracle/_ref/), with the
passes wired as the reference's Application wires them: path tracer →
accumulate, ReSTIR DI → A-trous. Both libraries are built here where the
reference's headers and RenderGraph.cpp exist; without them the tests skip.

CPU: every pass is a RenderPass with the reference pass's name and reflected
output, and execute() without a context returns silently with
RR_ERR_NOT_INITIALIZED (the reference's passes return silently when not
initialised). GPU: two frames through RenderGraph::execute, every image
bit-identical to the oracle.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GRAPH_LIB = ROOT / "oracle" / "_ref" / "librr_refgraph.so"
RGBA32F = 109   # rr::rhi::Format::R32G32B32A32_Sfloat (src/rhi/Types.h:42)
NAMES = [("PathTracerPass", "radiance_image"), ("AccumulatePass", "accumulated_image"),
         ("ReSTIRDIPass", "restir_di_output"), ("AtrousPass", "atrous_output")]


@pytest.fixture(scope="module")
def G(built, rr):
    if not GRAPH_LIB.exists():
        pytest.skip("the reference's RenderGraph was not built here (no reference checkout)")
    rr.lib()
    L = C.CDLL(str(GRAPH_LIB))
    P, U32 = C.c_void_p, C.c_uint32
    sig = {"rrg_create": (P, [P, P, U32, U32, U32, C.POINTER(U32), U32]), "rrg_destroy": (None, [P]),
           "rrg_pass_count": (C.c_int, [P]), "rrg_pass_name": (C.c_char_p, [P, C.c_int]),
           "rrg_pass_output": (C.c_char_p, [P, C.c_int, C.POINTER(C.c_int), C.POINTER(U32), C.POINTER(U32)]),
           "rrg_set_enabled": (None, [P, C.c_int, C.c_int]), "rrg_set_camera": (None, [P, P]),
           "rrg_set_stream": (None, [P, P]), "rrg_execute": (None, [P]), "rrg_status": (C.c_int, [P, C.c_int]),
           "rrg_image": (P, [P, C.c_int]), "rrg_read_image": (C.c_int, [P, C.c_int, P, C.c_size_t])}
    for k, (r, a) in sig.items():
        getattr(L, k).restype = r
        getattr(L, k).argtypes = a
    return L


def _di(m=8, k=4, r=15):
    return (C.c_uint32 * 3)(m, k, r)


def test_passes_are_reference_render_passes(G):
    g = G.rrg_create(None, None, 64, 48, 5, _di(), 5)
    try:
        assert G.rrg_pass_count(g) == 4
        for i, (name, out) in enumerate(NAMES):
            assert G.rrg_pass_name(g, i).decode() == name
            fmt, w, h = C.c_int(), C.c_uint32(), C.c_uint32()
            assert G.rrg_pass_output(g, i, C.byref(fmt), C.byref(w), C.byref(h)).decode() == out
            assert (fmt.value, w.value, h.value) == (RGBA32F, 64, 48)
        # not initialised (no context, scene or camera): each execute returns silently
        G.rrg_execute(g)
        assert [G.rrg_status(g, i) for i in range(4)] == [4, 4, 4, 4]   # RR_ERR_NOT_INITIALIZED
        # a disabled pass is skipped by RenderGraph::execute (RenderGraph.cpp:14-21)
        G.rrg_set_enabled(g, 0, 0)
        G.rrg_execute(g)
        assert G.rrg_status(g, 0) == 4
    finally:
        G.rrg_destroy(g)


@pytest.mark.gpu
def test_render_graph_frames_bit_exact(G, rr, O, ctx, torch_cuda):
    """Two frames of the Cornell box through RenderGraph::execute: each
    frame's radiance (1 spp, frame seed = the pass's frame counter), the
    running accumulation, the DI G-buffer and output (temporal reuse on the
    second frame) and the A-trous output equal the oracle's."""
    torch = torch_cuda
    hs = rr.HostScene.cornell(0)
    scene = rr.Scene(ctx, hs.arrays)
    osc = O.OracleScene(hs.arrays, use_bvh=False)
    W, H = 40, 32
    cam = rr.camera_data(rr.camera_desc(W, H))
    g = G.rrg_create(ctx.handle, scene.handle, W, H, 8, _di(16, 4, 15), 5)
    G.rrg_set_camera(g, C.byref(cam))
    G.rrg_set_stream(g, C.c_void_p(torch.cuda.current_stream().cuda_stream))

    def image(which):
        out = np.empty((H, W, 4), np.float32)
        assert G.rrg_read_image(g, which, out.ctypes.data, out.nbytes) == 0
        return out

    z = lambda: np.zeros((H, W, 4), np.float32)
    o_acc, o_g, o_n, o_out = z(), z(), z(), z()
    o_res = [z(), z()]
    try:
        for f in range(2):
            G.rrg_execute(g)
            torch.cuda.synchronize()
            assert [G.rrg_status(g, i) for i in range(4)] == [0, 0, 0, 0]
            rad, _ = O.pathtrace(osc, cam, f, 8, 1)
            O.accumulate(np.ascontiguousarray(rad[0]), o_acc, 1 if f == 0 else 0, f)
            p = O.di_params(f, 16, 1, 1, 4, 15, 20)
            cur, prev = o_res[f & 1], o_res[(f & 1) ^ 1]
            O.restir_di_initial(osc, cam, p, o_g, o_n, cur)
            O.restir_di_temporal(osc, cam, p, o_g, o_n, cur, prev)
            O.restir_di_spatial_shade(osc, cam, p, o_g, o_n, cur, o_out)
            o_den = O.atrous(o_out, o_g, o_n, 5)
            for which, want, what in ((0, rad[0], "radiance"), (1, o_acc, "accumulated"), (2, o_g, "G-buffer position"),
                                      (3, o_n, "G-buffer normal"), (4, o_out, "DI output"), (5, o_den, "A-trous")):
                got = image(which)
                assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"frame {f}: {what}"
    finally:
        G.rrg_destroy(g)
        scene.close()
