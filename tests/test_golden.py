"""Fixtures of tests/golden/: outputs of the reference's own shader text,
rewritten to C++ and run on the CPU by tests/golden/make_golden.py, on small
seeded inputs. The reference-text run and the oracle must still produce them
bit for bit, and so must the CUDA kernels through the C ABI."""
import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import make_golden  # noqa: E402


def _load(name):
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def _same(a, b, what):
    a, b = np.ascontiguousarray(a, np.float32), np.ascontiguousarray(b, np.float32)
    assert a.shape == b.shape, what
    bad = np.argwhere(a.view(np.uint32) != b.view(np.uint32))
    assert bad.size == 0, f"{what}: {len(bad)} words differ, first at {tuple(bad[0])}"


def test_oracle_reproduces_golden(rr, O):
    got = make_golden.compute(rr, O)
    for name, arrays in got.items():
        ref = _load(name)
        for k, v in arrays.items():
            _same(v, ref[k], f"{name}.{k}")
    # the fixtures are not trivial
    assert _load("cornell_pt")["images"][..., :3].mean() > 0.05
    assert (_load("restir_di")["gbuf_pos"][..., 3] > 0).mean() > 0.5


def test_reference_text_reproduces_golden(rr, O):
    import slang_ref
    if not slang_ref.available():
        pytest.skip("the reference checkout is not present")
    got = make_golden.compute_reference_text(rr, O, slang_ref)
    for name, arrays in got.items():
        ref = _load(name)
        for k, v in arrays.items():
            _same(v, ref[k], f"{name}.{k}")


@pytest.mark.gpu
def test_gpu_reproduces_golden(rr, ctx, torch_cuda):
    torch = torch_cuda
    st = torch.cuda.current_stream().cuda_stream
    L = rr.lib()
    hs = rr.HostScene.cornell(0)
    scene = rr.Scene(ctx, hs.arrays)
    c = make_golden.CORNELL_PT
    cam = rr.camera_data(rr.camera_desc(c["width"], c["height"]))
    out = torch.empty((c["spp"], c["height"], c["width"], 4), device="cuda")
    p = rr.PtParams(c["frame_seed"], c["max_bounces"], c["spp"], 0)
    ctx.check(L.rr_pathtracer_execute(ctx.handle, scene.handle, C.byref(cam), C.byref(p), out.data_ptr(), st))
    torch.cuda.synchronize()
    _same(out.cpu().numpy(), _load("cornell_pt")["images"], "cornell_pt.images")

    d = make_golden.DI
    W, H = d["width"], d["height"]
    cam = rr.camera_data(rr.camera_desc(W, H))
    dp = rr.DIParams(d["frame_seed"], d["candidates"], 1, 1, d["neighbors"], d["radius"], 20, 0)
    z = lambda: torch.zeros((H, W, 4), device="cuda")
    gpos, gnrm, res, out = z(), z(), z(), z()
    ctx.check(L.rr_restir_di_initial(ctx.handle, scene.handle, C.byref(cam), C.byref(dp), gpos.data_ptr(),
                                     gnrm.data_ptr(), res.data_ptr(), st))
    ctx.check(L.rr_restir_di_spatial_shade(ctx.handle, scene.handle, C.byref(cam), C.byref(dp), gpos.data_ptr(),
                                           gnrm.data_ptr(), res.data_ptr(), out.data_ptr(), st))
    torch.cuda.synchronize()
    ref = _load("restir_di")
    for k, t in (("gbuf_pos", gpos), ("gbuf_norm", gnrm), ("reservoir", res), ("output", out)):
        _same(t.cpu().numpy(), ref[k], f"restir_di.{k}")

    ping = [torch.empty_like(out), torch.empty_like(out)]
    ap = rr.AtrousParams(W, H, make_golden.ATROUS_ITERATIONS, 0, 0.25, 0.20, 1.0, 0)
    slot = C.c_uint32()
    ctx.check(L.rr_atrous_execute(ctx.handle, out.data_ptr(), gpos.data_ptr(), gnrm.data_ptr(), ping[0].data_ptr(),
                                  ping[1].data_ptr(), C.byref(ap), C.byref(slot), st))
    torch.cuda.synchronize()
    _same(ping[slot.value].cpu().numpy(), _load("atrous")["output"], "atrous.output")
    scene.close()
    hs.close()
