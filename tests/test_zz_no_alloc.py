"""The allocation-free A-trous entry point (rr_atrous_execute_static).

It serves callers that may not allocate device memory themselves or let a
library do so (fixed engine memory budgets, hosts that forbid cudaMalloc
during rendering). The test calls it through the C ABI several times in a
row and checks each result against the CPU oracle's A-trous (the restatement
of atrous.slang) and against the regular rr_atrous_execute on the same
inputs, with the tolerance the other parity tests use: bit-identical. This
file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RR_ERR_INVALID_ARGUMENT, RR_ERR_UNSUPPORTED = 1, 7


def _inputs(rng, H, W):
    rad = (rng.random((H, W, 4)) * 4).astype(np.float32)
    gpos = np.zeros((H, W, 4), np.float32)
    gpos[..., :3] = rng.normal(size=(H, W, 3)) * 0.3
    gpos[..., 3] = rng.uniform(0.5, 5.0, (H, W))
    gpos[rng.random((H, W)) < 0.1, 3] = -1.0          # primary-ray misses
    n = rng.normal(size=(H, W, 3)) + np.array([0.0, 0.0, 3.0])
    gnrm = np.zeros((H, W, 4), np.float32)
    gnrm[..., :3] = n / np.linalg.norm(n, axis=-1, keepdims=True)
    gnrm[..., :3] *= rng.uniform(0.5, 2.0, (H, W, 1)).astype(np.float32)   # not unit: the filter normalizes
    return rad, gpos, gnrm


def test_static_atrous_matches_oracle_and_regular_entry_point(rr, O, ctx, torch_cuda):
    torch = torch_cuda
    L = rr.lib()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(1234)
    # calls in a row: an odd size, a 7-iteration run, then 1080p
    for H, W, iters in ((67, 91, 5), (203, 360, 7), (1080, 1920, 5)):
        a_rad, a_pos, a_nrm = _inputs(rng, H, W)
        want = O.atrous(a_rad, a_pos, a_nrm, iters)
        rad, gpos, gnrm = (torch.from_numpy(a).cuda() for a in (a_rad, a_pos, a_nrm))
        p = rr.AtrousParams(W, H, iters, 0, 0.25, 0.20, 1.0, 0)
        out = torch.full_like(rad, float("nan"))
        st = L.rr_atrous_execute_static(rad.data_ptr(), gpos.data_ptr(), gnrm.data_ptr(), out.data_ptr(),
                                        C.byref(p), stream)
        assert st == 0, rr.RR_STATUS.get(st, st)
        ping = [torch.empty_like(rad), torch.empty_like(rad)]
        slot = C.c_uint32()
        ctx.check(L.rr_atrous_execute(ctx.handle, rad.data_ptr(), gpos.data_ptr(), gnrm.data_ptr(),
                                      ping[0].data_ptr(), ping[1].data_ptr(), C.byref(p), C.byref(slot), stream))
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32), err_msg=f"{W}x{H} vs oracle")
        np.testing.assert_array_equal(got.view(np.uint32), ping[slot.value].cpu().numpy().view(np.uint32),
                                      err_msg=f"{W}x{H} vs rr_atrous_execute")


def test_static_atrous_rejects_oversized_and_bad_arguments(rr, ctx, torch_cuda):
    torch = torch_cuda
    L = rr.lib()
    buf = torch.zeros((4, 4, 4), device="cuda")
    other = torch.zeros((4, 4, 4), device="cuda")
    too_big = rr.AtrousParams(4096, 4096, 5, 0, 0.25, 0.2, 1.0, 0)
    assert L.rr_atrous_execute_static(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), other.data_ptr(),
                                      C.byref(too_big), None) == RR_ERR_UNSUPPORTED
    # few enough pixels, but taller than the launch grid allows
    tall = rr.AtrousParams(4, 589824, 5, 0, 0.25, 0.2, 1.0, 0)
    assert L.rr_atrous_execute_static(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), other.data_ptr(),
                                      C.byref(tall), None) == RR_ERR_INVALID_ARGUMENT
    ok = rr.AtrousParams(4, 4, 5, 0, 0.25, 0.2, 1.0, 0)
    assert L.rr_atrous_execute_static(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(),
                                      C.byref(ok), None) == RR_ERR_INVALID_ARGUMENT   # input aliases output
    big = torch.zeros((8, 4, 4), device="cuda")
    half = big[4:]                                                                    # overlaps the input's tail
    assert L.rr_atrous_execute_static(big.data_ptr() + 16 * 4, other.data_ptr(), other.data_ptr(), half.data_ptr(),
                                      C.byref(ok), None) == RR_ERR_INVALID_ARGUMENT
    assert L.rr_atrous_execute_static(buf.data_ptr(), other.data_ptr(), other.data_ptr(), other.data_ptr(),
                                      C.byref(ok), None) == RR_ERR_INVALID_ARGUMENT   # G-buffer is the output
    assert L.rr_atrous_execute_static(None, None, None, None, C.byref(ok), None) == RR_ERR_INVALID_ARGUMENT
