"""The replica (multi-GPU) bookkeeping of bench.py on CPU: two gloo ranks
exchange their step times, agree on the slowest, get disjoint frame-seed
ranges and report the whole-job throughput; a rank that fails is seen by the
other as an error of the next collective, not as a hang."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from research_b200 import replicas
    got_ws, got_rank, _ = replicas.init("gloo", timeout_s=60)
    replicas.barrier(got_ws)
    ms = 10.0 + 5.0 * rank            # rank 1 is the slow one
    ms_max = replicas.max_over_ranks(got_ws, ms, "cpu")
    value = replicas.job_throughput(1_000_000, got_ws, ms_max)
    q.put((got_rank, got_ws, replicas.seed_base(got_rank), ms_max, value))
    replicas.barrier(got_ws)
    replicas.finish(got_ws)


def _failing_rank(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from research_b200 import replicas
    replicas.init("gloo", timeout_s=10)
    replicas.barrier(ws)
    if rank == 1:
        raise SystemExit(3)           # leaves between steps, before the timing exchange
    try:
        replicas.max_over_ranks(ws, 1.0, "cpu")
        q.put(("no error", rank))
    except Exception as e:            # the collective fails instead of hanging
        q.put(("error", type(e).__name__))


def test_two_replicas_agree_on_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, ws0, s0, m0, v0), (r1, ws1, s1, m1, v1) = out
    assert (r0, r1, ws0, ws1) == (0, 1, 2, 2)
    assert m0 == m1 == 15.0                      # max over ranks, on every rank
    assert v0 == v1 == pytest.approx(2 * 1_000_000 / 15e-3 / 1e6)
    from research_b200 import replicas
    assert s1 - s0 == replicas.SEED_STRIDE       # disjoint seed ranges
    replicas.check_seed_budget(replicas.SEED_STRIDE - 1)
    with pytest.raises(ValueError):
        replicas.check_seed_budget(replicas.SEED_STRIDE)


def test_a_failed_rank_surfaces_as_an_error():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    status = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
    assert status[0] == "error"
    assert procs[1].exitcode == 3


def test_single_process_needs_no_group():
    from research_b200 import replicas
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    assert replicas.env_ranks() == (1, 0, 0)
    assert replicas.max_over_ranks(1, 3.5) == 3.5
    assert replicas.job_throughput(2_073_600 * 4, 1, 36.8) == pytest.approx(225.39, rel=1e-3)
