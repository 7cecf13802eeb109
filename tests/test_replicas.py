"""Multi-process path of the benchmark on CPU: two gloo ranks join, time
their own replica, and agree on the job time (max over ranks) and the
whole-job throughput; a rank that never joins makes the other fail within
the process-group timeout instead of hanging."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    from hammurabix_b200 import replicas
    w, r, _ = replicas.init("gloo", 60)
    replicas.barrier(w)
    secs = 1.0 + r          # rank 1 is the slow replica
    t = replicas.max_over_ranks(secs, w)
    q.put((r, w, t, replicas.throughput(1000.0, w, t)))
    replicas.finish(w)


def test_two_gloo_ranks_agree_on_job_time_and_throughput():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    for _, w, t, v in out:
        assert w == 2 and t == 2.0 and v == 1000.0   # 2 ranks x 1000 units in 2 s


def _lonely(port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2",
                      RANK="0", LOCAL_RANK="0")
    from hammurabix_b200 import replicas
    try:
        replicas.init("gloo", 5)
        q.put("joined")
    except Exception as e:  # the second rank never arrives
        q.put(type(e).__name__)


def test_missing_rank_fails_within_the_timeout():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_lonely, args=(_free_port(), q))
    p.start()
    res = q.get(timeout=120)
    p.join(timeout=60)
    assert res != "joined"


def test_single_process_needs_no_group():
    from hammurabix_b200 import replicas
    assert replicas.max_over_ranks(3.5, 1) == 3.5
    assert replicas.throughput(10.0, 1, 2.0) == 5.0
