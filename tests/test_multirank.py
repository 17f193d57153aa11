"""The N > 1 host logic of bench.py on CPU: two gloo ranks partition the
ensemble members (no data-path collective) and reduce the per-rank points
(sum) and times (max) as the GPU runs do over NCCL."""
import multiprocessing as mp
import socket

from multirank_worker import worker


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_ensemble_partition_and_reductions_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, seeds0, pts0, tot0, mx0, all0), (r1, seeds1, pts1, tot1, mx1, all1) = res
    assert (r0, r1) == (0, 1)
    assert not set(seeds0) & set(seeds1)  # disjoint
    assert len(seeds0) + len(seeds1) == 64  # and complete
    assert tot0 == tot1 == pts0 + pts1 == all0 == all1
    assert mx0 == mx1 == 3.0
