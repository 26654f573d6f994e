"""Multi-GPU replicas (one process per GPU, no data-path collective), checked on CPU with two
gloo ranks: the barrier, the max-over-ranks time and the whole-job throughput."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from gaspacho2_b200.replicas import Replicas

    r = Replicas(backend="gloo", timeout_s=60)
    r.barrier()
    t = r.max_time(0.5 * (rank + 1))
    rate = r.throughput(3, 0.5 * (rank + 1))
    out.put((rank, t, rate))
    r.close()


def test_two_gloo_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    for _, t, rate in res:
        assert t == pytest.approx(1.0)          # the slower rank's time
        assert rate == pytest.approx(2 * 3 / 1.0)  # both ranks' steps over it


def test_single_process_is_a_replica_of_one(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from gaspacho2_b200.replicas import Replicas

    r = Replicas(backend="gloo")
    assert r.world == 1 and r.max_time(0.25) == 0.25 and r.throughput(4, 2.0) == 2.0
    r.close()
