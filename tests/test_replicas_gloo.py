"""Multi-GPU is replicas only: each rank runs an independent instance and the
only cross-rank steps are the barrier and the max/sum of scalars that
bench.py uses for whole-job throughput.  Exercised here with two gloo ranks
on the CPU, each running the CPU oracle on its own seeded instance."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    try:
        import bench
        from oracle.oracle import Oracle
        from oracle.seedfield import seed_field

        d = bench.Dist()
        n = 12
        o = Oracle(n, 4.0, 1.0, threads=1)
        u = o.rescale(o.divavg_free(seed_field(n, rank, 2.0, 3.0)))  # replica seed = rank
        R = o.R_parts(u)[0]
        d.barrier()
        t_max = d.max(float(rank + 1))
        iters = d.sum(3.0)
        R_sum = d.sum(R)
        d.close()
        q.put((rank, t_max, iters, R, R_sum))
    except Exception as e:  # pragma: no cover - reported to the parent
        q.put((rank, "error", repr(e)))


def test_two_gloo_replicas_reduce_like_bench():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert all(r[1] != "error" for r in out), out
    out.sort()
    assert [r[1] for r in out] == [2.0, 2.0]          # max over ranks of the timed region
    assert [r[2] for r in out] == [6.0, 6.0]          # whole-job iteration count
    assert out[0][3] != out[1][3]                      # independent instances
    assert out[0][4] == pytest.approx(out[0][3] + out[1][3])
