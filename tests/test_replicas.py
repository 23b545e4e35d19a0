"""The multi-GPU path of bench.py is replicas only (independent networks,
one per rank, no data-path collective): two gloo ranks on the CPU check the
max-over-ranks timing, the whole-job value and that every rank builds its
own network (seed + rank)."""
import os
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    # loopback only: resolving the host's name can take tens of seconds here
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), GLOO_SOCKET_IFNAME="lo")
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        ms = 100.0 + 50.0 * rank  # rank 1 is the slower replica
        worst = bench.max_over_ranks(ms, world, device="cpu")
        c, na = bench.build_network(rank, n=2000)  # the bench's network kind, small
        out[rank] = (worst, bench.replica_value(world, 10.0, worst), int(c.pre[:1000].sum()), na.n)
    finally:
        dist.destroy_process_group()


def test_two_replicas_on_gloo():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        out = man.dict()
        port = 29500 + (os.getpid() % 1000)
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(600)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == res[1][0] == 150.0  # both ranks see the slowest rank's time
    assert np.isclose(res[0][1], 2 * 10.0 / 0.150)
    assert res[0][2] != res[1][2] and res[0][3] == res[1][3] == 2000  # different networks, same size
