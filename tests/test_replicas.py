"""The multi-GPU form of the batched path is replicas: every rank runs its own
256-system batch (disjoint seeds), with no collective on the data path, and
the reported time is the maximum over ranks. Checked here with two gloo
ranks on the CPU: the ranks' systems differ, the timing reduction returns the
slowest rank's time on every rank, and each rank's systems run through the
CPU restatement independently."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import bench
    from oracle import esp_port as EP
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        sl = bench._systems(rank, 3)
        ms = 10.0 + 5.0 * rank  # each rank's own device time
        slowest = bench.max_over_ranks(ms, world)
        prm = EP.plan(sl[:1], bench.RCUT)
        _, _, F, E = EP.run_batch(sl[:1], prm, bench.RCUT + bench.SKIN, 0, bench.DT, threads=1)
        out[rank] = (slowest, [s.N for s in sl], float(sl[0].pos[0, 0]), float(E[0]))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 15.0  # max over ranks on every rank
    # disjoint replicas: different systems on each rank
    assert (res[0][1], res[0][2]) != (res[1][1], res[1][2])
    assert all(np.isfinite(r[3]) for r in res.values())
