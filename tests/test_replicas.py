"""The multi-GPU form of the benchmark is N independent replicas (a run does
not shard: each phase needs the whole PSD in another layout).  Its host logic,
run here as two gloo processes on the CPU: each rank simulates its own seeded
workload, the job's time is the slowest rank's, and the throughput counts
every rank's simulated hours."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench
from verb4d_b200 import workload as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, w, local = bench.rank_info()
        # per-rank inputs: the seed is offset by the rank, as in run_ours
        wl = W.make_workload(W.GridSpec(6, 7, 5, 4), seed=2 + r)
        ms_local = 100.0 + 50.0 * r          # a slower second replica
        ms = bench.max_over_ranks(ms_local)
        out[r] = (r, w, local, float(wl.fields["DVV"].sum()), ms,
                  bench.replica_throughput(1.0, ms / 1e3, w))
    finally:
        dist.destroy_process_group()


def test_two_replicas_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r in range(world):
        rank, w, local, dsum, ms, thr = res[r]
        assert (rank, w, local) == (r, world, r)
        assert ms == 150.0                      # every rank sees the slowest
        assert thr == pytest.approx(2 * 1.0 / 0.150)
    assert res[0][3] != res[1][3]               # distinct seeded inputs per rank


def test_single_process_is_identity():
    assert bench.max_over_ranks(12.5) == 12.5
    assert bench.replica_throughput(2.0, 4.0, 1) == 0.5
    assert np.isclose(bench.replica_throughput(2.0, 4.0, 8), 4.0)
