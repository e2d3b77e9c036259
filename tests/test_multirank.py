"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2): every
rank takes the same collective steps, the job's time is the max over ranks
and its work the sum; each rank of the batched workload advances its own
seeded case list (weak scaling, no data-path collective)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        r, w, _ = bench.dist_info()
        ms, work = bench.combine_over_ranks(dist, "cpu", 10.0 * (rank + 1), 100.0 + rank)
        cases = [(c[0], c[1], round(c[2], 6)) for c in bench.batched_cases(bench.SEED + r, 6)]
        out[rank] = (r, w, ms, work, cases)
    finally:
        dist.destroy_process_group()


def test_two_ranks_combine_time_and_work():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn",
                           join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for rank, (r, w, ms, work, _) in res.items():
        assert (r, w) == (rank, world)
        assert ms == pytest.approx(20.0) and work == pytest.approx(201.0)
    assert res[0][4] != res[1][4]  # each rank its own cases
    assert res[0][4] == [(c[0], c[1], round(c[2], 6))
                         for c in bench.batched_cases(bench.SEED, 6)]
