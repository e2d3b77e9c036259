"""Failure detection without a GPU fault.

On the GPU: the bounded device-side wait of the persistent kernels' barriers
gives up after its limit on a barrier that can never complete, reports
CFDB_ERR_DEVICE_TIMEOUT through the host, and leaves the context usable.
On the CPU (two gloo ranks): a rank that leaves before a collective makes the
survivor's next collective of the benchmark plumbing fail with an error
rather than wait for ever."""
import ctypes as C
import os
import socket
import time

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench
from cfdapp_b200 import cfdb


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_the_context_survives(ctx):
    L = ctx.lib
    L.cfdb_selftest_wait_timeout.argtypes = [C.c_void_p, C.c_double, C.POINTER(C.c_int)]
    released = C.c_int(-1)
    t0 = time.perf_counter()
    st = L.cfdb_selftest_wait_timeout(ctx.handle, 0.25, C.byref(released))
    took = time.perf_counter() - t0
    assert st == -5 and released.value == 2  # CFDB_ERR_DEVICE_TIMEOUT, both blocks returned
    assert 0.2 <= took < 5.0
    assert b"timed out" in L.cfdb_last_error(ctx.handle)
    # the same context still solves
    op = cfdb.POperator(ctx, 2, (32, 32))
    r = op.solve(cfdb.synth_rhs(2, 32), cfdb.LinearSolverSettings(absolute_tolerance=0.0,
                                                                  relative_tolerance=1e-8))
    assert r.status == "Converged"
    op.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=10))
    if rank == 1:
        os._exit(0)  # leaves between steps, with no collective in flight
    t0 = time.perf_counter()
    try:
        bench.combine_over_ranks(dist, "cpu", 1.0, 1.0)
        out[0] = ("completed", time.perf_counter() - t0)
    except Exception as e:  # the survivor learns of it as an error
        out[0] = (type(e).__name__, time.perf_counter() - t0)


def test_a_departed_rank_turns_the_next_collective_into_an_error():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
        res = dict(out)
    kind, took = res[0]
    assert kind != "completed" and took < 60.0
