"""The allocation-free p' solve (cfdb_pcg_solve_noalloc) against the regular
one (cfdb_poperator_solve_device), through the C ABI.

The entry point exists for callers that cannot allocate device memory when
they solve (a stream capture that must not gain allocations, an allocator
owned by another runtime, a loop that forbids cudaMalloc after start-up).  It
keeps its scratch in one fixed device array shared by every call, so the test
makes two calls in a row -- the second starts from the first call's leftover
scratch -- and checks both against the regular solve.  This file is collected
last so a failure here does not hide the other tests; it also passes alone.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(ctx, grid, b_dev, x_dev, settings):
    from cfdapp_b200 import cfdb
    L = ctx.lib
    L.cfdb_pcg_solve_noalloc.argtypes = [C.c_void_p, C.POINTER(cfdb._Grid), C.c_double, C.c_int,
                                         C.c_int64, C.POINTER(cfdb._LinSettings), C.c_void_p,
                                         C.c_void_p, C.POINTER(cfdb._LinResult)]
    res = cfdb._LinResult()
    st = L.cfdb_pcg_solve_noalloc(C.c_void_p(ctx.stream()), C.byref(grid), 1.0, 1, 0,
                                  C.byref(settings.c()), C.c_void_p(b_dev), C.c_void_p(x_dev),
                                  C.byref(res))
    return st, res


@pytest.mark.parametrize("dim,n", [(2, 96), (3, 24)])
def test_noalloc_matches_regular_solve_twice(ctx, dim, n):
    from cfdapp_b200 import cfdb
    b = cfdb.synth_rhs(dim, n)
    s = cfdb.LinearSolverSettings(absolute_tolerance=0.0, relative_tolerance=1e-8,
                                  max_iterations=20000)
    op = cfdb.POperator(ctx, dim, [n] * dim)
    ref = op.solve(b, s)
    assert ref.status == "Converged"
    grid = cfdb.grid(dim, [n] * dim)
    bd = ctx.to_device(b)
    xd = ctx.alloc(b.nbytes)
    try:
        for call in range(2):
            ctx.memset(xd, 0, b.nbytes)
            st, res = _noalloc(ctx, grid, bd, xd, s)
            assert st == cfdb.CFDB_OK, f"call {call}: status {st}"
            assert cfdb.SOLVER_STATUS[res.status] == "Converged"
            assert abs(res.iterations - ref.iterations) <= max(2, 0.02 * ref.iterations)
            x = ctx.download(xd, (b.size,))
            err = np.linalg.norm(x - ref.solution) / np.linalg.norm(ref.solution)
            assert err <= 1e-9, f"call {call}: relative difference {err:.3e}"
    finally:
        ctx.free(bd)
        ctx.free(xd)
        op.close()


def test_noalloc_rejects_oversize_grid(ctx):
    from cfdapp_b200 import cfdb
    s = cfdb.LinearSolverSettings(absolute_tolerance=0.0, relative_tolerance=1e-8,
                                  max_iterations=10)
    grid = cfdb.grid(2, (512, 512))  # 262144 cells > the fixed scratch
    st, _ = _noalloc(ctx, grid, 16, 16, s)
    assert st == -6  # CFDB_ERR_UNSUPPORTED: rejected before touching the pointers
