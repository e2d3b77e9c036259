"""The allocation-free p' solve (cfdb_pcg_solve_noalloc) against the regular
one (cfdb_poperator_solve_device) and against the oracle, through the C ABI.

The entry point exists for callers that cannot allocate device memory when
they solve: a host whose device memory belongs to another runtime's
allocator, or a loop that forbids cudaMalloc/cudaFree after start-up.  It
keeps its scratch in one fixed device array shared by every call, so the
tests make calls in a row -- each starts from the previous call's leftover
scratch -- and check each against the regular solve or the oracle.  This
file is collected last so a failure here does not hide the other tests; it
also passes alone.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFDB_ERR_UNSUPPORTED = -6


def _noalloc(ctx, grid, b_dev, x_dev, settings, *, rho=1.0, pinned=1, reference_cell=0,
             stream=None):
    from cfdapp_b200 import cfdb
    L = ctx.lib
    L.cfdb_pcg_solve_noalloc.argtypes = [C.c_void_p, C.POINTER(cfdb._Grid), C.c_double, C.c_int,
                                         C.c_int64, C.POINTER(cfdb._LinSettings), C.c_void_p,
                                         C.c_void_p, C.POINTER(cfdb._LinResult)]
    res = cfdb._LinResult()
    st = L.cfdb_pcg_solve_noalloc(C.c_void_p(ctx.stream() if stream is None else stream),
                                  C.byref(grid), rho, pinned, reference_cell,
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


# the largest grid the fixed scratch takes (65536 cells: the most blocks and
# partials), density 2.5 and an interior pinned cell, in 2D and 3D, each
# checked against the oracle's CG + Jacobi on the same system
@pytest.mark.parametrize("dim,n,ref_cell", [(2, (256, 256), 256 * 100 + 37),
                                            (3, (40, 40, 40), 40 * 40 * 20 + 40 * 7 + 11)])
def test_noalloc_matches_oracle_at_the_size_limit(ctx, dim, n, ref_cell):
    from cfdapp_b200 import cfdb
    from oracle import oracle as O
    cells = int(np.prod(n))
    assert cells <= 65536
    case = O.Case(dim, tuple(n), (1.0, 1.0, 1.0), [("wall", (0, 0, 0))] * (2 * dim),
                  [("fixed_gradient", 0.0)] * (2 * dim))
    ones = np.ones(cells)
    _, diag, off, _ = O.assemble_pprime(case, 2.5, np.zeros(case.faces()), ones, ones, ones,
                                        reference_cell=ref_cell)
    b = np.random.default_rng(7).standard_normal(cells) / cells
    b[ref_cell] = 0.0
    want = O.stencil_solve(case, diag, off, b, rel_tol=1e-10, max_iterations=50000)
    assert want.status == "Converged"
    s = cfdb.LinearSolverSettings(absolute_tolerance=0.0, relative_tolerance=1e-10,
                                  max_iterations=50000)
    grid = cfdb.grid(dim, n)
    bd = ctx.to_device(b)
    xd = ctx.alloc(b.nbytes)
    try:
        for call in range(2):
            ctx.memset(xd, 0, b.nbytes)
            st, res = _noalloc(ctx, grid, bd, xd, s, rho=2.5, reference_cell=ref_cell)
            assert st == cfdb.CFDB_OK, f"call {call}: status {st}"
            assert cfdb.SOLVER_STATUS[res.status] == "Converged"
            assert abs(res.iterations - want.iterations) <= max(2, 0.02 * want.iterations)
            x = ctx.download(xd, (cells,))
            err = np.linalg.norm(x - want.solution) / np.linalg.norm(want.solution)
            assert err <= 1e-9, f"call {call}: relative difference {err:.3e}"
            assert x[ref_cell] == 0.0
    finally:
        ctx.free(bd)
        ctx.free(xd)


def test_noalloc_iteration_cap_and_zero_rhs(ctx):
    from cfdapp_b200 import cfdb
    dim, n = 2, 64
    grid = cfdb.grid(dim, [n] * dim)
    b = cfdb.synth_rhs(dim, n)
    bd = ctx.to_device(b)
    xd = ctx.alloc(b.nbytes)
    try:
        # a budget of 5 iterations ends with MaxIterations after exactly 5
        ctx.memset(xd, 0, b.nbytes)
        s5 = cfdb.LinearSolverSettings(absolute_tolerance=0.0, relative_tolerance=1e-12,
                                       max_iterations=5)
        st, res = _noalloc(ctx, grid, bd, xd, s5)
        assert st == cfdb.CFDB_OK
        assert cfdb.SOLVER_STATUS[res.status] == "MaxIterations"
        assert res.iterations == 5
        # b = 0 from x0 = 0 converges at once (||r0|| = 0 <= abs_tol)
        ctx.memset(bd, 0, b.nbytes)
        ctx.memset(xd, 0, b.nbytes)
        s0 = cfdb.LinearSolverSettings(absolute_tolerance=1e-12, relative_tolerance=1e-8,
                                       max_iterations=100)
        st, res = _noalloc(ctx, grid, bd, xd, s0)
        assert st == cfdb.CFDB_OK
        assert cfdb.SOLVER_STATUS[res.status] == "Converged"
        assert res.iterations == 0
        assert not np.any(ctx.download(xd, (b.size,)))
    finally:
        ctx.free(bd)
        ctx.free(xd)


def test_noalloc_refuses_a_capturing_stream_and_keeps_the_capture(ctx):
    """The call waits for its own result, which a stream capture forbids: on
    a capturing stream it returns CFDB_ERR_UNSUPPORTED before issuing any
    work, and the caller's graph still captures and replays."""
    import torch

    from cfdapp_b200 import cfdb
    dim, n = 2, 32
    grid = cfdb.grid(dim, [n] * dim)
    s = cfdb.LinearSolverSettings(absolute_tolerance=0.0, relative_tolerance=1e-8,
                                  max_iterations=100)
    y = torch.zeros(4, device="cuda")
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    statuses = []
    with torch.cuda.graph(g, stream=side):
        y.add_(1.0)
        st, _ = _noalloc(ctx, grid, 16, 16, s, stream=side.cuda_stream)
        statuses.append(st)
    g.replay()
    torch.cuda.synchronize()
    assert statuses == [CFDB_ERR_UNSUPPORTED]
    assert float(y.sum()) == 4.0


def test_noalloc_rejects_oversize_grid(ctx):
    from cfdapp_b200 import cfdb
    s = cfdb.LinearSolverSettings(absolute_tolerance=0.0, relative_tolerance=1e-8,
                                  max_iterations=10)
    grid = cfdb.grid(2, (512, 512))  # 262144 cells > the fixed scratch
    st, _ = _noalloc(ctx, grid, 16, 16, s)
    assert st == CFDB_ERR_UNSUPPORTED  # rejected before touching the pointers
