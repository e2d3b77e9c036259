"""ctypes binding of libcfdb.so (include/cfdb.h).

The names mirror the reference's linear-solver interface
(include/cfd/algebra/LinearSolver.hpp): ``LinearSolverSettings``,
``SolverResult``, ``SolverStatus``.  The library is loaded from the package's
``lib/`` directory; when it is missing, or no sm_100 device is present, every
entry point raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libcfdb.so")

CFDB_OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "no usable sm_100 device",
          -4: "out of memory", -5: "device-side wait timed out", -6: "unsupported"}

SOLVER_STATUS = ["Converged", "MaxIterations", "Breakdown", "NonFiniteInput",
                 "NonFiniteResidual", "InvalidSystem"]
SIMPLE_STATUS = ["Converged", "MaxIterations", "MomentumFailure", "PressureCorrectionFailure",
                 "NonFiniteState", "InvalidConfiguration"]

KRYLOV = {"cg": 0, "bicgstab": 1}
PRECISION = {"fp64": 0, "fp32_refined": 1}
PRECOND = {"none": 0, "jacobi": 1, "learned_mg": 2}
MG_TAPS = 27
MG_MAX_LEVELS = 16


class CfdbError(RuntimeError):
    pass


class _Grid(C.Structure):
    _fields_ = [("dim", C.c_int), ("n", C.c_int64 * 3), ("len", C.c_double * 3)]


class _LinSettings(C.Structure):
    _fields_ = [("krylov", C.c_int), ("preconditioner", C.c_int), ("precision", C.c_int),
                ("abs_tol", C.c_double), ("rel_tol", C.c_double), ("max_iterations", C.c_int64),
                ("inner_rel_tol", C.c_double), ("max_refinements", C.c_int64)]


class _LinResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int64),
                ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("true_residual", C.c_double), ("refinements", C.c_int64),
                ("restarts", C.c_int64), ("device_ms", C.c_double),
                ("kernel_launches", C.c_int64), ("krylov_ms", C.c_double),
                ("krylov_bytes", C.c_double), ("krylov_launches", C.c_int64),
                ("fallback_iterations", C.c_int64)]


_lib = None


def library_path() -> str:
    return LIB_PATH


def load() -> C.CDLL:
    """Loads libcfdb.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.environ.get("CFDB_LIBRARY") or LIB_PATH  # another build of the same library
    if not os.path.exists(path):
        raise CfdbError(f"{path} is missing: build it with `python -m cfdapp_b200.build`")
    L = C.CDLL(path)
    vp, i64, dbl = C.c_void_p, C.c_int64, C.c_double
    L.cfdb_cuda_available.restype = C.c_int
    L.cfdb_create.argtypes = [C.c_int, vp, C.POINTER(vp)]
    L.cfdb_destroy.argtypes = [vp]
    L.cfdb_destroy.restype = None
    L.cfdb_last_error.argtypes = [vp]
    L.cfdb_last_error.restype = C.c_char_p
    L.cfdb_stream.argtypes = [vp]
    L.cfdb_stream.restype = vp
    L.cfdb_kernel_launches.argtypes = [vp]
    L.cfdb_kernel_launches.restype = i64
    L.cfdb_synth_rhs.argtypes = [i64, i64, i64, C.c_uint64, C.POINTER(dbl)]
    L.cfdb_poperator_create_uniform.argtypes = [vp, C.POINTER(_Grid), dbl, C.c_uint, C.c_int, i64,
                                                C.POINTER(vp)]
    L.cfdb_poperator_create_faces.argtypes = [vp, C.POINTER(_Grid), C.POINTER(dbl), C.c_int, i64,
                                              C.POINTER(vp)]
    L.cfdb_poperator_destroy.argtypes = [vp]
    L.cfdb_poperator_destroy.restype = None
    L.cfdb_poperator_cells.argtypes = [vp]
    L.cfdb_poperator_cells.restype = i64
    L.cfdb_poperator_apply.argtypes = [vp, vp, vp, vp]
    for name in ("cfdb_poperator_solve_device", "cfdb_poperator_solve_host"):
        getattr(L, name).argtypes = [vp, vp, C.POINTER(_LinSettings), vp, vp, C.POINTER(dbl), i64,
                                     C.POINTER(_LinResult)]
    L.cfdb_device_alloc.argtypes = [vp, C.c_size_t, C.POINTER(vp)]
    L.cfdb_device_free.argtypes = [vp, vp]
    L.cfdb_copy_to_device.argtypes = [vp, vp, vp, C.c_size_t]
    L.cfdb_copy_to_host.argtypes = [vp, vp, vp, C.c_size_t]
    L.cfdb_synchronize.argtypes = [vp]
    L.cfdb_memset_device.argtypes = [vp, vp, C.c_int, C.c_size_t]
    fp = C.POINTER(C.c_float)
    ip = C.POINTER(C.c_int)
    L.cfdb_mg_set_weights.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, fp, fp]
    L.cfdb_mg_get_weights.argtypes = [vp, C.c_int, ip, ip, ip, fp, fp]
    L.cfdb_mg_reset_weights.argtypes = [vp, C.c_int, C.c_int]
    L.cfdb_mg_apply.argtypes = [vp, vp, fp, fp]
    L.cfdb_mg_loss_grad.argtypes = [vp, vp, C.c_int, fp, C.POINTER(dbl), C.POINTER(dbl),
                                    C.POINTER(dbl)]
    _lib = L
    return L


def cuda_available() -> bool:
    """cfd::gpu::cudaAvailable() (include/cfd/gpu/GPUBackend.hpp:15)."""
    return bool(load().cfdb_cuda_available())


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Context:
    """A cfdb context on one device (and one stream)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        L = load()
        h = C.c_void_p()
        st = L.cfdb_create(device, C.c_void_p(stream) if stream else None, C.byref(h))
        if st != CFDB_OK:
            raise CfdbError(f"cfdb_create failed: {ERRORS.get(st, st)}")
        self._h = h
        self.lib = L

    @property
    def handle(self):
        return self._h

    def check(self, st: int, what: str):
        if st != CFDB_OK:
            msg = self.lib.cfdb_last_error(self._h).decode(errors="replace")
            raise CfdbError(f"{what}: {ERRORS.get(st, st)}: {msg}")

    def stream(self) -> int:
        return self.lib.cfdb_stream(self._h) or 0

    def launches(self) -> int:
        return int(self.lib.cfdb_kernel_launches(self._h))

    # learned preconditioner weights (cfdb_mg_*)
    def mg_set_weights(self, dim: int, kernels: np.ndarray, coarse_weights: np.ndarray,
                       nu: int = 2, coarse_sweeps: int = 50):
        """kernels: (levels, 27) float32 taps (x fastest); coarse_weights: (levels,)."""
        k = np.ascontiguousarray(kernels, dtype=np.float32).reshape(-1, MG_TAPS)
        c = np.ascontiguousarray(coarse_weights, dtype=np.float32).reshape(-1)
        if len(c) != len(k):
            raise ValueError("one coarse weight per kernel")
        fp = C.POINTER(C.c_float)
        self.check(self.lib.cfdb_mg_set_weights(self._h, dim, len(k), nu, coarse_sweeps,
                                                k.ctypes.data_as(fp), c.ctypes.data_as(fp)),
                   "cfdb_mg_set_weights")

    def mg_get_weights(self, dim: int) -> dict:
        lv, nu, cs = C.c_int(), C.c_int(), C.c_int()
        k = np.zeros((MG_MAX_LEVELS, MG_TAPS), dtype=np.float32)
        c = np.zeros(MG_MAX_LEVELS, dtype=np.float32)
        fp = C.POINTER(C.c_float)
        self.check(self.lib.cfdb_mg_get_weights(self._h, dim, C.byref(lv), C.byref(nu), C.byref(cs),
                                                k.ctypes.data_as(fp), c.ctypes.data_as(fp)),
                   "cfdb_mg_get_weights")
        n = lv.value
        return {"levels": n, "nu": nu.value, "coarse_sweeps": cs.value,
                "kernels": k[:n].copy(), "coarse_weights": c[:n].copy()}

    def mg_reset_weights(self, dim: int, trained: bool = True):
        self.check(self.lib.cfdb_mg_reset_weights(self._h, dim, int(trained)),
                   "cfdb_mg_reset_weights")

    def alloc(self, nbytes: int) -> int:
        p = C.c_void_p()
        self.check(self.lib.cfdb_device_alloc(self._h, nbytes, C.byref(p)), "cfdb_device_alloc")
        return p.value

    def free(self, ptr: int):
        self.check(self.lib.cfdb_device_free(self._h, C.c_void_p(ptr)), "cfdb_device_free")

    def to_device(self, arr: np.ndarray) -> int:
        arr = np.ascontiguousarray(arr)
        p = self.alloc(arr.nbytes)
        self.check(self.lib.cfdb_copy_to_device(self._h, C.c_void_p(p), arr.ctypes.data_as(C.c_void_p),
                                                arr.nbytes), "cfdb_copy_to_device")
        return p

    def upload(self, dst: int, arr: np.ndarray):
        arr = np.ascontiguousarray(arr)
        self.check(self.lib.cfdb_copy_to_device(self._h, C.c_void_p(dst), arr.ctypes.data_as(C.c_void_p),
                                                arr.nbytes), "cfdb_copy_to_device")

    def download(self, src: int, shape, dtype=np.float64) -> np.ndarray:
        out = np.empty(shape, dtype=dtype)
        self.check(self.lib.cfdb_copy_to_host(self._h, out.ctypes.data_as(C.c_void_p), C.c_void_p(src),
                                              out.nbytes), "cfdb_copy_to_host")
        return out

    def memset(self, dst: int, value: int, nbytes: int):
        self.check(self.lib.cfdb_memset_device(self._h, C.c_void_p(dst), value, nbytes),
                   "cfdb_memset_device")

    def synchronize(self):
        self.check(self.lib.cfdb_synchronize(self._h), "cfdb_synchronize")

    def close(self):
        if getattr(self, "_h", None):
            self.lib.cfdb_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class LinearSolverSettings:
    """LinearSolverSettings (LinearSolver.hpp:136-166) plus precision knobs."""
    absolute_tolerance: float = 1e-12
    relative_tolerance: float = 1e-10
    max_iterations: int = 1000
    type: str = "cg"
    preconditioner: str = "jacobi"
    precision: str = "fp64"
    inner_relative_tolerance: float = 0.0
    max_refinements: int = 0

    def c(self) -> _LinSettings:
        return _LinSettings(KRYLOV[self.type], PRECOND[self.preconditioner],
                            PRECISION[self.precision], self.absolute_tolerance,
                            self.relative_tolerance, self.max_iterations,
                            self.inner_relative_tolerance, self.max_refinements)


@dataclass
class SolverResult:
    """SolverResult (LinearSolver.hpp:110-134)."""
    status: str
    iterations: int
    initial_residual: float
    final_residual: float
    true_residual: float
    refinements: int
    restarts: int
    device_ms: float
    kernel_launches: int
    krylov_ms: float
    krylov_bytes: float
    krylov_launches: int
    fallback_iterations: int
    residual_history: np.ndarray
    solution: np.ndarray | None = None

    def converged(self) -> bool:
        return self.status == "Converged"


def grid(dim: int, n, length=(1.0, 1.0, 1.0)) -> _Grid:
    g = _Grid()
    g.dim = dim
    n = list(n) + [1, 1, 1]
    for a in range(3):
        g.n[a] = int(n[a]) if a < dim else 1
        g.len[a] = float(length[a]) if a < len(length) else 1.0
    return g


def synth_rhs(dim: int, n: int, seed: int = 20261203) -> np.ndarray:
    """The seeded synthetic p' RHS (see cfdb_synth_rhs)."""
    b = np.empty(n ** dim, dtype=np.float64)
    st = load().cfdb_synth_rhs(n, n, n if dim == 3 else 0, seed, _dp(b))
    if st != CFDB_OK:
        raise CfdbError("cfdb_synth_rhs failed")
    return b


class POperator:
    """The matrix-free p' operator on the device (cfdb_poperator_*)."""

    def __init__(self, ctx: Context, dim: int, n, length=(1.0, 1.0, 1.0), *, rho: float = 1.0,
                 face_coeff: np.ndarray | None = None, dirichlet_patch_mask: int = 0,
                 pinned: bool = True, reference_cell: int = 0):
        self.ctx = ctx
        self.dim = dim
        self.n = tuple(int(v) for v in n)
        g = grid(dim, n, length)
        h = C.c_void_p()
        if face_coeff is None:
            st = ctx.lib.cfdb_poperator_create_uniform(ctx.handle, C.byref(g), rho,
                                                       dirichlet_patch_mask, int(pinned),
                                                       reference_cell, C.byref(h))
        else:
            fc = np.ascontiguousarray(face_coeff, dtype=np.float64)
            st = ctx.lib.cfdb_poperator_create_faces(ctx.handle, C.byref(g), _dp(fc), int(pinned),
                                                     reference_cell, C.byref(h))
        ctx.check(st, "cfdb_poperator_create")
        self._h = h
        self.cells = int(ctx.lib.cfdb_poperator_cells(h))

    def update_faces(self, face_coeff: np.ndarray):
        """New face coefficients for an operator made from face coefficients
        (cfdb_poperator_update_faces): the device arrays, and a learned
        solve's hierarchy and graph, are kept; their values are refreshed."""
        fc = np.ascontiguousarray(face_coeff, dtype=np.float64)
        L = self.ctx.lib
        L.cfdb_poperator_update_faces.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]
        self.ctx.check(L.cfdb_poperator_update_faces(self.ctx.handle, self._h, _dp(fc)),
                       "cfdb_poperator_update_faces")

    def apply_device(self, x_dev: int, y_dev: int):
        self.ctx.check(self.ctx.lib.cfdb_poperator_apply(self.ctx.handle, self._h, C.c_void_p(x_dev),
                                                         C.c_void_p(y_dev)), "cfdb_poperator_apply")

    def apply(self, x: np.ndarray) -> np.ndarray:
        xd = self.ctx.to_device(np.asarray(x, dtype=np.float64))
        yd = self.ctx.alloc(8 * self.cells)
        try:
            self.apply_device(xd, yd)
            return self.ctx.download(yd, (self.cells,))
        finally:
            self.ctx.free(xd)
            self.ctx.free(yd)

    def _result(self, r: _LinResult, hist, cap, sol=None) -> SolverResult:
        if self._precond == PRECOND["learned_mg"]:
            m = r.iterations - r.fallback_iterations + 1
        elif self._precision == 0 or self._mixed_in_one_space():
            m = r.iterations + 1  # one entry per iteration
        else:
            m = r.refinements + 1  # FP32 solves inside FP64 refinement: one per refinement
        m = min(cap, m)
        return SolverResult(SOLVER_STATUS[r.status], r.iterations, r.initial_residual,
                            r.final_residual, r.true_residual, r.refinements, r.restarts,
                            r.device_ms, r.kernel_launches, r.krylov_ms, r.krylov_bytes,
                            r.krylov_launches, r.fallback_iterations, hist[:m].copy(), sol)

    def _mixed_in_one_space(self) -> bool:
        """Whether an FP32_REFINED solve of this operator runs the FP32
        Jacobi-PCG with FP64 residual replacement (rows of a multiple of 16
        bytes in FP32) rather than FP32 solves inside FP64 refinement."""
        return self.n[0] % 4 == 0 and not os.environ.get("CFDB_NO_TMA")

    def solve(self, b: np.ndarray, settings: LinearSolverSettings, x0: np.ndarray | None = None,
              history_cap: int | None = None) -> SolverResult:
        """Host buffers in and out (copies inside the call)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.cells) if x0 is None else np.array(x0, dtype=np.float64)
        cap = (settings.max_iterations + 1) if history_cap is None else history_cap
        hist = np.zeros(max(cap, 1))
        res = _LinResult()
        cs = settings.c()
        self._precision = cs.precision
        self._precond = cs.preconditioner
        self.ctx.check(self.ctx.lib.cfdb_poperator_solve_host(self.ctx.handle, self._h, C.byref(cs),
                                                              _dp(b), _dp(x), _dp(hist), cap,
                                                              C.byref(res)), "cfdb_poperator_solve_host")
        return self._result(res, hist, cap, x)

    def solve_inplace(self, b: np.ndarray, x: np.ndarray, settings: LinearSolverSettings,
                      history_cap: int = 0) -> SolverResult:
        """Host buffers used in place (float64, contiguous; pinned buffers let
        the copies run at full link speed): b in, x0 in x, solution out in x."""
        for a in (b, x):
            if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"] or a.size != self.cells:
                raise CfdbError("solve_inplace needs contiguous float64 arrays of the grid's size")
        hist = np.zeros(max(history_cap, 1))
        res = _LinResult()
        cs = settings.c()
        self._precision = cs.precision
        self._precond = cs.preconditioner
        self.ctx.check(self.ctx.lib.cfdb_poperator_solve_host(self.ctx.handle, self._h, C.byref(cs),
                                                              _dp(b), _dp(x), _dp(hist), history_cap,
                                                              C.byref(res)), "cfdb_poperator_solve_host")
        return self._result(res, hist, history_cap, x)

    def solve_device(self, b_dev: int, x_dev: int, settings: LinearSolverSettings,
                     history_cap: int = 0) -> SolverResult:
        """Device-resident b and x (x holds x0 on entry)."""
        hist = np.zeros(max(history_cap, 1))
        res = _LinResult()
        cs = settings.c()
        self._precision = cs.precision
        self._precond = cs.preconditioner
        self.ctx.check(self.ctx.lib.cfdb_poperator_solve_device(
            self.ctx.handle, self._h, C.byref(cs), C.c_void_p(b_dev), C.c_void_p(x_dev),
            _dp(hist) if history_cap > 0 else None, history_cap, C.byref(res)),
            "cfdb_poperator_solve_device")
        return self._result(res, hist, history_cap)

    # learned preconditioner (cfdb_mg_*)
    def mg_apply(self, r: np.ndarray) -> np.ndarray:
        """z = M r through the solve's V-cycle kernels (FP32)."""
        rr = np.ascontiguousarray(r, dtype=np.float32).reshape(-1)
        z = np.empty_like(rr)
        fp = C.POINTER(C.c_float)
        self.ctx.check(self.ctx.lib.cfdb_mg_apply(self.ctx.handle, self._h, rr.ctypes.data_as(fp),
                                                  z.ctypes.data_as(fp)), "cfdb_mg_apply")
        return z

    def mg_loss_grad(self, e: np.ndarray):
        """Loss and gradient of the context's network on error fields e (samples x cells)."""
        ee = np.ascontiguousarray(e, dtype=np.float32).reshape(-1, self.cells)
        loss = C.c_double()
        gk = np.zeros((MG_MAX_LEVELS, MG_TAPS))
        gc = np.zeros(MG_MAX_LEVELS)
        self.ctx.check(self.ctx.lib.cfdb_mg_loss_grad(
            self.ctx.handle, self._h, len(ee), ee.ctypes.data_as(C.POINTER(C.c_float)),
            C.byref(loss), _dp(gk), _dp(gc)), "cfdb_mg_loss_grad")
        return loss.value, gk, gc

    def close(self):
        if getattr(self, "_h", None):
            self.ctx.lib.cfdb_poperator_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ SIMPLE
VBC = {"wall": 0, "moving_wall": 1, "inlet": 2, "outlet": 3}
PBC = {"fixed_gradient": 0, "fixed_value": 1}
SCHEME = {"upwind": 0, "central": 1, "linear_upwind": 2, "lud": 2, "quick": 3}
FACE_FLUX = {"linear": 0, "rhie_chow": 1, "rhiechow": 1, "automatic": 2, "auto": 2}


class _SimpleCase(C.Structure):
    _fields_ = [("grid", _Grid), ("vbc_type", C.c_int * 6), ("vbc_value", (C.c_double * 3) * 6),
                ("pbc_type", C.c_int * 6), ("pbc_value", C.c_double * 6), ("rho", C.c_double),
                ("mu", C.c_double), ("nodes", C.POINTER(C.c_double) * 3)]


class _SimpleSettings(C.Structure):
    _fields_ = [("max_outer", C.c_int64), ("alpha_u", C.c_double), ("alpha_p", C.c_double),
                ("tol_u", C.c_double), ("tol_p", C.c_double), ("tol_c", C.c_double),
                ("scheme", C.c_int), ("face_flux", C.c_int), ("reference_cell", C.c_int64),
                ("momentum", _LinSettings), ("pressure", _LinSettings)]


class _SimpleResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int64), ("final_u", C.c_double),
                ("final_v", C.c_double), ("final_w", C.c_double), ("final_p", C.c_double),
                ("final_continuity", C.c_double), ("global_imbalance", C.c_double),
                ("momentum_linear_iterations", C.c_int64),
                ("pressure_linear_iterations", C.c_int64), ("device_ms", C.c_double),
                ("pressure_solve_ms", C.c_double), ("momentum_solve_ms", C.c_double),
                ("kernel_launches", C.c_int64)]


@dataclass
class SimpleCase:
    """A Cartesian case (MeshGeometry::createCartesian2D/3D, or with per-axis
    node coordinates createRectilinear2D / createGraded2D) + BCs + fluid."""
    dim: int
    n: tuple
    length: tuple = (1.0, 1.0, 1.0)
    vbc: tuple = ()     # per patch: (type, (vx, vy, vz))
    pbc: tuple = ()     # per patch: (type, value)
    rho: float = 1.0
    mu: float = 0.01
    nodes: tuple = ()   # per axis: n+1 node coordinates, or None for a uniform axis

    @staticmethod
    def cavity(dim: int, n: int, lid: float = 1.0, mu: float = 0.01, rho: float = 1.0):
        vbc = [("wall", (0.0, 0.0, 0.0))] * (2 * dim)
        vbc[3] = ("moving_wall", (lid, 0.0, 0.0))
        return SimpleCase(dim, (n,) * dim, (1.0, 1.0, 1.0), tuple(vbc),
                          tuple([("fixed_gradient", 0.0)] * (2 * dim)), rho, mu)

    @staticmethod
    def channel(nx: int, ny: int, lx: float, ly: float, inlet: float = 1.0, mu: float = 0.1,
                rho: float = 1.0):
        vbc = (("inlet", (inlet, 0.0, 0.0)), ("outlet", (0.0, 0.0, 0.0)),
               ("wall", (0.0, 0.0, 0.0)), ("wall", (0.0, 0.0, 0.0)))
        pbc = (("fixed_gradient", 0.0), ("fixed_value", 0.0), ("fixed_gradient", 0.0),
               ("fixed_gradient", 0.0))
        return SimpleCase(2, (nx, ny), (lx, ly, 1.0), vbc, pbc, rho, mu)

    def cells(self) -> int:
        return int(np.prod(self.n[: self.dim]))

    def faces(self) -> int:
        n = list(self.n) + [1, 1]
        nx, ny, nz = n[0], n[1], (n[2] if self.dim == 3 else 1)
        f = (nx + 1) * ny * nz + nx * (ny + 1) * nz
        return f + (nx * ny * (nz + 1) if self.dim == 3 else 0)

    def c(self) -> _SimpleCase:
        cs = _SimpleCase()
        cs.grid = grid(self.dim, self.n, self.length)
        for q in range(6):
            t, val = self.vbc[q] if q < len(self.vbc) else ("wall", (0, 0, 0))
            cs.vbc_type[q] = VBC[t]
            for k in range(3):
                cs.vbc_value[q][k] = float(val[k]) if k < len(val) else 0.0
            pt, pv = self.pbc[q] if q < len(self.pbc) else ("fixed_gradient", 0.0)
            cs.pbc_type[q] = PBC[pt]
            cs.pbc_value[q] = float(pv)
        cs.rho = self.rho
        cs.mu = self.mu
        self._node_arrays = []  # kept alive with the case while the struct is in use
        for a in range(3):
            nd = self.nodes[a] if a < len(self.nodes) else None
            if nd is None:
                cs.nodes[a] = None
            else:
                arr = np.ascontiguousarray(nd, dtype=np.float64)
                if arr.size != self.n[a] + 1:
                    raise CfdbError(f"axis {a}: {arr.size} node coordinates for {self.n[a]} cells")
                self._node_arrays.append(arr)
                cs.nodes[a] = _dp(arr)
        return cs


@dataclass
class SIMPLESettings:
    """SIMPLESettings (include/cfd/pressure_velocity/SIMPLESettings.hpp:42-145)."""
    max_iterations: int = 1000
    velocity_relaxation: float = 0.7
    pressure_relaxation: float = 0.3
    velocity_tolerance: float = 1e-8
    pressure_tolerance: float = 1e-8
    continuity_tolerance: float = 1e-8
    convection_scheme: str = "upwind"
    face_flux: str = "automatic"
    reference_cell: int = 0
    momentum_solver: LinearSolverSettings = None
    pressure_solver: LinearSolverSettings = None

    def __post_init__(self):
        if self.momentum_solver is None:
            self.momentum_solver = LinearSolverSettings(type="bicgstab", preconditioner="none")
        if self.pressure_solver is None:
            self.pressure_solver = LinearSolverSettings(type="bicgstab", preconditioner="none")

    def c(self) -> _SimpleSettings:
        return _SimpleSettings(self.max_iterations, self.velocity_relaxation,
                               self.pressure_relaxation, self.velocity_tolerance,
                               self.pressure_tolerance, self.continuity_tolerance,
                               SCHEME[self.convection_scheme], FACE_FLUX[self.face_flux],
                               self.reference_cell, self.momentum_solver.c(),
                               self.pressure_solver.c())


@dataclass
class SIMPLEResult:
    """SIMPLEResult (include/cfd/pressure_velocity/SIMPLEResult.hpp:80-200)."""
    status: str
    iterations: int
    final: dict
    momentum_linear_iterations: int
    pressure_linear_iterations: int
    device_ms: float
    pressure_solve_ms: float
    momentum_solve_ms: float
    kernel_launches: int
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    p: np.ndarray
    flux: np.ndarray
    history: np.ndarray

    def converged(self) -> bool:
        return self.status == "Converged"


def _simple_sigs(L):
    vp = C.c_void_p
    dp = C.POINTER(C.c_double)
    L.cfdb_simple_solve.argtypes = [vp, C.POINTER(_SimpleCase), C.POINTER(_SimpleSettings), dp, dp,
                                    dp, dp, dp, dp, C.POINTER(_SimpleResult)]
    L.cfdb_simple_create.argtypes = [vp, C.POINTER(_SimpleCase), C.POINTER(_SimpleSettings),
                                     C.POINTER(vp)]
    L.cfdb_simple_destroy.argtypes = [vp]
    L.cfdb_simple_destroy.restype = None
    L.cfdb_simple_set_state.argtypes = [vp, dp, dp, dp, dp]
    L.cfdb_simple_get_state.argtypes = [vp, dp, dp, dp, dp, dp]
    L.cfdb_simple_pressure_gradient.argtypes = [vp, dp, dp, dp]
    L.cfdb_simple_assemble_momentum.argtypes = [vp, C.c_int, dp, C.POINTER(dp), dp]
    L.cfdb_simple_iterate.argtypes = [vp, C.c_int64, dp, C.POINTER(_SimpleResult)]
    L.cfdb_simple_pprime_faces.argtypes = [vp, dp, C.POINTER(C.c_int), C.POINTER(C.c_int64)]


def _result(r: _SimpleResult, case, u, v, w, p, flux, hist) -> SIMPLEResult:
    final = dict(u=r.final_u, v=r.final_v, w=r.final_w, p=r.final_p,
                 continuity=r.final_continuity, global_imbalance=r.global_imbalance)
    return SIMPLEResult(SIMPLE_STATUS[r.status], r.iterations, final, r.momentum_linear_iterations,
                        r.pressure_linear_iterations, r.device_ms, r.pressure_solve_ms,
                        r.momentum_solve_ms, r.kernel_launches, u, v,
                        w if case.dim == 3 else np.zeros(0), p, flux,
                        hist[: 5 * r.iterations].reshape(-1, 5))


def simple_solve(ctx: Context, case: SimpleCase, settings: SIMPLESettings, u0=None, v0=None,
                 w0=None, p0=None) -> SIMPLEResult:
    """SIMPLE::solve on the device from host fields (zero fields by default)."""
    L = ctx.lib
    _simple_sigs(L)
    n = case.cells()
    u = np.zeros(n) if u0 is None else np.array(u0, dtype=np.float64)
    v = np.zeros(n) if v0 is None else np.array(v0, dtype=np.float64)
    w = np.zeros(n) if w0 is None else np.array(w0, dtype=np.float64)
    p = np.zeros(n) if p0 is None else np.array(p0, dtype=np.float64)
    flux = np.zeros(case.faces())
    hist = np.zeros(5 * max(settings.max_iterations, 1))
    r = _SimpleResult()
    ctx.check(L.cfdb_simple_solve(ctx.handle, C.byref(case.c()), C.byref(settings.c()), _dp(u),
                                  _dp(v), _dp(w), _dp(p), _dp(flux), _dp(hist), C.byref(r)),
              "cfdb_simple_solve")
    return _result(r, case, u, v, w, p, flux, hist)


class Simple:
    """Stage-level SIMPLE session (GpuSimpleDiscretization-like)."""

    def __init__(self, ctx: Context, case: SimpleCase, settings: SIMPLESettings):
        self.ctx, self.case, self.settings = ctx, case, settings
        _simple_sigs(ctx.lib)
        h = C.c_void_p()
        ctx.check(ctx.lib.cfdb_simple_create(ctx.handle, C.byref(case.c()), C.byref(settings.c()),
                                             C.byref(h)), "cfdb_simple_create")
        self._h = h

    def set_state(self, u, v, w, p):
        n = self.case.cells()
        arr = [np.ascontiguousarray(a if a is not None else np.zeros(n), dtype=np.float64)
               for a in (u, v, w, p)]
        self._keep = arr
        self.ctx.check(self.ctx.lib.cfdb_simple_set_state(self._h, *[_dp(a) for a in arr]),
                       "cfdb_simple_set_state")

    def get_state(self):
        n = self.case.cells()
        u, v, w, p = (np.zeros(n) for _ in range(4))
        f = np.zeros(self.case.faces())
        self.ctx.check(self.ctx.lib.cfdb_simple_get_state(self._h, _dp(u), _dp(v), _dp(w), _dp(p),
                                                          _dp(f)), "cfdb_simple_get_state")
        return u, v, (w if self.case.dim == 3 else np.zeros(0)), p, f

    def pressure_gradient(self):
        n = self.case.cells()
        g = [np.zeros(n) for _ in range(3)]
        self.ctx.check(self.ctx.lib.cfdb_simple_pressure_gradient(self._h, *[_dp(a) for a in g]),
                       "cfdb_simple_pressure_gradient")
        return g[: self.case.dim]

    def assemble_momentum(self, comp: int):
        n = self.case.cells()
        diag, rhs = np.zeros(n), np.zeros(n)
        off = [np.zeros(n) for _ in range(6)]
        offp = (C.POINTER(C.c_double) * 6)(*[_dp(o) for o in off])
        self.ctx.check(self.ctx.lib.cfdb_simple_assemble_momentum(self._h, comp, _dp(diag), offp,
                                                                  _dp(rhs)),
                       "cfdb_simple_assemble_momentum")
        return diag, off, rhs

    def pprime_faces(self):
        """(D_f in global face order, pinned, reference cell) of the last p' system."""
        f = np.zeros(self.case.faces())
        pin, ref = C.c_int(), C.c_int64()
        self.ctx.check(self.ctx.lib.cfdb_simple_pprime_faces(self._h, _dp(f), C.byref(pin),
                                                             C.byref(ref)),
                       "cfdb_simple_pprime_faces")
        return f, bool(pin.value), int(ref.value)

    def iterate(self, n: int) -> SIMPLEResult:
        hist = np.zeros(5 * max(n, 1))
        r = _SimpleResult()
        self.ctx.check(self.ctx.lib.cfdb_simple_iterate(self._h, n, _dp(hist), C.byref(r)),
                       "cfdb_simple_iterate")
        u, v, w, p, f = self.get_state()
        return _result(r, self.case, u, v, w, p, f, hist)

    def close(self):
        if getattr(self, "_h", None):
            self.ctx.lib.cfdb_simple_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ batched SIMPLE
class _BatchTuning(C.Structure):
    _fields_ = [("cell_threads", C.c_int), ("cell_tile", C.c_int), ("face_threads", C.c_int),
                ("face_tile", C.c_int), ("team_exponent", C.c_double),
                ("adaptive_teams", C.c_int), ("cell_stage_ms", C.c_double),
                ("face_stage_ms", C.c_double), ("pprime_solve_ms", C.c_double),
                ("candidates", C.c_int)]


class _BatchStats(C.Structure):
    _fields_ = [("graph_launches", C.c_int64), ("active", C.c_int), ("device_ms", C.c_double),
                ("kernel_launches", C.c_int64)]


def _batch_sigs(L):
    vp, i64 = C.c_void_p, C.c_int64
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    lp = C.POINTER(C.c_int64)
    _simple_sigs(L)
    L.cfdb_batch_create.argtypes = [vp, C.c_int, C.POINTER(_SimpleCase), C.POINTER(_SimpleSettings),
                                    i64, C.POINTER(vp)]
    L.cfdb_batch_destroy.argtypes = [vp]
    L.cfdb_batch_destroy.restype = None
    L.cfdb_batch_cases.argtypes = [vp]
    L.cfdb_batch_set_state.argtypes = [vp, C.c_int, dp, dp, dp, dp]
    L.cfdb_batch_get_state.argtypes = [vp, C.c_int, dp, dp, dp, dp, dp]
    L.cfdb_batch_autotune.argtypes = [vp, C.POINTER(_BatchTuning)]
    L.cfdb_batch_set_tuning.argtypes = [vp, C.POINTER(_BatchTuning)]
    L.cfdb_batch_get_tuning.argtypes = [vp, C.POINTER(_BatchTuning)]
    L.cfdb_batch_iterate.argtypes = [vp, i64, C.POINTER(_BatchStats)]
    L.cfdb_batch_profile_iteration.argtypes = [vp, ip, dp, C.c_int, ip]
    L.cfdb_batch_results.argtypes = [vp, C.POINTER(_SimpleResult)]
    L.cfdb_batch_history.argtypes = [vp, C.c_int, dp, i64, lp]
    L.cfdb_batch_plan_tiles.argtypes = [C.c_int, lp, C.c_int, ip, ip, lp]
    L.cfdb_batch_plan_teams.argtypes = [C.c_int, dp, lp, ip, C.c_int, i64, ip, ip]


def plan_tiles(counts, tile: int, lib=None):
    """Tile list of the batch's stage kernels (host only): (first, tile_case, tile_start)."""
    L = lib or load()
    _batch_sigs(L)
    cnt = np.ascontiguousarray(counts, dtype=np.int64)
    n = cnt.size
    first = np.zeros(n + 1, dtype=np.int32)
    ip, lp = C.POINTER(C.c_int), C.POINTER(C.c_int64)
    st = L.cfdb_batch_plan_tiles(n, cnt.ctypes.data_as(lp), tile, first.ctypes.data_as(ip), None, None)
    if st != 0:
        raise CfdbError(f"cfdb_batch_plan_tiles failed ({st})")
    tc = np.zeros(int(first[-1]), dtype=np.int32)
    ts = np.zeros(int(first[-1]), dtype=np.int64)
    st = L.cfdb_batch_plan_tiles(n, cnt.ctypes.data_as(lp), tile, first.ctypes.data_as(ip),
                                 tc.ctypes.data_as(ip), ts.ctypes.data_as(lp))
    if st != 0:
        raise CfdbError(f"cfdb_batch_plan_tiles failed ({st})")
    return first, tc, ts


def plan_teams(weight, cells, active, nblocks: int, min_cells_per_block: int = 2048, lib=None):
    """Krylov team table of the batch (host only): (team_first, block_case)."""
    L = lib or load()
    _batch_sigs(L)
    w = np.ascontiguousarray(weight, dtype=np.float64)
    c = np.ascontiguousarray(cells, dtype=np.int64)
    a = np.ascontiguousarray(active, dtype=np.int32)
    n = w.size
    tf = np.zeros(n + 1, dtype=np.int32)
    bc = np.zeros(nblocks, dtype=np.int32)
    ip = C.POINTER(C.c_int)
    st = L.cfdb_batch_plan_teams(n, w.ctypes.data_as(C.POINTER(C.c_double)),
                                 c.ctypes.data_as(C.POINTER(C.c_int64)), a.ctypes.data_as(ip),
                                 nblocks, min_cells_per_block, tf.ctypes.data_as(ip),
                                 bc.ctypes.data_as(ip))
    if st != 0:
        raise CfdbError(f"cfdb_batch_plan_teams failed ({st})")
    return tf, bc


@dataclass
class BatchTuning:
    cell_threads: int = 256
    cell_tile: int = 1024
    face_threads: int = 256
    face_tile: int = 1024
    team_exponent: float = 1.5
    adaptive_teams: bool = True
    cell_stage_ms: float = 0.0
    face_stage_ms: float = 0.0
    pprime_solve_ms: float = 0.0
    candidates: int = 0

    @staticmethod
    def of(t: _BatchTuning) -> "BatchTuning":
        return BatchTuning(t.cell_threads, t.cell_tile, t.face_threads, t.face_tile,
                           t.team_exponent, bool(t.adaptive_teams), t.cell_stage_ms,
                           t.face_stage_ms, t.pprime_solve_ms, t.candidates)

    def c(self) -> _BatchTuning:
        return _BatchTuning(self.cell_threads, self.cell_tile, self.face_threads, self.face_tile,
                            self.team_exponent, int(self.adaptive_teams), self.cell_stage_ms,
                            self.face_stage_ms, self.pprime_solve_ms, self.candidates)


class Batch:
    """Many independent SIMPLE cases of one dimension advanced together (cfdb_batch_*)."""

    def __init__(self, ctx: Context, cases, settings: SIMPLESettings, history_cap: int = 0):
        self.ctx, self.cases, self.settings = ctx, list(cases), settings
        self.history_cap = history_cap
        _batch_sigs(ctx.lib)
        arr = (_SimpleCase * len(self.cases))(*[c.c() for c in self.cases])
        h = C.c_void_p()
        ctx.check(ctx.lib.cfdb_batch_create(ctx.handle, len(self.cases), arr, C.byref(settings.c()),
                                            history_cap, C.byref(h)), "cfdb_batch_create")
        self._h = h

    def set_state(self, k: int, u=None, v=None, w=None, p=None):
        n = self.cases[k].cells()
        arr = [np.ascontiguousarray(a if a is not None else np.zeros(n), dtype=np.float64)
               for a in (u, v, w, p)]
        self.ctx.check(self.ctx.lib.cfdb_batch_set_state(self._h, k, *[_dp(a) for a in arr]),
                       "cfdb_batch_set_state")

    def get_state(self, k: int):
        case = self.cases[k]
        n = case.cells()
        u, v, w, p = (np.zeros(n) for _ in range(4))
        f = np.zeros(case.faces())
        self.ctx.check(self.ctx.lib.cfdb_batch_get_state(self._h, k, _dp(u), _dp(v), _dp(w), _dp(p),
                                                         _dp(f)), "cfdb_batch_get_state")
        return u, v, (w if case.dim == 3 else np.zeros(0)), p, f

    def autotune(self) -> BatchTuning:
        t = _BatchTuning()
        self.ctx.check(self.ctx.lib.cfdb_batch_autotune(self._h, C.byref(t)), "cfdb_batch_autotune")
        return BatchTuning.of(t)

    @property
    def tuning(self) -> BatchTuning:
        t = _BatchTuning()
        self.ctx.check(self.ctx.lib.cfdb_batch_get_tuning(self._h, C.byref(t)), "cfdb_batch_get_tuning")
        return BatchTuning.of(t)

    @tuning.setter
    def tuning(self, t: BatchTuning):
        self.ctx.check(self.ctx.lib.cfdb_batch_set_tuning(self._h, C.byref(t.c())),
                       "cfdb_batch_set_tuning")

    def iterate(self, n: int) -> dict:
        s = _BatchStats()
        self.ctx.check(self.ctx.lib.cfdb_batch_iterate(self._h, n, C.byref(s)), "cfdb_batch_iterate")
        return dict(graph_launches=s.graph_launches, active=s.active, device_ms=s.device_ms,
                    kernel_launches=s.kernel_launches)

    def profile_iteration(self) -> list:
        """One eager outer iteration with events around every launch: [(id, ms)];
        id: stage number, -1 momentum solve kernel, -2 p' solve kernel."""
        cap = 256
        ids = np.zeros(cap, dtype=np.int32)
        ms = np.zeros(cap)
        cnt = C.c_int()
        self.ctx.check(self.ctx.lib.cfdb_batch_profile_iteration(
            self._h, ids.ctypes.data_as(C.POINTER(C.c_int)), _dp(ms), cap, C.byref(cnt)),
            "cfdb_batch_profile_iteration")
        n = min(cnt.value, cap)
        return list(zip(ids[:n].tolist(), ms[:n].tolist()))

    def results(self) -> list:
        rs = (_SimpleResult * len(self.cases))()
        self.ctx.check(self.ctx.lib.cfdb_batch_results(self._h, rs), "cfdb_batch_results")
        out = []
        for r in rs:
            final = dict(u=r.final_u, v=r.final_v, w=r.final_w, p=r.final_p,
                         continuity=r.final_continuity, global_imbalance=r.global_imbalance)
            out.append(dict(status=SIMPLE_STATUS[r.status], iterations=r.iterations, final=final,
                            momentum_linear_iterations=r.momentum_linear_iterations,
                            pressure_linear_iterations=r.pressure_linear_iterations))
        return out

    def history(self, k: int) -> np.ndarray:
        cap = max(self.history_cap, 1)
        h = np.zeros(5 * cap)
        rows = C.c_int64()
        self.ctx.check(self.ctx.lib.cfdb_batch_history(self._h, k, _dp(h), cap, C.byref(rows)),
                       "cfdb_batch_history")
        return h[: 5 * rows.value].reshape(-1, 5)

    def close(self):
        if getattr(self, "_h", None):
            self.ctx.lib.cfdb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ result files
def _results_sigs(L):
    vp, i64 = C.c_void_p, C.c_int64
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    L.cfdb_write_results.argtypes = [C.POINTER(_SimpleCase), dp, dp, dp, dp, dp, i64, C.c_double,
                                     C.c_char_p, ip]
    L.cfdb_simple_write_results.argtypes = [vp, dp, i64, C.c_double, C.c_char_p, ip]
    L.cfdb_batch_write_results.argtypes = [vp, C.c_int, C.c_char_p, ip]


def write_results(case: SimpleCase, u, v, w, p, history, global_imbalance: float, directory: str,
                  lib=None) -> bool:
    """fields.csv, residuals.csv and solution.vtk in the reference's formats
    (host only); history: rows of {u, v, w, p, continuity}.  Returns whether
    the field files were written (all values finite)."""
    L = lib or load()
    _results_sigs(L)
    n = case.cells()
    arr = [np.ascontiguousarray(a if a is not None and np.size(a) else np.zeros(n), dtype=np.float64)
           for a in (u, v, w, p)]
    h = np.ascontiguousarray(np.asarray(history, dtype=np.float64).reshape(-1, 5))
    done = C.c_int()
    st = L.cfdb_write_results(C.byref(case.c()), *[_dp(a) for a in arr], _dp(h.reshape(-1)),
                              h.shape[0], float(global_imbalance), directory.encode(),
                              C.byref(done))
    if st != 0:
        raise CfdbError(f"cfdb_write_results failed ({st})")
    return bool(done.value)


def _simple_write_results(self, history, global_imbalance: float, directory: str) -> bool:
    _results_sigs(self.ctx.lib)
    h = np.ascontiguousarray(np.asarray(history, dtype=np.float64).reshape(-1, 5))
    done = C.c_int()
    self.ctx.check(self.ctx.lib.cfdb_simple_write_results(self._h, _dp(h.reshape(-1)), h.shape[0],
                                                          float(global_imbalance),
                                                          directory.encode(), C.byref(done)),
                   "cfdb_simple_write_results")
    return bool(done.value)


def _batch_write_results(self, k: int, directory: str) -> bool:
    _results_sigs(self.ctx.lib)
    done = C.c_int()
    self.ctx.check(self.ctx.lib.cfdb_batch_write_results(self._h, k, directory.encode(),
                                                         C.byref(done)),
                   "cfdb_batch_write_results")
    return bool(done.value)


Simple.write_results = _simple_write_results
Batch.write_results = _batch_write_results


# ------------------------------------------------------------------ CSR systems
CSR_PATH = {0: "stencil", 1: "faces"}


class _CsrInfo(C.Structure):
    _fields_ = [("dim", C.c_int), ("n", C.c_int64 * 3), ("path", C.c_int),
                ("faces_eligible", C.c_int), ("pinned", C.c_int), ("reference_cell", C.c_int64),
                ("learned_declined", C.c_int)]

    def as_dict(self) -> dict:
        return {"dim": self.dim, "n": tuple(self.n[: self.dim]), "path": CSR_PATH[self.path],
                "faces_eligible": bool(self.faces_eligible), "pinned": bool(self.pinned),
                "reference_cell": int(self.reference_cell),
                "learned_declined": bool(self.learned_declined)}


def _csr_sigs(L):
    if getattr(L, "_csr_sigs", False):
        return
    vp, i64, dbl = C.c_void_p, C.c_int64, C.c_double
    u64p = C.POINTER(C.c_uint64)
    L.cfdb_csr_analyze.argtypes = [i64, u64p, u64p, C.POINTER(dbl), C.POINTER(_CsrInfo)]
    L.cfdb_csr_solver_create.argtypes = [vp, C.POINTER(vp)]
    L.cfdb_csr_solver_destroy.argtypes = [vp]
    L.cfdb_csr_solver_destroy.restype = None
    L.cfdb_csr_solve_host.argtypes = [vp, C.POINTER(_LinSettings), i64, u64p, u64p, C.POINTER(dbl),
                                      C.POINTER(dbl), C.POINTER(dbl), C.POINTER(dbl), i64,
                                      C.POINTER(_LinResult), C.POINTER(_CsrInfo)]
    L._csr_sigs = True


def _csr_arrays(offsets, columns, values):
    ro = np.ascontiguousarray(offsets, dtype=np.uint64)
    ci = np.ascontiguousarray(columns, dtype=np.uint64)
    v = np.ascontiguousarray(values, dtype=np.float64)
    return ro, ci, v


def csr_analyze(offsets, columns, values) -> dict | None:
    """cfdb_csr_analyze: the recognised grid and path of a CSR matrix, or
    None when it is not a structured 5-/7-point operator (host only)."""
    L = load()
    _csr_sigs(L)
    ro, ci, v = _csr_arrays(offsets, columns, values)
    info = _CsrInfo()
    u64p = C.POINTER(C.c_uint64)
    st = L.cfdb_csr_analyze(len(ro) - 1, ro.ctypes.data_as(u64p), ci.ctypes.data_as(u64p), _dp(v),
                            C.byref(info))
    if st == -6:
        return None
    if st != CFDB_OK:
        raise CfdbError(f"cfdb_csr_analyze: {ERRORS.get(st, st)}")
    return info.as_dict()


class CsrSolver:
    """cfdb_csr_solver: solves of the reference's CSR LinearSystem."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        _csr_sigs(ctx.lib)
        h = C.c_void_p()
        ctx.check(ctx.lib.cfdb_csr_solver_create(ctx.handle, C.byref(h)), "cfdb_csr_solver_create")
        self._h = h
        self.info = None

    def solve(self, offsets, columns, values, b, settings: LinearSolverSettings,
              x0=None, history_cap: int | None = None) -> SolverResult:
        ro, ci, v = _csr_arrays(offsets, columns, values)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(len(b)) if x0 is None else np.array(x0, dtype=np.float64)
        cap = (settings.max_iterations + 1) if history_cap is None else history_cap
        hist = np.zeros(max(cap, 1))
        res = _LinResult()
        info = _CsrInfo()
        cs = settings.c()
        u64p = C.POINTER(C.c_uint64)
        self.ctx.check(self.ctx.lib.cfdb_csr_solve_host(
            self._h, C.byref(cs), len(ro) - 1, ro.ctypes.data_as(u64p), ci.ctypes.data_as(u64p),
            _dp(v), _dp(b), _dp(x), _dp(hist), cap, C.byref(res), C.byref(info)),
            "cfdb_csr_solve_host")
        self.info = info.as_dict() if info.dim else None
        if cs.preconditioner == PRECOND["learned_mg"] and self.info and self.info["path"] == "faces":
            m = res.iterations - res.fallback_iterations + 1
        else:
            m = res.iterations + 1
        m = min(cap, m) if res.status not in (3, 5) else 0
        return SolverResult(SOLVER_STATUS[res.status], res.iterations, res.initial_residual,
                            res.final_residual, res.true_residual, res.refinements, res.restarts,
                            res.device_ms, res.kernel_launches, res.krylov_ms, res.krylov_bytes,
                            res.krylov_launches, res.fallback_iterations, hist[:m].copy(), x)

    def close(self):
        if getattr(self, "_h", None):
            self.ctx.lib.cfdb_csr_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
