"""numpy FP64 restatement of the learned V-cycle preconditioner and of its
training loss (no counterpart in the reference: CFDApp preconditions its p'
CG with Jacobi, src/algebra/CG.cpp:14-148).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the device
network (cfdapp_b200/csrc/mg.cu) and of its gradient (mgtrain.cu); the
product never imports it.  Definitions, all in kernel space (a 2D grid
(nx, ny) is (nx, 1, ny)), arrays indexed [k, j, i]:

* level operator: (A x)_c = (sum of the cell's face coefficients) x_c
  - sum over interior faces D_f x_nb   (boundary faces enter the diagonal);
* coarse level: cells agglomerated 2x2(x2) along every axis longer than 1,
  coarse face coefficient = sum of the fine face coefficients it covers;
  coarsening stops after a level whose shortest active axis is <= 4 or
  whose cell count is <= 64 (never before level 1), or at an axis of 1;
* smoothing layer: x <- x + D^-1/2 (W * (D^-1/2 (r - A x))), W a 3x3x3
  kernel (2D weight sets: 3x3 in (x, y), stored in the middle plane);
* V-cycle: nu layers, restrict the residual by summation, cycle the next
  level, prolongate by injection scaled by c_l, nu layers; the coarsest
  level takes `coarse_sweeps` damped-Jacobi sweeps (0.8 D^-1) from 0;
* pinned reference cell: r[pin] reads as 0 and z[pin] = r[pin].
Loss of an error field e (e[pin] = 0): r = A e (r[pin] = 0), z = M r,
L = (z - e)^T A (z - e) / (e^T A e).
"""
from __future__ import annotations

import numpy as np

TAPS = 27


def kernel_faces(dim, n, faces):
    """Kernel-space face arrays from the global real-order face vector
    (x-faces, then y-faces, then z-faces)."""
    faces = np.asarray(faces, dtype=np.float64)
    if dim == 2:
        nx, ny = n
        nfx = (nx + 1) * ny
        fx = faces[:nfx].reshape(ny, 1, nx + 1)
        fz = faces[nfx:nfx + nx * (ny + 1)].reshape(ny + 1, 1, nx)
        return (nx, 1, ny), (fx, None, fz)
    nx, ny, nz = n
    nfx = (nx + 1) * ny * nz
    nfy = nx * (ny + 1) * nz
    fx = faces[:nfx].reshape(nz, ny, nx + 1)
    fy = faces[nfx:nfx + nfy].reshape(nz, ny + 1, nx)
    fz = faces[nfx + nfy:].reshape(nz + 1, ny, nx)
    return (nx, ny, nz), (fx, fy, fz)


class Level:
    def __init__(self, dims, f):
        self.dims = dims
        self.fx, self.fy, self.fz = f
        d = self.fx[:, :, :-1] + self.fx[:, :, 1:]
        if self.fy is not None:
            d = d + self.fy[:, :-1, :] + self.fy[:, 1:, :]
        d = d + self.fz[:-1] + self.fz[1:]
        self.diag = d
        self.isq = np.where(d > 0, 1.0 / np.sqrt(np.where(d > 0, d, 1.0)), 0.0)

    @property
    def shape(self):
        nx, ny, nz = self.dims
        return (nz, ny, nx)

    def apply(self, x):
        y = self.diag * x
        fx = self.fx[:, :, 1:-1]
        y[:, :, 1:] -= fx * x[:, :, :-1]
        y[:, :, :-1] -= fx * x[:, :, 1:]
        if self.fy is not None:
            fy = self.fy[:, 1:-1, :]
            y[:, 1:, :] -= fy * x[:, :-1, :]
            y[:, :-1, :] -= fy * x[:, 1:, :]
        fz = self.fz[1:-1]
        y[1:] -= fz * x[:-1]
        y[:-1] -= fz * x[1:]
        return y


def _pairs_sum(a, axis):
    """Sum adjacent pairs along `axis` (zero-padded to even length)."""
    n = a.shape[axis]
    if n == 1:
        return a
    if n % 2:
        pad = [(0, 0)] * a.ndim
        pad[axis] = (0, 1)
        a = np.pad(a, pad)
    sl0 = [slice(None)] * a.ndim
    sl1 = [slice(None)] * a.ndim
    sl0[axis] = slice(0, None, 2)
    sl1[axis] = slice(1, None, 2)
    return a[tuple(sl0)] + a[tuple(sl1)]


def _coarse_face(f, axis_face, n_fine, n_coarse, other_axes):
    """Coarse faces along array axis `axis_face`: fine positions 2*ic, the last
    one at the fine boundary; summed over pairs in the other axes."""
    pos = [min(2 * ic, n_fine) for ic in range(n_coarse + 1)]
    g = np.take(f, pos, axis=axis_face)
    for ax in other_axes:
        g = _pairs_sum(g, ax)
    return g


def coarsen(L: Level) -> Level:
    nx, ny, nz = L.dims
    c = lambda m: (m + 1) // 2 if m > 1 else 1
    cx, cy, cz = c(nx), c(ny), c(nz)
    # array axes: 0 = z, 1 = y, 2 = x
    fx = _coarse_face(L.fx, 2, nx, cx, (0, 1))
    fy = _coarse_face(L.fy, 1, ny, cy, (0, 2)) if L.fy is not None else None
    fz = _coarse_face(L.fz, 0, nz, cz, (1, 2))
    return Level((cx, cy, cz), (fx, fy, fz))


def hierarchy(dims, faces, dim):
    levels = [Level(dims, faces)]
    while True:
        L = levels[-1]
        nx, ny, nz = L.dims
        active = [nx, nz] if dim == 2 else [nx, ny, nz]
        mn = min(active)
        cells = nx * ny * nz
        if (len(levels) > 1 and (mn <= 4 or cells <= 64)) or mn == 1 or len(levels) == 16:
            return levels
        levels.append(coarsen(L))


def kernel_taps(dim, w):
    """Kernel-space 3x3x3 array [dk, dj, di] from a 27-tap weight row."""
    w = np.asarray(w, dtype=np.float64)
    if dim == 3:
        return w.reshape(3, 3, 3)
    K = np.zeros((3, 3, 3))
    real = w[9:18].reshape(3, 3)  # [dj_real, di]
    K[:, 1, :] = real             # real y -> kernel z
    return K


def conv(K, v):
    nz, ny, nx = v.shape
    p = np.pad(v, 1)
    out = np.zeros_like(v)
    for dk in range(3):
        for dj in range(3):
            for di in range(3):
                if K[dk, dj, di] != 0.0:
                    out += K[dk, dj, di] * p[dk:dk + nz, dj:dj + ny, di:di + nx]
    return out


def restrict(a, coarse_shape):
    g = a
    for ax in range(3):
        g = _pairs_sum(g, ax)
    assert g.shape == coarse_shape
    return g


def prolong(ec, fine_shape):
    nz, ny, nx = fine_shape
    return ec[np.ix_(np.arange(nz) // 2, np.arange(ny) // 2, np.arange(nx) // 2)]


class VCycle:
    """The network with weights (kernels[levels][27], coarse[levels], nu, coarse_sweeps)."""

    def __init__(self, dim, levels, kernels, coarse, nu=2, coarse_sweeps=50):
        self.dim = dim
        self.L = levels
        self.kernels = [kernel_taps(dim, k) for k in kernels]
        self.coarse = list(coarse)
        self.nu = nu
        self.coarse_sweeps = coarse_sweeps

    def K(self, l):
        return self.kernels[min(l, len(self.kernels) - 1)]

    def c(self, l):
        return self.coarse[min(l, len(self.coarse) - 1)]

    def cycle(self, l, r):
        L = self.L[l]
        if l == len(self.L) - 1:
            x = np.zeros_like(r)
            inv = L.isq * L.isq
            for _ in range(self.coarse_sweeps):
                x = x + 0.8 * inv * (r - L.apply(x))
            return x
        K = self.K(l)
        x = np.zeros_like(r)
        for _ in range(self.nu):
            x = x + L.isq * conv(K, L.isq * (r - L.apply(x)))
        rc = restrict(r - L.apply(x), self.L[l + 1].shape)
        ec = self.cycle(l + 1, rc)
        x = x + self.c(l) * prolong(ec, L.shape)
        for _ in range(self.nu):
            x = x + L.isq * conv(K, L.isq * (r - L.apply(x)))
        return x

    def apply(self, r, pin=-1):
        r = np.array(r, dtype=np.float64).reshape(self.L[0].shape)
        flat = r.reshape(-1)
        rp = flat[pin] if pin >= 0 else 0.0
        if pin >= 0:
            flat[pin] = 0.0
        z = self.cycle(0, r).reshape(-1)
        if pin >= 0:
            z[pin] = rp
        return z

    def loss(self, e, pin=-1):
        L0 = self.L[0]
        e = np.array(e, dtype=np.float64).reshape(-1)
        if pin >= 0:
            e[pin] = 0.0
        E = e.reshape(L0.shape)
        r = L0.apply(E).reshape(-1)
        if pin >= 0:
            r[pin] = 0.0
        z = self.apply(r, pin)
        d = (z - e).reshape(L0.shape)
        return float(np.sum(d * L0.apply(d)) / np.sum(E * L0.apply(E)))


def free_params(dim):
    """Indices of the independent taps of a point-symmetric kernel (t <= 26 - t)."""
    if dim == 2:
        return [t for t in range(9, 18) if t <= 26 - t]
    return [t for t in range(TAPS) if t <= 26 - t]


def random_faces(dim, n, seed, neumann=True):
    """Positive lognormal face coefficients in global real order (test data);
    boundary faces 0 (all-Neumann) unless neumann=False."""
    rng = np.random.default_rng(seed)
    if dim == 2:
        nx, ny = n
        fx = np.exp(rng.normal(size=(ny, nx + 1)) * 0.5)
        fy = np.exp(rng.normal(size=(ny + 1, nx)) * 0.5)
        if neumann:
            fx[:, 0] = fx[:, -1] = 0.0
            fy[0, :] = fy[-1, :] = 0.0
        return np.concatenate([fx.ravel(), fy.ravel()])
    nx, ny, nz = n
    fx = np.exp(rng.normal(size=(nz, ny, nx + 1)) * 0.5)
    fy = np.exp(rng.normal(size=(nz, ny + 1, nx)) * 0.5)
    fz = np.exp(rng.normal(size=(nz + 1, ny, nx)) * 0.5)
    if neumann:
        fx[:, :, 0] = fx[:, :, -1] = 0.0
        fy[:, 0, :] = fy[:, -1, :] = 0.0
        fz[0] = fz[-1] = 0.0
    return np.concatenate([fx.ravel(), fy.ravel(), fz.ravel()])


def random_weights(dim, levels, seed):
    """A point-symmetric weight set near damped Jacobi (test data)."""
    rng = np.random.default_rng(seed)
    k = np.zeros((levels, 27))
    for l in range(levels):
        w = np.zeros(27)
        idx = free_params(dim)
        w[idx] = rng.normal(size=len(idx)) * 0.05
        w[13] += 0.8
        w = w + w[::-1] - np.where(np.arange(27) == 13, w, 0)  # point-symmetric
        k[l] = w
    return k, 1.0 + 0.1 * rng.normal(size=levels)
