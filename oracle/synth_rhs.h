/* Seeded synthetic right-hand side for the isolated pressure-correction solve
 * (oracle copy; test infrastructure only).
 *
 * Definition (the same one the product library's cfdb_synth_rhs implements):
 *   SplitMix64 stream seeded with `seed`.  For m = 0..31 draw, in this order,
 *   kx, ky[, kz] = 1 + (next() >> 58)           (uniform integers in [1, 64])
 *   phx, phy[, phz] = (next() >> 11) * 2^-53 * 2*pi   (uniform in [0, 2 pi))
 *   a_m = 1 / (kx^2 + ky^2 [+ kz^2]).
 *   f(x) = sum_m a_m cos(pi kx x + phx) cos(pi ky y + phy) [cos(pi kz z + phz)]
 *   at the cell centres of the unit square / cube, summed over m in order,
 *   each term evaluated as ((a_m * cx) * cy) [* cz].
 *   b_i = V f_i - V * mean(f)   with V the (uniform) cell volume and mean(f)
 *   the sequential FP64 sum of f over cells in cell-id order divided by the
 *   cell count (the volume-weighted mean on a uniform grid); then b_0 = 0 for
 *   the pinned reference cell.
 */
#ifndef CFDB_ORACLE_SYNTH_RHS_H
#define CFDB_ORACLE_SYNTH_RHS_H

#include <math.h>
#include <stdint.h>
#include <stdlib.h>

static inline uint64_t oracle_splitmix64(uint64_t* state) {
  uint64_t z = (*state += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

/* nz == 0 selects 2D.  b must hold nx*ny*(nz ? nz : 1) doubles.  Returns 0 on
 * success, -1 on allocation failure. */
static inline int oracle_synth_rhs(int64_t nx, int64_t ny, int64_t nz, uint64_t seed, double* b) {
  const double pi = 3.14159265358979323846;
  const int dim3 = nz > 0;
  const int64_t nzz = dim3 ? nz : 1;
  const int64_t n = nx * ny * nzz;
  const int modes = 32;
  double* cx = (double*)malloc(sizeof(double) * (size_t)(nx + ny + nzz));
  if (!cx) return -1;
  double* cy = cx + nx;
  double* cz = cy + ny;
  for (int64_t i = 0; i < n; ++i) b[i] = 0.0;
  uint64_t s = seed;
  for (int m = 0; m < modes; ++m) {
    const double kx = (double)(1 + (oracle_splitmix64(&s) >> 58));
    const double ky = (double)(1 + (oracle_splitmix64(&s) >> 58));
    const double kz = dim3 ? (double)(1 + (oracle_splitmix64(&s) >> 58)) : 0.0;
    const double phx = (double)(oracle_splitmix64(&s) >> 11) * 0x1.0p-53 * (2.0 * pi);
    const double phy = (double)(oracle_splitmix64(&s) >> 11) * 0x1.0p-53 * (2.0 * pi);
    const double phz = dim3 ? (double)(oracle_splitmix64(&s) >> 11) * 0x1.0p-53 * (2.0 * pi) : 0.0;
    const double a = 1.0 / (kx * kx + ky * ky + kz * kz);
    for (int64_t i = 0; i < nx; ++i) cx[i] = cos(pi * kx * (((double)i + 0.5) / (double)nx) + phx);
    for (int64_t j = 0; j < ny; ++j) cy[j] = cos(pi * ky * (((double)j + 0.5) / (double)ny) + phy);
    if (dim3)
      for (int64_t k = 0; k < nz; ++k) cz[k] = cos(pi * kz * (((double)k + 0.5) / (double)nz) + phz);
    for (int64_t k = 0; k < nzz; ++k)
      for (int64_t j = 0; j < ny; ++j)
        for (int64_t i = 0; i < nx; ++i) {
          double t = (a * cx[i]) * cy[j];
          if (dim3) t = t * cz[k];
          b[(k * ny + j) * nx + i] += t;
        }
  }
  double sum = 0.0;
  for (int64_t i = 0; i < n; ++i) sum += b[i];
  const double mean = sum / (double)n;
  const double vol = dim3 ? 1.0 / ((double)nx * (double)ny * (double)nz) : 1.0 / ((double)nx * (double)ny);
  for (int64_t i = 0; i < n; ++i) b[i] = vol * b[i] - vol * mean;
  b[0] = 0.0;
  free(cx);
  return 0;
}

#endif
