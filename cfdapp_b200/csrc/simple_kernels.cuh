// Launch wrappers of the SIMPLE stage kernels (simple_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "cfdb.h"
#include "simple_geo.cuh"

namespace cfdb {

void launch_mass_flux(const SGeo& G, double rho, const double* const U[3], double* F, cudaStream_t s);
void launch_scalar_face_values(const SGeo& G, const int* ptype, const double* pvalue,
                               const double* phi, double* fv, cudaStream_t s);
void launch_gg_sweep(const SGeo& G, const double* phi, const double* fv, const double* const prev[3],
                     double* const out[3], cudaStream_t s);
void launch_velocity_gradient(const SGeo& G, const double* uc, int comp, double* const g[3],
                              cudaStream_t s);
void launch_assemble_momentum(const SGeo& G, double mu, int scheme, int comp, const double* uc,
                              const double* F, const double* gradPc, const double* const gu[3],
                              double alpha, double* diag, double* const off[6], double* rhs,
                              cudaStream_t s);
void launch_response(const SGeo& G, const double* diag, double* d, cudaStream_t s);
void launch_rhie_chow(const SGeo& G, double rho, double alpha, const double* p,
                      const double* const gp[3], const double* const d[3], double* F,
                      cudaStream_t s);
void launch_pprime_faces(const SGeo& G, double rho, const double* const d[3], double* D,
                         cudaStream_t s);
void launch_pprime_rhs(const SGeo& G, const double* F, int pin, int64_t ref, double* rhs,
                       cudaStream_t s);
void launch_pressure_update(int64_t n, double alpha, const double* pp, double* p, cudaStream_t s);
void launch_velocity_correct(int64_t n, const double* us, const double* d, const double* g,
                             double* u, cudaStream_t s);
void launch_flux_correct(const SGeo& G, const double* Fs, const double* D, const double* pp,
                         double* F, cudaStream_t s);
int residual_sums_blocks(const SGeo& G);
void launch_residual_sums(const SGeo& G, const double* F, double* partials, cudaStream_t s);
void launch_nonfinite(int64_t n, const double* v, unsigned* flag, cudaStream_t s);

// Host helpers of the single-case session (simple.cu), shared with the batch.
SGeo simple_geometry(const cfdb_simple_case& cs);
bool simple_wall_offsets(const SGeo& G);  // the wall stencil needs velocity gradients
cfdb_status simple_validate(cfdb_context* ctx, const cfdb_simple_case* cs,
                            const cfdb_simple_settings* st);

}  // namespace cfdb
