// The reference's link-time GPU seam implemented on libcfdb.
//
// The reference compiles exactly one implementation of its GPU interfaces
// into its core library: CPU stubs (src/gpu/*.cpp) or its CUDA library
// (src/CMakeLists.txt:311-317).  This translation unit takes that slot for
// the linear-solver part of the seam:
//   cfd::gpu::cudaAvailable        include/cfd/gpu/GPUBackend.hpp:15
//   cfd::gpu::makeGpuCG            include/cfd/gpu/GpuLinearSolver.hpp:48-50
//   cfd::gpu::makeGpuBiCGSTAB      include/cfd/gpu/GpuLinearSolver.hpp:52-54
//   cfd::gpu::gpuExecutionStats    include/cfd/gpu/GPUExecutionStats.hpp:146-150
// so that the reference's own LinearSolverFactory (src/algebra/
// LinearSolverFactory.cpp:14-33), and every SIMPLE solve whose
// solver.json asks for "backend": "GPU", reach libcfdb unchanged.  A solve
// hands the CSR LinearSystem to cfdb_csr_solve_host, which recognises the
// structured 5-/7-point operator of the reference's Cartesian meshes and
// solves it on the device.  A system of another shape is refused with
// SolverStatus::InvalidSystem and a logged reason: there is no CPU solver
// behind this seam.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cfd/algebra/LinearSystem.hpp"
#include "cfd/algebra/Preconditioner.hpp"
#include "cfd/core/Logger.hpp"
#include "cfd/gpu/GPUBackend.hpp"
#include "cfd/gpu/GPUExecutionStats.hpp"
#include "cfd/gpu/GpuLinearSolver.hpp"
#include "cfdb_shim.hpp"

static_assert(sizeof(cfd::Index) == sizeof(uint64_t), "CSR indices are 64-bit");

namespace cfd::gpu {

bool cudaAvailable() { return cfdb_cuda_available() != 0; }

GPUExecutionStats& gpuExecutionStats() noexcept {
  static GPUExecutionStats stats;
  return stats;
}

void resetGpuExecutionStats() noexcept { gpuExecutionStats() = GPUExecutionStats{}; }

}  // namespace cfd::gpu

namespace cfdb_shim {

using cfd::algebra::LinearSolverType;
using cfd::algebra::PreconditionerType;
using cfd::algebra::SolverStatus;

cfdb_context* thread_context() {
  // One context per host thread, created on first use and kept for the
  // life of the process (the reference's GPU state is per thread too).
  thread_local cfdb_context* ctx = nullptr;
  if (!ctx) {
    if (cfdb_create(0, nullptr, &ctx) != CFDB_OK || !ctx)
      throw std::runtime_error("cfdb: no usable sm_100 device for the GPU backend");
  }
  return ctx;
}

std::string last_error(cfdb_context* ctx) {
  const char* m = ctx ? cfdb_last_error(ctx) : nullptr;
  return m ? std::string(m) : std::string();
}

cfdb_linear_settings linear_settings(const cfd::algebra::LinearSolverSettings& s) {
  cfdb_linear_settings c{};
  c.krylov = s.type == LinearSolverType::CG ? CFDB_KRYLOV_CG : CFDB_KRYLOV_BICGSTAB;
  c.preconditioner = s.preconditioner == PreconditionerType::Jacobi ? CFDB_PRECOND_JACOBI
                                                                     : CFDB_PRECOND_NONE;
  c.precision = CFDB_PRECISION_FP64;
  c.abs_tol = s.absoluteTolerance;
  c.rel_tol = s.relativeTolerance;
  c.max_iterations = static_cast<int64_t>(s.maxIterations);
  if (s.type == LinearSolverType::CG) {
    if (const char* env = std::getenv("CFDB_GPU_CG_PRECONDITIONER")) {
      const std::string v(env);
      if (v == "learned_mg") c.preconditioner = CFDB_PRECOND_LEARNED_MG;
      else if (v == "jacobi") c.preconditioner = CFDB_PRECOND_JACOBI;
      else if (v == "none") c.preconditioner = CFDB_PRECOND_NONE;
    }
  }
  return c;
}

namespace {

SolverStatus solver_status(int s) {
  switch (s) {
    case CFDB_SOLVER_CONVERGED: return SolverStatus::Converged;
    case CFDB_SOLVER_MAX_ITERATIONS: return SolverStatus::MaxIterations;
    case CFDB_SOLVER_BREAKDOWN: return SolverStatus::Breakdown;
    case CFDB_SOLVER_NONFINITE_INPUT: return SolverStatus::NonFiniteInput;
    case CFDB_SOLVER_NONFINITE_RESIDUAL: return SolverStatus::NonFiniteResidual;
    default: return SolverStatus::InvalidSystem;
  }
}

// A cfd::algebra::LinearSolver whose solve() runs on the device through
// cfdb_csr_solve_host.  Like the reference's GPU solvers it keeps its device
// buffers between solves (mutable state behind a const solve(), one host
// thread, GpuLinearSolverCuda.cpp:327-334).
class CfdbLinearSolver final : public cfd::algebra::LinearSolver {
 public:
  explicit CfdbLinearSolver(cfd::algebra::LinearSolverSettings settings)
      : LinearSolver(settings) {}
  ~CfdbLinearSolver() override {
    if (solver_) cfdb_csr_solver_destroy(solver_);
  }
  using LinearSolver::solve;

  cfd::algebra::SolverResult solve(const cfd::algebra::LinearSystem& system,
                                   const cfd::algebra::Vector& initialGuess) const override {
    const auto t0 = std::chrono::steady_clock::now();
    const cfd::algebra::SparseMatrix& A = system.matrix();
    const cfd::algebra::Vector& b = system.rhs();
    const cfd::Index n = system.size();
    cfd::algebra::SolverResult result;
    result.solution = initialGuess;
    result.backendUsed = cfd::algebra::LinearSolverBackend::GPU;
    if (initialGuess.size() != n) {  // as CG.cpp:23-26
      result.status = SolverStatus::NonFiniteInput;
      return result;
    }
    cfdb_context* ctx = thread_context();
    if (!solver_ && cfdb_csr_solver_create(ctx, &solver_) != CFDB_OK)
      throw std::runtime_error("cfdb: cfdb_csr_solver_create failed: " + last_error(ctx));
    const cfdb_linear_settings cs = linear_settings(settings_);
    const int64_t cap = std::min<int64_t>(cs.max_iterations + 1, int64_t(1) << 24);
    std::vector<double> hist(static_cast<size_t>(std::max<int64_t>(cap, 1)));
    cfdb_linear_result r{};
    cfdb_csr_info info{};
    const cfdb_status st = cfdb_csr_solve_host(
        solver_, &cs, static_cast<int64_t>(n), reinterpret_cast<const uint64_t*>(A.rowOffsetsData()),
        reinterpret_cast<const uint64_t*>(A.columnIndicesData()), A.valuesData(), b.data(),
        result.solution.data(), hist.data(), cap, &r, &info);
    if (st == CFDB_ERR_UNSUPPORTED) {
      cfd::Logger::instance().warning("cfdb GPU solver: " + last_error(ctx) +
                                      " -- reported as InvalidSystem (no CPU solver behind the "
                                      "GPU backend)");
      result.solution = initialGuess;
      result.status = SolverStatus::InvalidSystem;
      return result;
    }
    if (st != CFDB_OK) throw std::runtime_error("cfdb: " + last_error(ctx));
    if (info.learned_declined)
      cfd::Logger::instance().warning(
          "cfdb GPU solver: the learned preconditioner needs the p' face operator; this system "
          "was solved by Jacobi-PCG");
    result.status = solver_status(r.status);
    result.iterations = static_cast<cfd::Index>(r.iterations);
    result.initialResidual = r.initial_residual;
    result.finalResidual = r.final_residual;
    result.restarts = static_cast<cfd::Index>(r.restarts);
    if (r.status != CFDB_SOLVER_NONFINITE_INPUT && r.status != CFDB_SOLVER_INVALID_SYSTEM) {
      int64_t m = r.iterations + 1;
      if (cs.preconditioner == CFDB_PRECOND_LEARNED_MG && info.path == CFDB_CSR_PATH_FACES)
        m = r.iterations - r.fallback_iterations + 1;
      m = std::min(m, cap);
      result.residualHistory.assign(hist.begin(), hist.begin() + m);
    }
    // execution statistics (GPUExecutionStats.hpp:16-150)
    auto& stats = cfd::gpu::gpuExecutionStats();
    const uint64_t vec = static_cast<uint64_t>(n) * sizeof(double);
    const uint64_t bands = info.path == CFDB_CSR_PATH_FACES
                               ? 0
                               : static_cast<uint64_t>(n) * 7 * sizeof(double);
    stats.hostToDeviceBytes += 2 * vec + bands;
    stats.hostToDeviceCalls += info.path == CFDB_CSR_PATH_FACES ? 2 : 9;
    stats.deviceToHostBytes += vec + static_cast<uint64_t>(result.residualHistory.size()) * 8;
    stats.deviceToHostCalls += 2;
    stats.kernelLaunches += static_cast<uint64_t>(r.kernel_launches);
    stats.kernelSeconds += r.device_ms * 1e-3;
    stats.synchronizations += 1;
    stats.gpuLinearSolves += 1;
    stats.gpuLinearSolverIterations += static_cast<uint64_t>(r.iterations);
    stats.gpuSolveSeconds +=
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return result;
  }

 private:
  mutable cfdb_csr_solver* solver_ = nullptr;
};

// The reference's factories take an optional caller-built preconditioner
// object; the device solvers apply Jacobi themselves, so a Jacobi object is
// honoured as the Jacobi setting and any other object is not served here.
bool preconditioner_supported(const std::shared_ptr<cfd::algebra::Preconditioner>& p,
                              cfd::algebra::LinearSolverSettings& settings) {
  if (!p) return true;
  if (dynamic_cast<const cfd::algebra::JacobiPreconditioner*>(p.get())) {
    settings.preconditioner = PreconditionerType::Jacobi;
    return true;
  }
  cfd::Logger::instance().warning(
      "cfdb GPU backend: a caller-supplied preconditioner other than Jacobi has no device "
      "implementation");
  return false;
}

}  // namespace
}  // namespace cfdb_shim

namespace cfd::gpu {

std::unique_ptr<cfd::algebra::LinearSolver> makeGpuCG(
    cfd::algebra::LinearSolverSettings settings,
    std::shared_ptr<cfd::algebra::Preconditioner> preconditioner) {
  if (!cudaAvailable() || !cfdb_shim::preconditioner_supported(preconditioner, settings))
    return nullptr;
  settings.type = cfd::algebra::LinearSolverType::CG;
  return std::make_unique<cfdb_shim::CfdbLinearSolver>(settings);
}

std::unique_ptr<cfd::algebra::LinearSolver> makeGpuBiCGSTAB(
    cfd::algebra::LinearSolverSettings settings,
    std::shared_ptr<cfd::algebra::Preconditioner> preconditioner) {
  if (!cudaAvailable() || !cfdb_shim::preconditioner_supported(preconditioner, settings))
    return nullptr;
  settings.type = cfd::algebra::LinearSolverType::BiCGSTAB;
  return std::make_unique<cfdb_shim::CfdbLinearSolver>(settings);
}

}  // namespace cfd::gpu
