// Driver around the reference's own CPU implementation of the SIMPLE / p'
// path, linked against oracle/_ref/libcfdref.a (built from the reference's
// sources by oracle/Makefile.ref).  Test infrastructure only: it produces
// golden vectors and the timed CPU baseline; the product never links it.
//
// Commands (key=value arguments, binary float64 outputs under out=DIR):
//
//   poisson dim=2|3 n=N [seed=S] [rtol=1e-8] [maxit=M] [pre=jacobi|none]
//           [solver=cg|bicgstab] [out=DIR] [dump_matrix=1] [direct=1] [repeat=R]
//           [check_direct=1] [maxits=a,b,...]
//       p' system of the reference's assemblePressureCorrection
//       (PressureCorrectionEquation.cpp:341) with unit response
//       coefficients, rho = 1, all-FixedGradient(0) pressure patches and
//       cell 0 pinned, on createCartesian2D(n,n,1,1) /
//       createCartesian3D(n,n,n,1,1,1); RHS = oracle_synth_rhs(seed);
//       solved by the reference CG (CG.cpp:14) + JacobiPreconditioner
//       (Preconditioner.cpp:34) from x0 = 0 with absoluteTolerance = 0.
//
//   simple dim=2|3 nx= ny= [nz=] [lx=1 ly=1 lz=1] [rho=1] [mu=0.01]
//          [flow=cavity|channel] [lid=1] [inlet=1] [au=0.7] [ap=0.3]
//          [tolu=1e-6] [tolp=1e-6] [tolc=1e-6] [outer=N]
//          [scheme=upwind|central|lud|quick] [flux=auto|linear|rhiechow]
//          [mabs=1e-10] [mrel=1e-8] [mmax=500]
//          [psolver=cg|bicgstab] [ppre=jacobi|none] [pabs=0] [prel=1e-8] [pmax=5000]
//          [mbackend=cpu|gpu] [pbackend=cpu|gpu] [gradex=R gradey=R cluster=both|start|end]
//          [out=DIR]
//       the reference SIMPLE::solve (SIMPLE.cpp:148) on a uniform Cartesian
//       lid-driven cavity (Wall x3 + MovingWall{lid,0}) or channel (Inlet
//       {inlet,0} left, Outlet right, Walls; pressure FixedValue(0) at the
//       outlet), pressure FixedGradient(0) elsewhere.  Writes u v [w] p flux
//       and the residual histories.
//
//   csr in=DIR [solver=bicgstab|cg] [pre=none|jacobi] [atol=1e-12] [rtol=1e-10]
//       [maxit=1000] [out=DIR]
//       a stored CSR LinearSystem (DIR/{offsets,columns}.bin as uint64,
//       DIR/{values,rhs,x0}.bin as float64) solved by the reference BiCGSTAB
//       (BiCGSTAB.cpp:48) or CG from the stored initial guess; writes the
//       solution and the residual history.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <stdexcept>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "cfd/algebra/BiCGSTAB.hpp"
#include "cfd/algebra/CG.hpp"
#include "cfd/algebra/LinearSystem.hpp"
#include "cfd/algebra/Preconditioner.hpp"
#include "cfd/boundary/FixedGradient.hpp"
#include "cfd/boundary/FixedValue.hpp"
#include "cfd/boundary/Inlet.hpp"
#include "cfd/boundary/MovingWall.hpp"
#include "cfd/boundary/Outlet.hpp"
#include "cfd/boundary/Wall.hpp"
#include "cfd/fields/ScalarField.hpp"
#include "cfd/fields/SurfaceField.hpp"
#include "cfd/fields/VectorField.hpp"
#include "cfd/gpu/GPUExecutionStats.hpp"
#include "cfd/mesh/MeshGeometry.hpp"
#include "cfd/mesh/MeshGrading.hpp"
#include "cfd/physics/FluidProperties.hpp"
#include "cfd/pressure_velocity/PressureCorrectionEquation.hpp"
#include "cfd/pressure_velocity/SIMPLE.hpp"
#include "synth_rhs.h"

#ifdef _OPENMP
#include <omp.h>
static int ompThreads() { return omp_get_max_threads(); }
#else
static int ompThreads() { return 1; }
#endif

using namespace cfd;

namespace {

using Args = std::map<std::string, std::string>;

std::string get(const Args& a, const std::string& k, const std::string& d) {
  auto it = a.find(k);
  return it == a.end() ? d : it->second;
}
double getd(const Args& a, const std::string& k, double d) {
  auto it = a.find(k);
  return it == a.end() ? d : std::strtod(it->second.c_str(), nullptr);
}
long long geti(const Args& a, const std::string& k, long long d) {
  auto it = a.find(k);
  return it == a.end() ? d : std::strtoll(it->second.c_str(), nullptr, 10);
}

void writeBin(const std::string& path, const double* data, size_t n) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(data), static_cast<std::streamsize>(n * sizeof(double)));
}
void writeBin(const std::string& path, const std::vector<double>& v) {
  writeBin(path, v.data(), v.size());
}

const char* solverStatusText(algebra::SolverStatus s) {
  switch (s) {
    case algebra::SolverStatus::Converged: return "Converged";
    case algebra::SolverStatus::MaxIterations: return "MaxIterations";
    case algebra::SolverStatus::Breakdown: return "Breakdown";
    case algebra::SolverStatus::NonFiniteInput: return "NonFiniteInput";
    case algebra::SolverStatus::NonFiniteResidual: return "NonFiniteResidual";
    case algebra::SolverStatus::InvalidSystem: return "InvalidSystem";
  }
  return "?";
}

const char* simpleStatusName(pressure_velocity::SIMPLEStatus s) {
  using S = pressure_velocity::SIMPLEStatus;
  switch (s) {
    case S::Converged: return "Converged";
    case S::MaxIterations: return "MaxIterations";
    case S::MomentumFailure: return "MomentumFailure";
    case S::PressureCorrectionFailure: return "PressureCorrectionFailure";
    case S::NonFiniteState: return "NonFiniteState";
    case S::InvalidConfiguration: return "InvalidConfiguration";
    case S::Cancelled: return "Cancelled";
    case S::Stagnated: return "Stagnated";
    case S::Diverging: return "Diverging";
  }
  return "?";
}

mesh::Mesh makeMesh(int dim, long long nx, long long ny, long long nz, double lx, double ly,
                    double lz) {
  if (dim == 3) return mesh::MeshGeometry::createCartesian3D(nx, ny, nz, lx, ly, lz);
  return mesh::MeshGeometry::createCartesian2D(nx, ny, lx, ly);
}

// gradex=R / gradey=R (geometric ratio, cluster=both|start|end): the 2D
// mesh of MeshGeometry::createGraded2D (MeshGeometry.hpp:236-240).
mesh::AxisGrading grading(const Args& a, const std::string& key) {
  mesh::AxisGrading g;
  const double ratio = getd(a, key, 1.0);
  if (ratio != 1.0) {
    g.type = mesh::GradingType::Geometric;
    g.ratio = ratio;
    const std::string c = get(a, "cluster", "both");
    g.cluster = c == "start" ? mesh::GradingCluster::Start
                : c == "end" ? mesh::GradingCluster::End
                             : mesh::GradingCluster::Both;
  }
  return g;
}

// The isolated p' matrix through the reference's own assembly
// (assemblePressureCorrection with unit response, rho = 1, Neumann patches,
// cell 0 pinned).
algebra::SparseMatrix referenceMatrix(const mesh::Mesh& m, int dim) {
  const Index cells = m.numberOfCells();
  boundary::BoundaryConditionSet pBCs;
  for (const auto& patch : m.boundaryPatches())
    pBCs.set(m, patch.name(), std::make_unique<boundary::FixedGradient>(0.0));
  const fields::ScalarField one(cells, 1.0);
  const fields::SurfaceField zeroFlux(m.numberOfFaces(), 0.0);
  pressure_velocity::PressureCorrectionOptions opts;
  auto assembly = pressure_velocity::assemblePressureCorrection(
      m, zeroFlux, one, one, 1.0, 0, pBCs, opts, dim == 3 ? &one : nullptr);
  return algebra::SparseMatrix(assembly.system.matrix());
}

// The same matrix written directly in CSR (ascending columns, diagonal summed
// in face order, same coefficient expression), O(n) instead of the triplet
// sort: only used to keep the timed CPU-baseline setup short at 2048^2 /
// 256^3; `check_direct=1` verifies it equals referenceMatrix bit for bit.
algebra::SparseMatrix directMatrix(const mesh::Mesh& m, int dim, long long n) {
  const Index cells = m.numberOfCells();
  const double delta = 1.0 / static_cast<double>(n);
  const double area = dim == 3 ? delta * delta : delta;
  std::vector<double> coef(n + 1, 0.0);
  for (long long f = 1; f < n; ++f) {
    const double cP = (static_cast<double>(f - 1) + 0.5) * delta;
    const double cN = (static_cast<double>(f) + 0.5) * delta;
    const double node = static_cast<double>(f) * delta;
    const double dPf = std::fabs(node - cP), dNf = std::fabs(node - cN);
    const double dFace = ((dNf * 1.0) + (dPf * 1.0)) / (dPf + dNf);
    coef[f] = 1.0 * area * dFace / std::fabs(cN - cP);
  }
  const long long nx = n, ny = n, nz = dim == 3 ? n : 1;
  const long long stride[3] = {1, nx, nx * ny};
  std::vector<Index> offsets(cells + 1, 0);
  std::vector<Index> cols;
  std::vector<double> vals;
  cols.reserve(cells * (dim == 3 ? 7 : 5));
  vals.reserve(cells * (dim == 3 ? 7 : 5));
  for (Index c = 0; c < cells; ++c) {
    const long long ijk[3] = {static_cast<long long>(c % nx), static_cast<long long>((c / nx) % ny),
                              static_cast<long long>(c / (nx * ny))};
    if (c == 0) {
      cols.push_back(0);
      vals.push_back(1.0);
      offsets[c + 1] = cols.size();
      continue;
    }
    double diag = 0.0;
    for (int ax = 0; ax < dim; ++ax) {
      if (ijk[ax] > 0) diag += coef[ijk[ax]];
      if (ijk[ax] < (ax == 2 ? nz : (ax == 1 ? ny : nx)) - 1) diag += coef[ijk[ax] + 1];
    }
    for (int ax = dim - 1; ax >= 0; --ax)
      if (ijk[ax] > 0) {
        cols.push_back(c - stride[ax]);
        vals.push_back(-coef[ijk[ax]]);
      }
    cols.push_back(c);
    vals.push_back(diag);
    for (int ax = 0; ax < dim; ++ax)
      if (ijk[ax] < (ax == 2 ? nz : (ax == 1 ? ny : nx)) - 1) {
        cols.push_back(c + stride[ax]);
        vals.push_back(-coef[ijk[ax] + 1]);
      }
    offsets[c + 1] = cols.size();
  }
  return algebra::SparseMatrix(cells, cells, std::move(vals), std::move(cols), std::move(offsets));
}

int runPoisson(const Args& a) {
  const int dim = static_cast<int>(geti(a, "dim", 2));
  const long long n = geti(a, "n", 64);
  const auto seed = static_cast<uint64_t>(geti(a, "seed", 20261203));
  const std::string out = get(a, "out", "");
  const mesh::Mesh m = makeMesh(dim, n, n, n, 1.0, 1.0, 1.0);
  const Index cells = m.numberOfCells();

  std::vector<double> b(cells);
  oracle_synth_rhs(n, n, dim == 3 ? n : 0, seed, b.data());
  algebra::Vector rhs(cells);
  for (Index i = 0; i < cells; ++i) rhs[i] = b[i];
  const bool direct = geti(a, "direct", 0) != 0;
  const algebra::LinearSystem system(direct ? directMatrix(m, dim, n) : referenceMatrix(m, dim),
                                     rhs);

  algebra::LinearSolverSettings s;
  s.absoluteTolerance = getd(a, "atol", 0.0);
  s.relativeTolerance = getd(a, "rtol", 1e-8);
  s.maxIterations = static_cast<Index>(geti(a, "maxit", 100000));
  std::shared_ptr<algebra::Preconditioner> pre;
  if (get(a, "pre", "jacobi") == "jacobi") pre = std::make_shared<algebra::JacobiPreconditioner>();
  std::unique_ptr<algebra::LinearSolver> solver;
  if (get(a, "solver", "cg") == "bicgstab")
    solver = std::make_unique<algebra::BiCGSTAB>(s, pre);
  else
    solver = std::make_unique<algebra::CG>(s, pre);

  if (geti(a, "check_direct", 0) != 0) {
    const algebra::SparseMatrix A = referenceMatrix(m, dim), B = directMatrix(m, dim, n);
    bool same = A.nonZeros() == B.nonZeros();
    for (Index k = 0; same && k < A.nonZeros(); ++k)
      same = A.valuesData()[k] == B.valuesData()[k] && A.columnIndicesData()[k] == B.columnIndicesData()[k];
    for (Index r = 0; same && r <= A.rows(); ++r) same = A.rowOffsetsData()[r] == B.rowOffsetsData()[r];
    std::printf("{\"direct_matches_reference\": %s}\n", same ? "true" : "false");
    return same ? 0 : 1;
  }
  // maxits=a,b,... times one solve from x0 = 0 per iteration budget on the
  // same matrix (the difference of two budgets is the per-iteration cost
  // without the solve's setup) and reports `maxit_seconds`.
  const std::string maxits = get(a, "maxits", "");
  if (!maxits.empty()) {
    std::string times;
    size_t pos = 0;
    while (pos <= maxits.size()) {
      const size_t comma = maxits.find(',', pos);
      const std::string tok = maxits.substr(pos, comma == std::string::npos ? std::string::npos
                                                                            : comma - pos);
      algebra::LinearSolverSettings sk = s;
      sk.maxIterations = static_cast<Index>(std::strtoll(tok.c_str(), nullptr, 10));
      std::unique_ptr<algebra::LinearSolver> sv;
      if (get(a, "solver", "cg") == "bicgstab")
        sv = std::make_unique<algebra::BiCGSTAB>(sk, pre);
      else
        sv = std::make_unique<algebra::CG>(sk, pre);
      const auto t0 = std::chrono::steady_clock::now();
      const algebra::SolverResult rk = sv->solve(system);
      const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      times += (times.empty() ? "" : ", ") + std::string("[") + tok + ", " +
               std::to_string(rk.iterations) + ", " + std::to_string(sec) + "]";
      if (comma == std::string::npos) break;
      pos = comma + 1;
    }
    std::printf("{\"maxit_seconds\": [%s], \"cells\": %zu, \"threads\": %d}\n", times.c_str(),
                static_cast<size_t>(cells), ompThreads());
    return 0;
  }
  // repeat=R times the same solve R times (each from x0 = 0); the summary
  // reports the last one and `repeat_seconds` lists all.
  const long long repeat = std::max(1LL, geti(a, "repeat", 1));
  std::string times;
  algebra::SolverResult r;
  double seconds = 0.0;
  for (long long q = 0; q < repeat; ++q) {
    const auto t0 = std::chrono::steady_clock::now();
    r = solver->solve(system);
    seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    times += (q ? ", " : "") + std::to_string(seconds);
  }

  // FP64 true residual of the returned solution.
  const algebra::Vector ax = system.matrix().multiply(r.solution);
  double rr = 0.0, bb = 0.0;
  for (Index i = 0; i < cells; ++i) {
    const double d = rhs[i] - ax[i];
    rr += d * d;
    bb += rhs[i] * rhs[i];
  }
  std::printf(
      "{\"status\": \"%s\", \"iterations\": %zu, \"initial_residual\": %.17g, "
      "\"final_residual\": %.17g, \"true_rel_residual\": %.17g, \"seconds\": %.6f, "
      "\"cells\": %zu, \"nnz\": %zu, \"threads\": %d, \"repeat_seconds\": [%s]}\n",
      solverStatusText(r.status), static_cast<size_t>(r.iterations), r.initialResidual,
      r.finalResidual, std::sqrt(rr) / std::sqrt(bb), seconds, static_cast<size_t>(cells),
      static_cast<size_t>(system.matrix().nonZeros()), ompThreads(), times.c_str());
  if (!out.empty()) {
    writeBin(out + "/rhs.bin", b);
    writeBin(out + "/x.bin", r.solution.data(), cells);
    writeBin(out + "/hist.bin", r.residualHistory);
    if (geti(a, "dump_matrix", 0) != 0) {
      const auto& A = system.matrix();
      std::vector<double> off(A.rows() + 1), col(A.nonZeros());
      for (Index i = 0; i <= A.rows(); ++i) off[i] = static_cast<double>(A.rowOffsetsData()[i]);
      for (Index k = 0; k < A.nonZeros(); ++k) col[k] = static_cast<double>(A.columnIndicesData()[k]);
      writeBin(out + "/csr_offsets.bin", off);
      writeBin(out + "/csr_columns.bin", col);
      writeBin(out + "/csr_values.bin", A.valuesData(), A.nonZeros());
    }
  }
  return 0;
}

algebra::LinearSolverSettings linSettings(const Args& a, const std::string& prefix,
                                          const std::string& type, double abs, double rel,
                                          long long maxit, const std::string& pre) {
  algebra::LinearSolverSettings s;
  s.absoluteTolerance = getd(a, prefix + "abs", abs);
  s.relativeTolerance = getd(a, prefix + "rel", rel);
  s.maxIterations = static_cast<Index>(geti(a, prefix + "max", maxit));
  s.type = get(a, prefix + "solver", type) == "cg" ? algebra::LinearSolverType::CG
                                                   : algebra::LinearSolverType::BiCGSTAB;
  s.preconditioner = get(a, prefix + "pre", pre) == "jacobi" ? algebra::PreconditionerType::Jacobi
                                                             : algebra::PreconditionerType::None;
  s.backend = get(a, prefix + "backend", "cpu") == "gpu" ? algebra::LinearSolverBackend::GPU
                                                         : algebra::LinearSolverBackend::CPU;
  return s;
}

int runSimple(const Args& a) {
  const int dim = static_cast<int>(geti(a, "dim", 2));
  const long long nx = geti(a, "nx", 16), ny = geti(a, "ny", nx), nz = geti(a, "nz", nx);
  const double lx = getd(a, "lx", 1.0), ly = getd(a, "ly", 1.0), lz = getd(a, "lz", 1.0);
  const std::string out = get(a, "out", "");
  const std::string flow = get(a, "flow", "cavity");
  const bool graded = dim == 2 && (a.count("gradex") || a.count("gradey"));
  const mesh::Mesh m = graded ? mesh::MeshGeometry::createGraded2D(nx, ny, lx, ly, grading(a, "gradex"),
                                                                    grading(a, "gradey"))
                              : makeMesh(dim, nx, ny, nz, lx, ly, lz);
  const Index cells = m.numberOfCells();
  const physics::FluidProperties fluid(getd(a, "rho", 1.0), getd(a, "mu", 0.01));

  boundary::BoundaryConditionSet vBCs, pBCs;
  const double lid = getd(a, "lid", 1.0), inlet = getd(a, "inlet", 1.0);
  for (const auto& patch : m.boundaryPatches()) {
    const std::string& name = patch.name();
    if (flow == "channel" && (name == "left" || name == "xmin")) {
      vBCs.set(m, name, std::make_unique<boundary::Inlet>(Vector2{inlet, 0.0}));
      pBCs.set(m, name, std::make_unique<boundary::FixedGradient>(0.0));
    } else if (flow == "channel" && (name == "right" || name == "xmax")) {
      vBCs.set(m, name, std::make_unique<boundary::Outlet>());
      pBCs.set(m, name, std::make_unique<boundary::FixedValue>(0.0));
    } else if (flow == "cavity" && (name == "top" || name == "ymax")) {
      vBCs.set(m, name, std::make_unique<boundary::MovingWall>(Vector2{lid, 0.0}));
      pBCs.set(m, name, std::make_unique<boundary::FixedGradient>(0.0));
    } else {
      vBCs.set(m, name, std::make_unique<boundary::Wall>());
      pBCs.set(m, name, std::make_unique<boundary::FixedGradient>(0.0));
    }
  }

  pressure_velocity::SIMPLESettings s;
  s.maxIterations = static_cast<Index>(geti(a, "outer", 1000));
  s.velocityRelaxation = getd(a, "au", 0.7);
  s.pressureRelaxation = getd(a, "ap", 0.3);
  s.velocityTolerance = getd(a, "tolu", 1e-6);
  s.pressureTolerance = getd(a, "tolp", 1e-6);
  s.continuityTolerance = getd(a, "tolc", 1e-6);
  s.momentumSolver = linSettings(a, "m", "bicgstab", 1e-10, 1e-8, 500, "none");
  s.pressureSolver = linSettings(a, "p", "cg", 0.0, 1e-8, 5000, "jacobi");
  const std::string scheme = get(a, "scheme", "upwind");
  s.convectionScheme = scheme == "central" ? discretization::ConvectionScheme::Central
                       : scheme == "lud"   ? discretization::ConvectionScheme::LinearUpwind
                       : scheme == "quick" ? discretization::ConvectionScheme::QUICK
                                           : discretization::ConvectionScheme::Upwind;
  const std::string flux = get(a, "flux", "auto");
  s.faceFlux = flux == "linear"     ? pressure_velocity::FaceFluxScheme::Linear
               : flux == "rhiechow" ? pressure_velocity::FaceFluxScheme::RhieChow
                                    : pressure_velocity::FaceFluxScheme::Automatic;

  fields::VectorField U0(cells, Vector2{0.0, 0.0});
  fields::ScalarField p0(cells, 0.0);
  const pressure_velocity::SIMPLE simple(s, 0);
  const auto t0 = std::chrono::steady_clock::now();
  const auto r = simple.solve(m, fluid, vBCs, pBCs, U0, p0);
  const double seconds =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

  std::printf(
      "{\"status\": \"%s\", \"iterations\": %zu, \"final_u\": %.17g, \"final_v\": %.17g, "
      "\"final_w\": %.17g, \"final_p\": %.17g, \"final_continuity\": %.17g, "
      "\"global_imbalance\": %.17g, \"momentum_linear_iterations\": %zu, "
      "\"pressure_linear_iterations\": %zu, \"seconds\": %.6f, \"pressure_solve_seconds\": %.6f, "
      "\"momentum_assembly_seconds\": %.6f, \"momentum_solve_seconds\": %.6f, "
      "\"pressure_assembly_seconds\": %.6f, \"cells\": %zu, \"faces\": %zu, "
      "\"gpu_simple_loop\": %s, \"gpu_fallback_reason\": \"%s\", \"gpu_linear_solves\": %llu, "
      "\"gpu_backend_fallbacks\": %llu}\n",
      simpleStatusName(r.status), static_cast<size_t>(r.iterations), r.finalUResidual,
      r.finalVResidual, r.finalWResidual, r.finalPressureResidual, r.finalContinuityResidual,
      r.globalMassImbalance, static_cast<size_t>(r.momentumLinearIterations),
      static_cast<size_t>(r.pressureLinearIterations), seconds, r.stageSeconds.pressureSolve,
      r.stageSeconds.momentumAssembly, r.stageSeconds.momentumSolve,
      r.stageSeconds.pressureAssembly, static_cast<size_t>(cells),
      static_cast<size_t>(m.numberOfFaces()), r.residentSimpleLoop ? "true" : "false",
      r.gpuDiscretizationFallbackReason.c_str(),
      static_cast<unsigned long long>(gpu::gpuExecutionStats().gpuLinearSolves),
      static_cast<unsigned long long>(gpu::gpuExecutionStats().gpuBackendFallbacks));
  if (!out.empty()) {
    std::vector<double> u(cells), v(cells), w(cells), p(cells);
    for (Index i = 0; i < cells; ++i) {
      u[i] = r.velocity[i].x;
      v[i] = r.velocity[i].y;
      w[i] = r.velocity[i].z;
      p[i] = r.pressure[i];
    }
    writeBin(out + "/u.bin", u);
    writeBin(out + "/v.bin", v);
    if (dim == 3) writeBin(out + "/w.bin", w);
    writeBin(out + "/p.bin", p);
    writeBin(out + "/flux.bin", r.massFlux.data(), r.massFlux.size());
    std::vector<double> hist;
    for (size_t k = 0; k < r.uResidualHistory.size(); ++k) {
      hist.push_back(r.uResidualHistory[k]);
      hist.push_back(r.vResidualHistory[k]);
      hist.push_back(dim == 3 ? r.wResidualHistory[k] : 0.0);
      hist.push_back(r.pressureResidualHistory[k]);
      hist.push_back(r.continuityHistory[k]);
    }
    writeBin(out + "/hist.bin", hist);
    if (graded) {  // the node coordinates of each axis (the generating vertex grid)
      const mesh::StructuredGrid* sg = m.structuredGrid();
      std::vector<double> xn(nx + 1), yn(ny + 1);
      for (long long i = 0; i <= nx; ++i) xn[i] = sg->vertex(i, 0).x;
      for (long long j = 0; j <= ny; ++j) yn[j] = sg->vertex(0, j).y;
      writeBin(out + "/x_nodes.bin", xn);
      writeBin(out + "/y_nodes.bin", yn);
    }
  }
  return 0;
}

template <typename T>
std::vector<T> readBin(const std::string& path) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) throw std::runtime_error("cannot read " + path);
  const std::streamsize bytes = f.tellg();
  f.seekg(0);
  std::vector<T> v(static_cast<size_t>(bytes) / sizeof(T));
  f.read(reinterpret_cast<char*>(v.data()), bytes);
  return v;
}

int runCsr(const Args& a) {
  const std::string in = get(a, "in", "");
  const std::string out = get(a, "out", "");
  std::vector<uint64_t> ro = readBin<uint64_t>(in + "/offsets.bin");
  std::vector<uint64_t> ci = readBin<uint64_t>(in + "/columns.bin");
  std::vector<double> va = readBin<double>(in + "/values.bin");
  const std::vector<double> rhs = readBin<double>(in + "/rhs.bin");
  const std::vector<double> x0 = readBin<double>(in + "/x0.bin");
  const Index n = ro.size() - 1;
  std::vector<Index> off(ro.begin(), ro.end()), col(ci.begin(), ci.end());
  algebra::Vector b(n), x(n);
  for (Index i = 0; i < n; ++i) {
    b[i] = rhs[i];
    x[i] = x0[i];
  }
  const algebra::LinearSystem system(
      algebra::SparseMatrix(n, n, std::move(va), std::move(col), std::move(off)), b);
  algebra::LinearSolverSettings s;
  s.absoluteTolerance = getd(a, "atol", 1e-12);
  s.relativeTolerance = getd(a, "rtol", 1e-10);
  s.maxIterations = static_cast<Index>(geti(a, "maxit", 1000));
  std::shared_ptr<algebra::Preconditioner> pre;
  if (get(a, "pre", "none") == "jacobi") pre = std::make_shared<algebra::JacobiPreconditioner>();
  std::unique_ptr<algebra::LinearSolver> solver;
  if (get(a, "solver", "bicgstab") == "cg")
    solver = std::make_unique<algebra::CG>(s, pre);
  else
    solver = std::make_unique<algebra::BiCGSTAB>(s, pre);
  const algebra::SolverResult r = solver->solve(system, x);
  const algebra::Vector ax = system.matrix().multiply(r.solution);
  double rr = 0.0;
  for (Index i = 0; i < n; ++i) rr += (b[i] - ax[i]) * (b[i] - ax[i]);
  std::printf(
      "{\"status\": \"%s\", \"iterations\": %zu, \"restarts\": %zu, \"initial_residual\": %.17g, "
      "\"final_residual\": %.17g, \"true_residual\": %.17g, \"history\": %zu}\n",
      solverStatusText(r.status), static_cast<size_t>(r.iterations),
      static_cast<size_t>(r.restarts), r.initialResidual, r.finalResidual, std::sqrt(rr),
      r.residualHistory.size());
  if (!out.empty()) {
    writeBin(out + "/x.bin", r.solution.data(), n);
    writeBin(out + "/hist.bin", r.residualHistory);
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: ref_driver poisson|simple|csr key=value ...\n");
    return 2;
  }
  Args a;
  for (int i = 2; i < argc; ++i) {
    const std::string kv = argv[i];
    const auto eq = kv.find('=');
    if (eq == std::string::npos) {
      std::fprintf(stderr, "bad argument %s\n", argv[i]);
      return 2;
    }
    a[kv.substr(0, eq)] = kv.substr(eq + 1);
  }
  const std::string cmd = argv[1];
  try {
    if (cmd == "poisson") return runPoisson(a);
    if (cmd == "simple") return runSimple(a);
    if (cmd == "csr") return runCsr(a);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_driver: %s\n", e.what());
    return 1;
  }
  std::fprintf(stderr, "unknown command %s\n", cmd.c_str());
  return 2;
}
