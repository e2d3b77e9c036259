// cfd::pressure_velocity::SIMPLE (include/cfd/pressure_velocity/SIMPLE.hpp,
// unmodified) with its outer loop on the GPU.
//
// This translation unit replaces the reference's SIMPLE.cpp in a link with
// libcfdb.  SIMPLE::solve takes the GPU loop (cfdb_simple_* sessions: every
// stage on the device, only scalars cross per outer iteration) when the
// caller asks for the GPU on both linear solvers -- `"backend": "GPU"` for
// the momentum and the pressure solver in solver.json, the condition under
// which the reference runs its own resident loop (SIMPLE.cpp:348-380) -- and
// the case is one the device path implements: a uniform Cartesian mesh of
// MeshGeometry::createCartesian2D/3D, laminar flow with constant
// properties, Wall / MovingWall / Inlet / Outlet velocity and FixedGradient
// / FixedValue pressure patches, Green-Gauss gradients, no momentum source,
// temperature or buoyancy, and no adaptive relaxation or CPU solver
// fallback; rectilinear 2D meshes (createRectilinear2D / createGraded2D) are
// taken too.  Every other call runs the reference's own loop (compiled
// beside the shim as ReferenceCpuSIMPLE, simple_reference_bridge.cpp), and
// the reason the GPU loop was not taken is recorded in
// gpuDiscretizationFallbackReason, as the reference records its own
// refusals (SIMPLE.cpp:307-324); its linear solves still reach the GPU
// through cfd::gpu::makeGpuCG / makeGpuBiCGSTAB when their backend is GPU.
//
// The GPU loop keeps the reference's contract: the same statuses
// (configuration errors are left to the reference loop, which reports them
// as InvalidConfiguration), the residual histories and final residuals of
// every completed outer iteration, the progress callback and cancellation
// check once per outer iteration, and the convergence decision of the
// reference's own OuterIterationMonitor (SolverRobustness.cpp:361-384) fed
// with the device's residuals.  Setting CFDB_GPU_SIMPLE=0 in the
// environment keeps every solve on the reference loop.
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "cfd/algebra/LinearSolverFallback.hpp"
#include "cfd/boundary/FixedGradient.hpp"
#include "cfd/boundary/FixedValue.hpp"
#include "cfd/boundary/Inlet.hpp"
#include "cfd/boundary/MovingWall.hpp"
#include "cfd/boundary/Outlet.hpp"
#include "cfd/boundary/Wall.hpp"
#include "cfd/core/Exception.hpp"
#include "cfd/core/Logger.hpp"
#include "cfd/mesh/MeshGeometry.hpp"
#include "cfd/mesh/MeshGrading.hpp"
#include "cfd/pressure_velocity/SIMPLE.hpp"
#include "cfd/solver/SolverRobustness.hpp"
#include "cfdb_shim.hpp"

namespace cfdb_shim {
namespace {

using cfd::Index;
using cfd::Real;
using cfd::pressure_velocity::SIMPLEResult;
using cfd::pressure_velocity::SIMPLESettings;
using cfd::pressure_velocity::SIMPLEStatus;

bool same_vec(const cfd::Vector2& a, const cfd::Vector2& b) {
  return a.x == b.x && a.y == b.y && a.z == b.z;
}

bool same_mesh(const cfd::mesh::Mesh& ref, const cfd::mesh::Mesh& mesh) {
  bool same = ref.numberOfCells() == mesh.numberOfCells() &&
              ref.numberOfFaces() == mesh.numberOfFaces() &&
              ref.boundaryPatches().size() == mesh.boundaryPatches().size();
  for (Index c = 0; same && c < mesh.numberOfCells(); ++c)
    same = same_vec(ref.cell(c).centroid(), mesh.cell(c).centroid()) &&
           ref.cell(c).volume() == mesh.cell(c).volume();
  for (Index f = 0; same && f < mesh.numberOfFaces(); ++f) {
    const cfd::mesh::Face& a = ref.face(f);
    const cfd::mesh::Face& b = mesh.face(f);
    same = a.owner() == b.owner() && a.neighbor() == b.neighbor() &&
           same_vec(a.centroid(), b.centroid()) && same_vec(a.areaVector(), b.areaVector());
  }
  for (size_t p = 0; same && p < mesh.boundaryPatches().size(); ++p)
    same = ref.boundaryPatches()[p].name() == mesh.boundaryPatches()[p].name() &&
           ref.boundaryPatches()[p].faceIds() == mesh.boundaryPatches()[p].faceIds();
  return same;
}

// A 2D structured block whose vertices form a tensor product of two node
// lists and whose mesh is exactly createRectilinear2D of them
// (MeshGeometry.cpp:518-555, createGraded2D included); fills the grid and
// the node coordinates on success.
bool rectilinear_2d(const cfd::mesh::Mesh& mesh, cfdb_grid* g, std::vector<double> nodes[3],
                    std::string* why) {
  const cfd::mesh::StructuredGrid* sg = mesh.structuredGrid();
  if (!sg || sg->isThreeDimensional() || sg->vertices.size() != (sg->nx + 1) * (sg->ny + 1))
    return false;
  const Index nx = sg->nx, ny = sg->ny;
  std::vector<double> xn(nx + 1), yn(ny + 1);
  for (Index i = 0; i <= nx; ++i) xn[i] = sg->vertex(i, 0).x;
  for (Index j = 0; j <= ny; ++j) yn[j] = sg->vertex(0, j).y;
  for (Index j = 0; j <= ny; ++j)
    for (Index i = 0; i <= nx; ++i)
      if (sg->vertex(i, j).x != xn[i] || sg->vertex(i, j).y != yn[j]) return false;
  try {
    const cfd::mesh::Mesh ref = cfd::mesh::MeshGeometry::createRectilinear2D(
        cfd::mesh::AxisSpacing::fromNodes(xn), cfd::mesh::AxisSpacing::fromNodes(yn));
    if (!same_mesh(ref, mesh)) return false;
  } catch (const cfd::InvalidArgumentError&) {
    return false;
  }
  g->dim = 2;
  g->n[0] = static_cast<int64_t>(nx);
  g->n[1] = static_cast<int64_t>(ny);
  g->n[2] = 1;
  g->len[0] = xn[nx] - xn[0];
  g->len[1] = yn[ny] - yn[0];
  g->len[2] = 1.0;
  nodes[0] = std::move(xn);
  nodes[1] = std::move(yn);
  (void)why;
  return true;
}

// The mesh is exactly createCartesian2D/3D(n..., L...) (same cells, faces,
// patches and geometry, bit for bit); fills the grid on success.
bool uniform_cartesian(const cfd::mesh::Mesh& mesh, cfdb_grid* g, std::string* why) {
  const cfd::mesh::StructuredGrid* sg = mesh.structuredGrid();
  if (!sg || mesh.structuredBlocks().size() > 1) {
    *why = "the mesh is not one structured block";
    return false;
  }
  const int dim = sg->isThreeDimensional() ? 3 : 2;
  const Index n[3] = {sg->nx, sg->ny, dim == 3 ? sg->nz : 1};
  if (n[0] < 2 || n[1] < 2 || (dim == 3 && n[2] < 2) || mesh.numberOfCells() != n[0] * n[1] * n[2]) {
    *why = "the structured block does not match the cell count";
    return false;
  }
  // the uniform spacing from the first cell's centre ((0 + 0.5) * delta),
  // then the length whose division by the cell count gives that spacing
  const cfd::Vector2& c0 = mesh.cell(0).centroid();
  const Real first[3] = {c0.x, c0.y, c0.z};
  Real len[3] = {1.0, 1.0, 1.0};
  for (int a = 0; a < dim; ++a) {
    const Real delta = 2.0 * first[a];
    Real L = delta * static_cast<Real>(n[a]);
    for (int t = 0; t < 4 && L / static_cast<Real>(n[a]) != delta; ++t)
      L = std::nextafter(L, (L / static_cast<Real>(n[a]) < delta) ? INFINITY : -INFINITY);
    if (!(L > 0.0) || L / static_cast<Real>(n[a]) != delta) {
      *why = "the cell spacing is not that of a uniform Cartesian mesh";
      return false;
    }
    len[a] = L;
  }
  const cfd::mesh::Mesh ref =
      dim == 3 ? cfd::mesh::MeshGeometry::createCartesian3D(n[0], n[1], n[2], len[0], len[1], len[2])
               : cfd::mesh::MeshGeometry::createCartesian2D(n[0], n[1], len[0], len[1]);
  if (!same_mesh(ref, mesh)) {
    *why = "the mesh differs from MeshGeometry::createCartesian" + std::to_string(dim) + "D";
    return false;
  }
  g->dim = dim;
  for (int a = 0; a < 3; ++a) {
    g->n[a] = static_cast<int64_t>(n[a]);
    g->len[a] = len[a];
  }
  return true;
}

// Patch order of the C ABI: xmin, xmax, ymin, ymax, zmin, zmax.
bool boundary_conditions(const cfd::mesh::Mesh& mesh, int dim,
                         const cfd::boundary::BoundaryConditionSet& vbcs,
                         const cfd::boundary::BoundaryConditionSet& pbcs, cfdb_simple_case* cs,
                         std::string* why) {
  for (int p = 0; p < 2 * dim; ++p) {
    const std::string name = mesh.boundaryPatches()[p].name();
    if (!vbcs.has(name) || !pbcs.has(name)) {
      *why = "patch " + name + " has no boundary condition";
      return false;
    }
    const cfd::boundary::BoundaryCondition& vb = vbcs.get(name);
    const cfd::boundary::BoundaryCondition& pb = pbcs.get(name);
    for (int c = 0; c < 3; ++c) cs->vbc_value[p][c] = 0.0;
    if (dynamic_cast<const cfd::boundary::Wall*>(&vb)) {
      cs->vbc_type[p] = CFDB_VBC_WALL;
    } else if (const auto* mw = dynamic_cast<const cfd::boundary::MovingWall*>(&vb)) {
      cs->vbc_type[p] = CFDB_VBC_MOVING_WALL;
      cs->vbc_value[p][0] = mw->velocity().x;
      cs->vbc_value[p][1] = mw->velocity().y;
      cs->vbc_value[p][2] = mw->velocity().z;
    } else if (const auto* in = dynamic_cast<const cfd::boundary::Inlet*>(&vb)) {
      cs->vbc_type[p] = CFDB_VBC_INLET;
      cs->vbc_value[p][0] = in->velocity().x;
      cs->vbc_value[p][1] = in->velocity().y;
      cs->vbc_value[p][2] = in->velocity().z;
    } else if (dynamic_cast<const cfd::boundary::Outlet*>(&vb)) {
      cs->vbc_type[p] = CFDB_VBC_OUTLET;
    } else {
      *why = "velocity condition " + std::string(vb.name()) + " on patch " + name +
             " has no device implementation";
      return false;
    }
    if (const auto* fg = dynamic_cast<const cfd::boundary::FixedGradient*>(&pb)) {
      cs->pbc_type[p] = CFDB_PBC_FIXED_GRADIENT;
      cs->pbc_value[p] = fg->gradient();
    } else if (const auto* fv = dynamic_cast<const cfd::boundary::FixedValue*>(&pb)) {
      cs->pbc_type[p] = CFDB_PBC_FIXED_VALUE;
      cs->pbc_value[p] = fv->value();
    } else {
      *why = "pressure condition " + std::string(pb.name()) + " on patch " + name +
             " has no device implementation";
      return false;
    }
  }
  return true;
}

int scheme_of(cfd::discretization::ConvectionScheme s) {
  using S = cfd::discretization::ConvectionScheme;
  switch (s) {
    case S::Upwind: return CFDB_SCHEME_UPWIND;
    case S::Central: return CFDB_SCHEME_CENTRAL;
    case S::LinearUpwind: return CFDB_SCHEME_LINEAR_UPWIND;
    case S::QUICK: return CFDB_SCHEME_QUICK;
  }
  return -1;
}

struct Plan {
  cfdb_simple_case cs{};
  cfdb_simple_settings ss{};
  cfdb_simple* session = nullptr;
  std::vector<double> nodes[3];  // node coordinates of a rectilinear mesh
};

bool gpu_loop_requested(const SIMPLESettings& s) {
  const char* env = std::getenv("CFDB_GPU_SIMPLE");
  if (env && std::string(env) == "0") return false;
  return s.momentumSolver.backend == cfd::algebra::LinearSolverBackend::GPU &&
         s.pressureSolver.backend == cfd::algebra::LinearSolverBackend::GPU;
}

// Whether the GPU loop takes this call; on success the session is created.
bool plan_gpu_loop(const SIMPLESettings& settings, Index referenceCell,
                   cfd::turbulence::TurbulenceModel* turbulence, const cfd::fields::ScalarField* T,
                   const cfd::physics::BoussinesqBuoyancy* buoyancy,
                   const cfd::fields::VectorField* momentumSource, const cfd::mesh::Mesh& mesh,
                   const cfd::physics::FluidProperties& fluid,
                   const cfd::boundary::BoundaryConditionSet& vbcs,
                   const cfd::boundary::BoundaryConditionSet& pbcs,
                   const cfd::fields::VectorField& U0, const cfd::fields::ScalarField& p0,
                   Plan* plan, std::string* why) {
  if (!cfdb_cuda_available()) {
    *why = "no usable sm_100 device";
    return false;
  }
  // configuration errors: the reference loop reports them (InvalidConfiguration)
  try {
    cfd::pressure_velocity::validateSIMPLESettings(settings);
    (void)cfd::algebra::makeLinearSolverWithFallback(settings.momentumSolver,
                                                     settings.robustness.linearSolverFallback);
    (void)cfd::algebra::makeLinearSolverWithFallback(settings.pressureSolver,
                                                     settings.robustness.linearSolverFallback);
  } catch (const cfd::InvalidArgumentError&) {
    *why = "invalid settings";
    return false;
  }
  if (U0.size() != mesh.numberOfCells() || p0.size() != mesh.numberOfCells() ||
      referenceCell >= mesh.numberOfCells()) {
    *why = "initial fields or reference cell do not fit the mesh";
    return false;
  }
  if (turbulence && turbulence->name() != "laminar") {
    *why = "turbulence model " + std::string(turbulence->name());
    return false;
  }
  if (T || buoyancy || momentumSource) {
    *why = "temperature, buoyancy or a momentum source";
    return false;
  }
  if (settings.robustness.linearSolverFallback.enabled ||
      settings.robustness.adaptiveRelaxation.enabled) {
    *why = "the linear-solver fallback or adaptive relaxation";
    return false;
  }
  if (settings.gradientScheme != cfd::discretization::GradientScheme::GreenGauss ||
      settings.nonOrthogonalCorrections > 1) {
    *why = "least-squares gradients or non-orthogonal corrector passes";
    return false;
  }
  for (const auto* ls : {&settings.momentumSolver, &settings.pressureSolver})
    if (ls->type == cfd::algebra::LinearSolverType::GMRES) {
      *why = "GMRES";
      return false;
    }
  const int scheme = scheme_of(settings.convectionScheme);
  if (scheme < 0) {
    *why = "convection scheme";
    return false;
  }
  std::string uniform_why;
  if (!uniform_cartesian(mesh, &plan->cs.grid, &uniform_why)) {
    if (!rectilinear_2d(mesh, &plan->cs.grid, plan->nodes, why)) {
      *why = uniform_why + ", and it is not a rectilinear 2D mesh either";
      return false;
    }
    for (int a = 0; a < 2; ++a) plan->cs.nodes[a] = plan->nodes[a].data();
  }
  const int dim = plan->cs.grid.dim;
  if (!boundary_conditions(mesh, dim, vbcs, pbcs, &plan->cs, why)) return false;
  plan->cs.rho = fluid.density();
  plan->cs.mu = fluid.dynamicViscosity();
  cfdb_simple_settings& ss = plan->ss;
  ss.max_outer = static_cast<int64_t>(settings.maxIterations);
  ss.alpha_u = settings.velocityRelaxation;
  ss.alpha_p = settings.pressureRelaxation;
  ss.tol_u = settings.velocityTolerance;
  ss.tol_p = settings.pressureTolerance;
  ss.tol_c = settings.continuityTolerance;
  ss.scheme = scheme;
  ss.face_flux = cfd::pressure_velocity::resolveFaceFluxScheme(settings.faceFlux, dim) ==
                         cfd::pressure_velocity::FaceFluxScheme::RhieChow
                     ? CFDB_FLUX_RHIE_CHOW
                     : CFDB_FLUX_LINEAR;
  ss.reference_cell = static_cast<int64_t>(referenceCell);
  ss.momentum = linear_settings(settings.momentumSolver);
  ss.pressure = linear_settings(settings.pressureSolver);
  cfdb_context* ctx = thread_context();
  if (cfdb_simple_create(ctx, &plan->cs, &ss, &plan->session) != CFDB_OK) {
    *why = "the device session refused the case: " + last_error(ctx);
    plan->session = nullptr;
    return false;
  }
  return true;
}

SIMPLEStatus simple_status(int s) {
  switch (s) {
    case CFDB_SIMPLE_MOMENTUM_FAILURE: return SIMPLEStatus::MomentumFailure;
    case CFDB_SIMPLE_PRESSURE_FAILURE: return SIMPLEStatus::PressureCorrectionFailure;
    case CFDB_SIMPLE_NONFINITE_STATE: return SIMPLEStatus::NonFiniteState;
    case CFDB_SIMPLE_INVALID_CONFIGURATION: return SIMPLEStatus::InvalidConfiguration;
    default: return SIMPLEStatus::MaxIterations;
  }
}

SIMPLEResult run_gpu_loop(Plan& plan, const SIMPLESettings& settings,
                          const cfd::pressure_velocity::SIMPLEProgressCallback& progress,
                          const cfd::pressure_velocity::SIMPLECancellationCheck& cancelled,
                          const cfd::mesh::Mesh& mesh, const cfd::fields::VectorField& U0,
                          const cfd::fields::ScalarField& p0) {
  const auto t0 = std::chrono::steady_clock::now();
  const auto seconds = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
  cfdb_context* ctx = thread_context();
  cfdb_simple* s = plan.session;
  const int dim = plan.cs.grid.dim;
  const bool three = dim == 3;
  const Index cells = mesh.numberOfCells();
  SIMPLEResult result;
  result.faceFlux = cfd::pressure_velocity::resolveFaceFluxScheme(settings.faceFlux, dim);
  result.gpuDiscretization = true;
  result.residentPressureSolve = true;
  result.residentSimpleLoop = true;
  std::vector<double> u(cells), v(cells), w(cells), p(cells), flux(mesh.numberOfFaces());
  bool finite = true;
  for (Index c = 0; c < cells; ++c) {
    u[c] = U0[c].x;
    v[c] = U0[c].y;
    w[c] = U0[c].z;
    p[c] = p0[c];
    finite = finite && std::isfinite(u[c]) && std::isfinite(v[c]) && std::isfinite(p[c]) &&
             (!three || std::isfinite(w[c]));
  }
  auto check = [&](cfdb_status st, const char* what) {
    if (st != CFDB_OK) {
      cfdb_simple_destroy(s);
      throw std::runtime_error(std::string("cfdb: ") + what + ": " + last_error(ctx));
    }
  };
  check(cfdb_simple_set_state(s, u.data(), v.data(), three ? w.data() : nullptr, p.data()),
        "cfdb_simple_set_state");
  SIMPLEStatus finalStatus = SIMPLEStatus::MaxIterations;
  cfd::solver::OuterIterationMonitor monitor(
      settings.robustness,
      cfd::solver::OuterConvergenceTolerances{settings.velocityTolerance,
                                              settings.pressureTolerance,
                                              settings.continuityTolerance,
                                              settings.turbulenceTolerance},
      settings.velocityRelaxation, settings.pressureRelaxation);
  result.stageSeconds.setup = seconds(t0, std::chrono::steady_clock::now());
  if (!finite) finalStatus = SIMPLEStatus::NonFiniteState;  // SIMPLE.cpp:240-246
  for (Index it = 0; finite && it < settings.maxIterations; ++it) {
    if (cancelled && cancelled()) {
      finalStatus = SIMPLEStatus::Cancelled;
      break;
    }
    double row[5] = {0, 0, 0, 0, 0};
    cfdb_simple_result r{};
    check(cfdb_simple_iterate(s, 1, row, &r), "cfdb_simple_iterate");
    result.stageSeconds.momentumSolve += r.momentum_solve_ms * 1e-3;
    result.stageSeconds.pressureSolve += r.pressure_solve_ms * 1e-3;
    result.momentumLinearIterations += static_cast<Index>(r.momentum_linear_iterations);
    result.pressureLinearIterations += static_cast<Index>(r.pressure_linear_iterations);
    if (r.status == CFDB_SIMPLE_MOMENTUM_FAILURE || r.status == CFDB_SIMPLE_NONFINITE_STATE ||
        r.status == CFDB_SIMPLE_INVALID_CONFIGURATION) {
      finalStatus = simple_status(r.status);
      break;
    }
    ++result.momentumPredictorPasses;
    if (r.status == CFDB_SIMPLE_PRESSURE_FAILURE) {
      finalStatus = SIMPLEStatus::PressureCorrectionFailure;
      break;
    }
    ++result.pressureCorrectionPasses;
    result.uResidualHistory.push_back(r.final_u);
    result.vResidualHistory.push_back(r.final_v);
    result.pressureResidualHistory.push_back(r.final_p);
    result.continuityHistory.push_back(r.final_continuity);
    if (three) result.wResidualHistory.push_back(r.final_w);
    result.iterations = it + 1;
    result.finalUResidual = r.final_u;
    result.finalVResidual = r.final_v;
    result.finalWResidual = three ? r.final_w : 0.0;
    result.finalPressureResidual = r.final_p;
    result.finalContinuityResidual = r.final_continuity;
    result.globalMassImbalance = r.global_imbalance;
    if (progress)
      progress(cfd::pressure_velocity::SIMPLEIterationProgress{
          result.iterations, settings.maxIterations, r.final_u, r.final_v, r.final_p,
          r.final_continuity, r.global_imbalance, result.finalWResidual, three});
    const cfd::solver::OuterIterationVerdict verdict = monitor.record(cfd::solver::OuterResidualSample{
        r.final_u, r.final_v, r.final_p, r.final_continuity, r.global_imbalance, std::nullopt,
        three ? std::optional<Real>(r.final_w) : std::nullopt});
    if (verdict == cfd::solver::OuterIterationVerdict::Converged) {
      finalStatus = SIMPLEStatus::Converged;
      break;
    }
    if (verdict == cfd::solver::OuterIterationVerdict::Diverging) {
      finalStatus = SIMPLEStatus::Diverging;
      break;
    }
    if (verdict == cfd::solver::OuterIterationVerdict::Stagnated) {
      finalStatus = SIMPLEStatus::Stagnated;
      break;
    }
  }
  check(cfdb_simple_get_state(s, u.data(), v.data(), three ? w.data() : nullptr, p.data(),
                              flux.data()),
        "cfdb_simple_get_state");
  cfdb_simple_destroy(s);
  plan.session = nullptr;
  result.velocity = cfd::fields::VectorField(cells);
  result.pressure = cfd::fields::ScalarField(cells);
  result.massFlux = cfd::fields::SurfaceField(mesh.numberOfFaces());
  for (Index c = 0; c < cells; ++c) {
    result.velocity[c] = cfd::Vector2{u[c], v[c], three ? w[c] : 0.0};
    result.pressure[c] = p[c];
  }
  for (Index f = 0; f < mesh.numberOfFaces(); ++f) result.massFlux[f] = flux[f];
  result.status = finalStatus;
  result.robustness = monitor.takeDiagnostics();
  result.stageSeconds.total = seconds(t0, std::chrono::steady_clock::now());
  return result;
}

}  // namespace
}  // namespace cfdb_shim

namespace cfd::pressure_velocity {

SIMPLE::SIMPLE(SIMPLESettings settings, Index referenceCell,
               cfd::turbulence::TurbulenceModel* turbulenceModel,
               const cfd::fields::ScalarField* temperature,
               const cfd::physics::BoussinesqBuoyancy* buoyancy,
               SIMPLEProgressCallback progressCallback, SIMPLECancellationCheck cancellationCheck)
    : settings_(std::move(settings)),
      referenceCell_(referenceCell),
      turbulenceModel_(turbulenceModel),
      temperature_(temperature),
      buoyancy_(buoyancy),
      progressCallback_(std::move(progressCallback)),
      cancellationCheck_(std::move(cancellationCheck)) {}

const SIMPLESettings& SIMPLE::settings() const noexcept { return settings_; }
Index SIMPLE::referenceCell() const noexcept { return referenceCell_; }
void SIMPLE::setMomentumSource(const cfd::fields::VectorField* source) noexcept {
  momentumSource_ = source;
}
const cfd::fields::VectorField* SIMPLE::momentumSource() const noexcept { return momentumSource_; }

SIMPLEResult SIMPLE::solve(const cfd::mesh::Mesh& mesh, const cfd::physics::FluidProperties& fluid,
                           const cfd::boundary::BoundaryConditionSet& velocityBoundaries,
                           const cfd::boundary::BoundaryConditionSet& pressureBoundaries,
                           cfd::fields::VectorField initialVelocity,
                           cfd::fields::ScalarField initialPressure) const {
  std::string reason;
  if (cfdb_shim::gpu_loop_requested(settings_)) {
    cfdb_shim::Plan plan;
    if (cfdb_shim::plan_gpu_loop(settings_, referenceCell_, turbulenceModel_, temperature_,
                                 buoyancy_, momentumSource_, mesh, fluid, velocityBoundaries,
                                 pressureBoundaries, initialVelocity, initialPressure, &plan,
                                 &reason))
      return cfdb_shim::run_gpu_loop(plan, settings_, progressCallback_, cancellationCheck_, mesh,
                                     initialVelocity, initialPressure);
    cfd::Logger::instance().warning("SIMPLE: GPU outer loop not taken (" + reason +
                                    "); running the reference loop");
  }
  SIMPLEResult result = cfdb_shim::solve_with_reference_cpu(
      settings_, referenceCell_, turbulenceModel_, temperature_, buoyancy_, progressCallback_,
      cancellationCheck_, momentumSource_, mesh, fluid, velocityBoundaries, pressureBoundaries,
      std::move(initialVelocity), std::move(initialPressure));
  if (!reason.empty() && result.gpuDiscretizationFallbackReason.empty())
    result.gpuDiscretizationFallbackReason = reason;
  return result;
}

}  // namespace cfd::pressure_velocity
