// Internal declarations of the C++ shim that implements the reference's
// link-time GPU seam on top of libcfdb's C ABI (include/cfdb.h).  Compiled
// against the reference's own, unmodified headers.
#pragma once

#include <string>

#include "cfd/algebra/LinearSolver.hpp"
#include "cfd/boundary/BoundaryCondition.hpp"
#include "cfd/fields/ScalarField.hpp"
#include "cfd/fields/VectorField.hpp"
#include "cfd/mesh/Mesh.hpp"
#include "cfd/physics/BoussinesqBuoyancy.hpp"
#include "cfd/physics/FluidProperties.hpp"
#include "cfd/pressure_velocity/SIMPLEProgress.hpp"
#include "cfd/pressure_velocity/SIMPLEResult.hpp"
#include "cfd/pressure_velocity/SIMPLESettings.hpp"
#include "cfd/turbulence/TurbulenceModel.hpp"
#include "cfdb.h"

namespace cfdb_shim {

// One cfdb context on device 0 for the calling thread's GPU work; throws
// std::runtime_error when no usable device is present.
cfdb_context* thread_context();

// The reference's linear-solver settings as cfdb settings: CG / BiCGSTAB,
// None / Jacobi, tolerances and iteration cap.  The preconditioner of CG
// solves can be switched by the environment variable
// CFDB_GPU_CG_PRECONDITIONER = none | jacobi | learned_mg (unset: as the
// settings ask); learned_mg selects the learned preconditioner inside
// flexible CG, which the reference's settings cannot name.
cfdb_linear_settings linear_settings(const cfd::algebra::LinearSolverSettings& s);

// The message of the context's last error.
std::string last_error(cfdb_context* ctx);

// The reference's own CPU SIMPLE loop (src/pressure_velocity/SIMPLE.cpp,
// compiled under another class name beside this shim), for the
// configurations the GPU loop does not take.
cfd::pressure_velocity::SIMPLEResult solve_with_reference_cpu(
    const cfd::pressure_velocity::SIMPLESettings& settings, cfd::Index referenceCell,
    cfd::turbulence::TurbulenceModel* turbulenceModel, const cfd::fields::ScalarField* temperature,
    const cfd::physics::BoussinesqBuoyancy* buoyancy,
    const cfd::pressure_velocity::SIMPLEProgressCallback& progressCallback,
    const cfd::pressure_velocity::SIMPLECancellationCheck& cancellationCheck,
    const cfd::fields::VectorField* momentumSource, const cfd::mesh::Mesh& mesh,
    const cfd::physics::FluidProperties& fluid,
    const cfd::boundary::BoundaryConditionSet& velocityBoundaries,
    const cfd::boundary::BoundaryConditionSet& pressureBoundaries,
    cfd::fields::VectorField initialVelocity, cfd::fields::ScalarField initialPressure);

}  // namespace cfdb_shim
