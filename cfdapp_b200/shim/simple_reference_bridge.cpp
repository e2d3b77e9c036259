// The reference's CPU SIMPLE loop under another class name.
//
// The shim defines cfd::pressure_velocity::SIMPLE itself (simple_resident.cpp)
// so that ProjectRunner and every other caller of the unmodified
// SIMPLE.hpp reach the GPU loop.  For the configurations that loop does not
// take it defers to the reference's own loop: the maintainer compiles the
// reference's src/pressure_velocity/SIMPLE.cpp with
// -DSIMPLE=ReferenceCpuSIMPLE, and this file -- compiled with the same
// definition -- is the one place that names that class.
#ifndef SIMPLE
#error "compile with -DSIMPLE=ReferenceCpuSIMPLE (see cfdapp_b200/shim/Makefile)"
#endif
#include "cfd/pressure_velocity/SIMPLE.hpp"
#include "cfdb_shim.hpp"

namespace cfdb_shim {

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
    cfd::fields::VectorField initialVelocity, cfd::fields::ScalarField initialPressure) {
  cfd::pressure_velocity::SIMPLE cpu(settings, referenceCell, turbulenceModel, temperature,
                                     buoyancy, progressCallback, cancellationCheck);
  cpu.setMomentumSource(momentumSource);
  return cpu.solve(mesh, fluid, velocityBoundaries, pressureBoundaries, std::move(initialVelocity),
                   std::move(initialPressure));
}

}  // namespace cfdb_shim
