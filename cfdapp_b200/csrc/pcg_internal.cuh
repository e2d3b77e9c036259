// Internal entry points of the p' operator shared with the SIMPLE driver.
#pragma once

#include <cstdint>

#include "cfdb.h"

namespace cfdb {
struct LearnedSolver;
struct FineOperator;
cfdb_status poperator_bind_faces(cfdb_context* ctx, cfdb_poperator* op, const double* D, bool fp32);
// The operator as the learned preconditioner sees it, with its solver state
// (created on first use) and coefficient version.
void poperator_learned(cfdb_poperator* op, FineOperator* fo, LearnedSolver** solver,
                       uint64_t* version);
}
