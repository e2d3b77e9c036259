// Internal entry points of the p' operator shared with the SIMPLE driver.
#pragma once

#include "cfdb.h"

namespace cfdb {
cfdb_status poperator_bind_faces(cfdb_context* ctx, cfdb_poperator* op, const double* D, bool fp32);
}
