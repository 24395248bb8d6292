// fast.h -- set-up of the FAST arithmetic tables (fast_tables.cu).
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <vector>
#include "../../include/acs.h"
#include "acs_dev.cuh"

namespace acs {

struct FastPlan;

// Builds the per-case metric tables on the device, fills CaseDev::mx/my/fc.  Needs the binary
// porous structure (epsilon1, liga_poros) in {(1,0), (phi,1)} of every case.
int fast_create(std::vector<CaseDev>& cases, const acs_grid* grids, const acs_params* params, FastPlan** out);
void fast_destroy(FastPlan* f);

int fail(int code, const std::string& msg);

}  // namespace acs
