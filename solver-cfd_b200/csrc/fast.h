// fast.h -- interface of the fused FAST-arithmetic kernels (kernels_fast.cu).
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <vector>
#include "../../include/acs.h"
#include "acs_dev.cuh"

namespace acs {

struct FastPlan;

int fast_create(std::vector<CaseDev>& cases, const acs_grid* grids, const acs_params* params, FastPlan** out);
void fast_destroy(FastPlan* f);
void fast_u(FastPlan* f, const CaseDev* dc, CaseCtl* dk, const Tile* tiles, int ntiles, int ncases, cudaStream_t s);
void fast_v(FastPlan* f, const CaseDev* dc, CaseCtl* dk, const Tile* tiles, int ntiles, int ncases, cudaStream_t s);
void fast_p(FastPlan* f, const CaseDev* dc, CaseCtl* dk, const Tile* tiles, int ntiles, int ncases, cudaStream_t s);
void fast_s(FastPlan* f, bool is_c, const CaseDev* dc, CaseCtl* dk, const Tile* tiles, int ntiles, int ncases, cudaStream_t s);
void fast_timed(FastPlan* f, int kernel, const CaseDev* dc, CaseCtl* dk, const Tile* tiles, int ntiles, int ncases, cudaStream_t s);
int fast_u_launches(const FastPlan* f);
int fast_v_launches(const FastPlan* f);
int fast_p_launches(const FastPlan* f);
int fast_s_launches(const FastPlan* f);

int fail(int code, const std::string& msg);

}  // namespace acs
