// kernels.h -- kernel declarations shared between the kernel sources and the host launcher.
#pragma once
#include <cuda_runtime.h>
#include "acs_dev.cuh"

namespace acs {

// exact-arithmetic path (kernels_exact.cu); launchers so no kernel template crosses units.
// stage = 1..3; `is_c` selects solve_C (true) or solve_Z (false).
void launch_u_stage_exact(int stage, const CaseDev*, CaseCtl*, const Tile*, int ntiles, cudaStream_t);
void launch_v_stage_exact(int stage, const CaseDev*, CaseCtl*, const Tile*, int ntiles, cudaStream_t);
void launch_s_stage_exact(bool is_c, int stage, const CaseDev*, CaseCtl*, const Tile*, int ntiles, cudaStream_t);
void launch_p_exact(const CaseDev*, CaseCtl*, const Tile*, int ntiles, cudaStream_t);
// FAST-arithmetic per-stage kernels (kernels_fast.cu), same launch structure
void launch_u_stage_fast(int stage, const CaseDev*, CaseCtl*, const Tile*, int ntiles, cudaStream_t);
void launch_v_stage_fast(int stage, const CaseDev*, CaseCtl*, const Tile*, int ntiles, cudaStream_t);
void launch_s_stage_fast(bool is_c, int stage, const CaseDev*, CaseCtl*, const Tile*, int ntiles, cudaStream_t);
void launch_p_fast(const CaseDev*, CaseCtl*, const Tile*, int ntiles, cudaStream_t);
// boundary passes, one block per case (see kernels_exact.cu for `which`)
void launch_bc_uv(const CaseDev*, const CaseCtl*, int ncases, int which, cudaStream_t);
void launch_bc_cell(const CaseDev*, const CaseCtl*, int ncases, int which, cudaStream_t);

// cell-centred u, v (comp_mean) and |U| of one case (output.cu)
cudaError_t launch_cell_fields(const double* um, const double* vm, int nx, int ny, int pitch, double* u, double* v,
                               double* mag, cudaStream_t s);

// loop control (control.cu)
__global__ void k_control(const CaseDev*, CaseCtl*, int* iters, double* err, int* n_active);
__global__ void k_loop_cond(int* n_active, long long* iter_count, long long max_iters,
                            cudaGraphConditionalHandle handle);
__global__ void k_loop_flag(int* n_active, long long* iter_count, int* host_flag);

}  // namespace acs
