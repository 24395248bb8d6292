// kernels_fast.cu -- the graph engine's per-stage kernels with the FAST arithmetic.
//
// Same launch structure as kernels_exact.cu (one thread per node, 32 x 8 tiles over every active
// case, one launch per Runge-Kutta stage, the boundary passes of kernels_exact.cu in between), with
// the per-node residuals of points_fast.cuh.  A large case then spreads each stage over the whole
// GPU instead of one thread-block cluster.  No array a launch reads is written by the same launch,
// so loads go through the read-only path.
//
// Reference (OpenMp_Multicore/): solve_U equations.f90:244-301, solve_V :546-603, solve_P
// :607-665, solve_Z :669-719, solve_C :769-819.
#include <cuda_runtime.h>
#include "acs_dev.cuh"
#include "kernels.h"
#include "points_fast.cuh"

namespace acs {
namespace {

using PT = PtFastT<LdRO>;

template <int STAGE>
__global__ void __launch_bounds__(256) k_u_stage_fast(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                      const Tile* __restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  if (!ctl[t.c].active) return;
  const CaseDev& d = cs[t.c];
  const CaseCtl& k = ctl[t.c];
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  const double* uin = STAGE == 1 ? d.U[k.ru[R_TAU]] : d.S[STAGE - 2];
  double* uout = STAGE == 3 ? d.U[k.ru[R_NTAU]] : d.S[STAGE - 1];
  const double* utau = d.U[k.ru[R_TAU]];
  const double* um = d.U[k.ru[R_PHYS]];
  const double* vt = d.V[k.rv[R_TAU]];
  const double* pn = d.P[k.rp_read];
  double a = 0.0;
  if (i >= 3 && i <= d.nx - 1 && j >= 2 && j <= d.ny - 1) {
    const double RU = PT::ru(d, uin, vt, pn, i, j);
    const long long q = lin(i, j, d.pitch);
    const double r = ((__ldg(um + q) - __ldg(utau + q)) + RU * d.dt) * d.dtau;
    if (STAGE == 1) uout[q] = __ldg(utau + q) + r;
    if (STAGE == 2) uout[q] = 0.75 * __ldg(utau + q) + 0.25 * (__ldg(uin + q) + r);
    if (STAGE == 3) uout[q] = 1.0 / 3.0 * __ldg(utau + q) + 2.0 / 3.0 * (__ldg(uin + q) + r);
    a = fabs(r);
  }
  if (STAGE == 3) block_max_to(&ctl[t.c].res_u, a);
}

template <int STAGE>
__global__ void __launch_bounds__(256) k_v_stage_fast(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                      const Tile* __restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  if (!ctl[t.c].active) return;
  const CaseDev& d = cs[t.c];
  const CaseCtl& k = ctl[t.c];
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  const double* vin = STAGE == 1 ? d.V[k.rv[R_TAU]] : d.S[STAGE - 2];
  double* vout = STAGE == 3 ? d.V[k.rv[R_NTAU]] : d.S[STAGE - 1];
  const double* vtau = d.V[k.rv[R_TAU]];
  const double* vm = d.V[k.rv[R_PHYS]];
  const double* ut = d.U[k.ru[R_TAU]];
  const double* pn = d.P[k.rp_read];
  const double* T = d.T[k.rt[R_PHYS]];
  double a = 0.0;
  if (i >= 2 && i <= d.nx - 1 && j >= 3 && j <= d.ny - 1) {
    const double RV = PT::rv(d, ut, vin, pn, T, i, j);
    const long long q = lin(i, j, d.pitch);
    const double r = ((__ldg(vm + q) - __ldg(vtau + q)) + RV * d.dt) * d.dtau;
    if (STAGE == 1) vout[q] = __ldg(vtau + q) + r;
    if (STAGE == 2) vout[q] = 0.75 * __ldg(vtau + q) + 0.25 * (__ldg(vin + q) + r);
    if (STAGE == 3) vout[q] = 1.0 / 3.0 * __ldg(vtau + q) + 2.0 / 3.0 * (__ldg(vin + q) + r);
    a = fabs(r);
  }
  if (STAGE == 3) block_max_to(&ctl[t.c].res_v, a);
}

__global__ void __launch_bounds__(256) k_p_fast(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                const Tile* __restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  if (!ctl[t.c].active) return;
  const CaseDev& d = cs[t.c];
  const CaseCtl& k = ctl[t.c];
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  double a = 0.0;
  if (i >= 2 && i <= d.nx - 1 && j >= 2 && j <= d.ny - 1) {
    double r;
    d.P[k.rp[1]][lin(i, j, d.pitch)] = PT::p_update(d, d.P[k.rp[0]], d.U[k.ru[R_NTAU]], d.V[k.rv[R_NTAU]], i, j, &r);
    a = fabs(r);
  }
  block_max_to(&ctl[t.c].res_p, a);
}

template <bool IS_C, int STAGE>
__global__ void __launch_bounds__(256) k_s_stage_fast(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                      const Tile* __restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  if (!ctl[t.c].active || !ctl[t.c].scalars) return;
  const CaseDev& d = cs[t.c];
  const CaseCtl& k = ctl[t.c];
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  double* const* F = IS_C ? d.C : d.T;
  const int* rr = IS_C ? k.rc : k.rt;
  const double* zin = STAGE == 1 ? F[rr[R_TAU]] : d.S[STAGE - 2];
  double* zout = STAGE == 3 ? F[rr[R_NTAU]] : d.S[STAGE - 1];
  const double* ztau = F[rr[R_TAU]];
  const double* z = F[rr[R_PHYS]];
  if (i >= 2 && i <= d.nx - 1 && j >= 2 && j <= d.ny - 1) {
    const double R = PT::template rs<IS_C>(d, d.U[k.ru[R_NTAU]], d.V[k.rv[R_NTAU]], zin, i, j);
    const long long q = lin(i, j, d.pitch);
    const double r = ((__ldg(z + q) - __ldg(ztau + q)) + R * d.dt) * d.dtau;
    if (STAGE == 1) zout[q] = __ldg(ztau + q) + r;
    if (STAGE == 2) zout[q] = 0.75 * __ldg(ztau + q) + 0.25 * (__ldg(zin + q) + r);
    if (STAGE == 3) zout[q] = 1.0 / 3.0 * __ldg(ztau + q) + 2.0 / 3.0 * (__ldg(zin + q) + r);
  }
}

template <int S>
void go_u(const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  k_u_stage_fast<S><<<n, dim3(TILE_X, TILE_Y), 0, s>>>(c, k, t);
}
template <int S>
void go_v(const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  k_v_stage_fast<S><<<n, dim3(TILE_X, TILE_Y), 0, s>>>(c, k, t);
}
template <bool IC, int S>
void go_s(const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  k_s_stage_fast<IC, S><<<n, dim3(TILE_X, TILE_Y), 0, s>>>(c, k, t);
}

}  // namespace

void launch_u_stage_fast(int stage, const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  if (stage == 1) go_u<1>(c, k, t, n, s);
  else if (stage == 2) go_u<2>(c, k, t, n, s);
  else go_u<3>(c, k, t, n, s);
}
void launch_v_stage_fast(int stage, const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  if (stage == 1) go_v<1>(c, k, t, n, s);
  else if (stage == 2) go_v<2>(c, k, t, n, s);
  else go_v<3>(c, k, t, n, s);
}
void launch_s_stage_fast(bool is_c, int stage, const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  if (is_c) {
    if (stage == 1) go_s<true, 1>(c, k, t, n, s);
    else if (stage == 2) go_s<true, 2>(c, k, t, n, s);
    else go_s<true, 3>(c, k, t, n, s);
  } else {
    if (stage == 1) go_s<false, 1>(c, k, t, n, s);
    else if (stage == 2) go_s<false, 2>(c, k, t, n, s);
    else go_s<false, 3>(c, k, t, n, s);
  }
}
void launch_p_fast(const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  k_p_fast<<<n, dim3(TILE_X, TILE_Y), 0, s>>>(c, k, t);
}

}  // namespace acs
