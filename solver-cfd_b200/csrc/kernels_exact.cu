// kernels_exact.cu -- FP64 kernels that reproduce the reference's rounding bit for bit.
//
// Built with -fmad=false: every product and sum is rounded separately and each expression keeps
// the Fortran evaluation order (left to right, `x**2.d0` = x*x, `x**0.5d0` = sqrt(x)), so the
// results are bit-identical to the reference arithmetic compiled without fused multiply-add.
// One thread per node, one launch per Runge-Kutta stage; boundary passes are separate
// one-block-per-case launches.  Every launch covers all active cases of a batch through a tile
// table; inactive cases (converged or failed) return at once.
//
// Reference (OpenMp_Multicore/): RESU equations.f90:2-116 (+ upwind_Ui/Uj :120-240),
// solve_U :244-301, RESV :305-420 (+ upwind_Vi/Vj :423-542), solve_V :546-603, solve_P :607-665,
// solve_Z :669-719, RESZ :723-765, solve_C :769-819, RESC :823-867, boundary.f90:1-159,
// main.f90:116-186 (control).
#include <cuda_runtime.h>
#include "acs_dev.cuh"
#include "kernels.h"

#include "points_exact.cuh"
#include "bc_exact.cuh"

namespace acs {
using namespace exact;

// ---- solve_U stage s (s = 1,2,3; equations.f90:259-298) ---------------------------------------
template <int STAGE>
__global__ void __launch_bounds__(256) k_u_stage_exact(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                       const Tile* __restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  if (!ctl[t.c].active) return;
  const CaseDev& d = cs[t.c];
  const CaseCtl& k = ctl[t.c];
  const G g(d);
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  const double* uin = STAGE == 1 ? d.U[k.ru[R_TAU]] : d.S[STAGE - 2];
  double* uout = STAGE == 3 ? d.U[k.ru[R_NTAU]] : d.S[STAGE - 1];
  const double* utau = d.U[k.ru[R_TAU]];
  const double* um = d.U[k.ru[R_PHYS]];
  const double* vt = d.V[k.rv[R_TAU]];
  const double* pn = d.P[k.rp_read];
  double a = 0.0;
  if (i >= 3 && i <= d.nx - 1 && j >= 2 && j <= d.ny - 1) {
    const bool quick = d.scheme == 0 && j >= 3 && j <= d.ny - 2;
    const double RU = quick ? resu_quick(d, g, uin, vt, pn, i, j) : resu_upwind(d, g, uin, vt, pn, i, j);
    const long long q = g.o(i, j);
    const double r = ((um[q] - utau[q]) + RU * d.dt) * d.dtau;
    if (STAGE == 1) uout[q] = utau[q] + r;
    if (STAGE == 2) uout[q] = 0.75 * utau[q] + 0.25 * (uin[q] + r);
    if (STAGE == 3) uout[q] = 1.0 / 3.0 * utau[q] + 2.0 / 3.0 * (uin[q] + r);
    a = fabs(r);
  }
  if (STAGE == 3) block_max_to(&ctl[t.c].res_u, a);
}

// ---- solve_V stage s (equations.f90:561-600) --------------------------------------------------
template <int STAGE>
__global__ void __launch_bounds__(256) k_v_stage_exact(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                       const Tile* __restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  if (!ctl[t.c].active) return;
  const CaseDev& d = cs[t.c];
  const CaseCtl& k = ctl[t.c];
  const G g(d);
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
    const bool quick = d.scheme == 0 && i >= 3 && i <= d.nx - 2;
    const double RV = quick ? resv_quick(d, g, ut, vin, pn, T, i, j) : resv_upwind(d, g, ut, vin, pn, T, i, j);
    const long long q = g.o(i, j);
    const double r = ((vm[q] - vtau[q]) + RV * d.dt) * d.dtau;
    if (STAGE == 1) vout[q] = (vtau[q] + r);
    if (STAGE == 2) vout[q] = (0.75 * vtau[q] + 0.25 * (vin[q] + r));
    if (STAGE == 3) vout[q] = 1.0 / 3.0 * vtau[q] + 2.0 / 3.0 * (vin[q] + r);
    a = fabs(r);
  }
  if (STAGE == 3) block_max_to(&ctl[t.c].res_v, a);
}

// ---- solve_P: the three stages share RP, so they fuse pointwise (equations.f90:620-662) -----
__global__ void __launch_bounds__(256) k_p_exact(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                 const Tile* __restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  if (!ctl[t.c].active) return;
  const CaseDev& d = cs[t.c];
  const CaseCtl& k = ctl[t.c];
  const G g(d);
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  const double* p = d.P[k.rp[0]];
  double* pn = d.P[k.rp[1]];
  const double* un = d.U[k.ru[R_NTAU]];
  const double* vn = d.V[k.rv[R_NTAU]];
  double a = 0.0;
  if (i >= 2 && i <= d.nx - 1 && j >= 2 && j <= d.ny - 1) {
    const double Aew = g.ym[j + 1] - g.ym[j], Ans = g.xm[i + 1] - g.xm[i];
    const double dudx = un[g.o(i + 1, j)] * Aew - un[g.o(i, j)] * Aew;
    const double dvdy = vn[g.o(i, j + 1)] * Ans - vn[g.o(i, j)] * Ans;
    double RP = -(dudx + dvdy);
    if (d.continuity == 1) RP = RP / ((g.ym[j + 1] - g.ym[j]) * (g.xm[i + 1] - g.xm[i]));
    const long long q = g.o(i, j);
    const double p0 = p[q];
    const double pi1 = p0 + d.dtau * RP * d.beta;
    const double pi2 = 0.75 * p0 + 0.25 * (pi1 + d.dtau * RP * d.beta);
    const double r = d.dtau * RP * d.beta;
    pn[q] = 1.0 / 3.0 * p0 + 2.0 / 3.0 * (pi2 + r);
    a = fabs(r);
  }
  block_max_to(&ctl[t.c].res_p, a);
}

// ---- solve_Z / solve_C stage s (equations.f90:679-716, 779-816) -------------------------------
template <bool IS_C, int STAGE>
__global__ void __launch_bounds__(256) k_s_stage_exact(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                       const Tile* __restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  if (!ctl[t.c].active || !ctl[t.c].scalars) return;
  const CaseDev& d = cs[t.c];
  const CaseCtl& k = ctl[t.c];
  const G g(d);
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  double* const* F = IS_C ? d.C : d.T;
  const int* rr = IS_C ? k.rc : k.rt;
  const double* zin = STAGE == 1 ? F[rr[R_TAU]] : d.S[STAGE - 2];
  double* zout = STAGE == 3 ? F[rr[R_NTAU]] : d.S[STAGE - 1];
  const double* ztau = F[rr[R_TAU]];
  const double* z = F[rr[R_PHYS]];
  const double* un = d.U[k.ru[R_NTAU]];
  const double* vn = d.V[k.rv[R_NTAU]];
  if (i >= 2 && i <= d.nx - 1 && j >= 2 && j <= d.ny - 1) {
    const double R = res_scalar<IS_C>(d, g, un, vn, zin, i, j);
    const long long q = g.o(i, j);
    const double r = ((z[q] - ztau[q]) + R * d.dt) * d.dtau;
    if (STAGE == 1) zout[q] = ztau[q] + r;
    if (STAGE == 2) zout[q] = 0.75 * ztau[q] + 0.25 * (zin[q] + r);
    if (STAGE == 3) zout[q] = 1.0 / 3.0 * ztau[q] + 2.0 / 3.0 * (zin[q] + r);
  }
}

__global__ void k_bc_uv(const CaseDev* __restrict__ cs, const CaseCtl* __restrict__ ctl, int which) {
  const int c = blockIdx.x;
  if (!ctl[c].active) return;
  const CaseDev& d = cs[c];
  const CaseCtl& k = ctl[c];
  double *um, *vm;
  if (which < 3) {
    um = which == 2 ? d.U[k.ru[R_NTAU]] : d.S[which];
    vm = d.V[k.rv[R_TAU]];
  } else {
    um = d.U[k.ru[R_TAU]];
    vm = which == 5 ? d.V[k.rv[R_NTAU]] : d.S[which - 3];
  }
  bc_uv_block(d, um, vm);
}

// which: 0 = p (P[pn]); 1..3 = T written by stage (S0, S1, T[ntau]); 4..6 = C likewise.
__global__ void k_bc_cell(const CaseDev* __restrict__ cs, const CaseCtl* __restrict__ ctl, int which) {
  const int c = blockIdx.x;
  if (!ctl[c].active) return;
  const CaseDev& d = cs[c];
  const CaseCtl& k = ctl[c];
  if (which == 0) { bc_cell_block(d, d.P[k.rp[1]], true, 0.0); return; }
  if (!k.scalars) return;
  const bool isC = which >= 4;
  const int s = isC ? which - 4 : which - 1;
  double* z = s == 2 ? (isC ? d.C[k.rc[R_NTAU]] : d.T[k.rt[R_NTAU]]) : d.S[s];
  bc_cell_block(d, z, false, isC ? d.C_in : d.T_in);
}

namespace {
template <int S>
void go_u(const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  k_u_stage_exact<S><<<n, dim3(TILE_X, TILE_Y), 0, s>>>(c, k, t);
}
template <int S>
void go_v(const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  k_v_stage_exact<S><<<n, dim3(TILE_X, TILE_Y), 0, s>>>(c, k, t);
}
template <bool IC, int S>
void go_s(const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  k_s_stage_exact<IC, S><<<n, dim3(TILE_X, TILE_Y), 0, s>>>(c, k, t);
}
}  // namespace

void launch_u_stage_exact(int stage, const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  if (stage == 1) go_u<1>(c, k, t, n, s);
  else if (stage == 2) go_u<2>(c, k, t, n, s);
  else go_u<3>(c, k, t, n, s);
}
void launch_v_stage_exact(int stage, const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  if (stage == 1) go_v<1>(c, k, t, n, s);
  else if (stage == 2) go_v<2>(c, k, t, n, s);
  else go_v<3>(c, k, t, n, s);
}
void launch_s_stage_exact(bool is_c, int stage, const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
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
void launch_p_exact(const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  k_p_exact<<<n, dim3(TILE_X, TILE_Y), 0, s>>>(c, k, t);
}
void launch_bc_uv(const CaseDev* c, const CaseCtl* k, int ncases, int which, cudaStream_t s) {
  k_bc_uv<<<ncases, 128, 0, s>>>(c, k, which);
}
void launch_bc_cell(const CaseDev* c, const CaseCtl* k, int ncases, int which, cudaStream_t s) {
  k_bc_cell<<<ncases, 128, 0, s>>>(c, k, which);
}

}  // namespace acs
