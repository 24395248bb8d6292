// warmstart.cu -- device side of the learned warm start (no counterpart in the reference).
//
// Between two physical steps the network sees each case's fields on a canvas and predicts the
// change of the per-step increment, relative to the size of that increment.  With inc the
// increment over the step just completed and s[f] its RMS over the case (per field), the
// candidate starts of the next pseudo-time loop are
//   plain:    the stale pseudo-iterate the reference starts from (main.f90:145-149 skipped),
//   extrap:   x + inc, or with order 2 x + (2 inc - incp) (incp: the increment one step
//             earlier; the quadratic through the starts of the last three steps),
//   learned:  x + a[f] * inc + s[f] * scale[f] * Y     (Y = network output, a[f] = scale[8+f],
//             normally 1; a field whose increment is not predictable can take 0 or 1 there),
// each with the boundary passes applied.  The initial residual -- the dtau-scaled max-norm of
// the U and V stage-1 updates and of the pressure update, i.e. the quantities whose maximum is
// the reference's `error` (main.f90:138-142, equations.f90:298,600,662) -- is evaluated for
// every candidate (built in the stage scratch S[0..2]) and the smallest one is committed.  The
// pseudo-time loop then iterates to the same tolerance from whichever start was kept.
//
// Compiled with -fmad=false: the residual evaluation reuses the exact point functions.
#include <cuda_runtime.h>

#include "acs_dev.cuh"
#include "points_exact.cuh"
#include "bc_exact.cuh"
#include "warmstart.h"

namespace acs {
using namespace exact;

namespace {

constexpr int WT = 256;

// running max that keeps a NaN once it has been seen (a broken start is never kept)
__device__ inline void acc_max(double& a, double v) { a = (v != v || v > a) ? v : a; }

__device__ inline bool in_field(const CaseDev& d, int f, int i, int j) {
  const int w = f == 0 ? d.nx + 1 : d.nx, h = f == 1 ? d.ny + 1 : d.ny;
  return i >= 1 && i <= w && j >= 1 && j <= h;
}

// the physical-step fields; for p the buffer the momentum routines read (the latest pressure)
__device__ inline double* phys_field(const CaseDev& d, const CaseCtl& k, int f) {
  switch (f) {
    case 0: return d.U[k.ru[R_PHYS]];
    case 1: return d.V[k.rv[R_PHYS]];
    case 2: return d.P[k.rp_read];
    case 3: return d.T[k.rt[R_PHYS]];
    default: return d.C[k.rc[R_PHYS]];
  }
}

// per node: incp = inc, inc = x - prev, prev = x; per case and field the sum of inc^2 into ss[c*8 + f]
__global__ void __launch_bounds__(WT) k_ws_history(const CaseDev* __restrict__ dc, const CaseCtl* __restrict__ dk,
                                                   const WsCase* __restrict__ dw, int H, int W, int has_prev,
                                                   double* __restrict__ ss) {
  __shared__ double acc[WS_FIELDS];
  const int c = blockIdx.y;
  const int q = blockIdx.x * WT + threadIdx.x;
  if (threadIdx.x < WS_FIELDS) acc[threadIdx.x] = 0.0;
  __syncthreads();
  double sq[WS_FIELDS] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (q < H * W) {
    const CaseDev& d = dc[c];
    const CaseCtl& k = dk[c];
    const WsCase& w = dw[c];
    const int i = q % W + 1, j = q / W + 1;
    if (i <= d.nx + 1 && j <= d.ny + 1) {
      const long long n = lin(i, j, d.pitch);
#pragma unroll
      for (int f = 0; f < WS_FIELDS; ++f)
        if (in_field(d, f, i, j)) {
          const double a = phys_field(d, k, f)[n];
          const double di = has_prev ? a - w.prev[f][n] : 0.0;
          w.incp[f][n] = w.inc[f][n];
          w.inc[f][n] = di;
          w.prev[f][n] = a;
          sq[f] = di * di;
        }
    }
  }
#pragma unroll
  for (int f = 0; f < WS_FIELDS; ++f) {
    double v = sq[f];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&acc[f], v);
  }
  __syncthreads();
  if (threadIdx.x < WS_FIELDS && acc[threadIdx.x] != 0.0) atomicAdd(&ss[c * WS_OUT + threadIdx.x], acc[threadIdx.x]);
}

// s[c][f] = RMS of inc_f over the field's nodes (1 where it is 0 or not finite)
__global__ void k_ws_scale(const CaseDev* __restrict__ dc, const double* __restrict__ ss, double* __restrict__ sc,
                           float* __restrict__ out) {
  const int c = blockIdx.x, f = threadIdx.x;
  if (f >= WS_OUT) return;
  const CaseDev& d = dc[c];
  double v = 1.0;
  if (f < WS_FIELDS) {
    const double cnt = f == 0 ? (double)(d.nx + 1) * d.ny : f == 1 ? (double)d.nx * (d.ny + 1) : (double)d.nx * d.ny;
    const double r = sqrt(ss[c * WS_OUT + f] / cnt);
    if (r > 0.0 && r < 1e300) v = r;
  }
  sc[c * WS_OUT + f] = v;
  if (out) out[c * WS_OUT + f] = (float)v;
}

__global__ void __launch_bounds__(WT) k_ws_features(const CaseDev* __restrict__ dc, const CaseCtl* __restrict__ dk,
                                                    const WsCase* __restrict__ dw, int H, int W,
                                                    const double* __restrict__ sc, float* __restrict__ X) {
  const int c = blockIdx.y;
  const int q = blockIdx.x * WT + threadIdx.x;
  if (q >= H * W) return;
  const CaseDev& d = dc[c];
  const CaseCtl& k = dk[c];
  const WsCase& w = dw[c];
  const int x = q % W, y = q / W, i = x + 1, j = y + 1;
  float* o = X + ((long long)c * H * W + q) * WS_IN;
  const long long n = (i <= d.nx + 1 && j <= d.ny + 1) ? lin(i, j, d.pitch) : 0;
#pragma unroll
  for (int f = 0; f < WS_FIELDS; ++f) {
    float v = 0.f, dv = 0.f;
    if (in_field(d, f, i, j)) {
      v = (float)phys_field(d, k, f)[n];
      dv = (float)(w.inc[f][n] / sc[c * WS_OUT + f]);
    }
    o[f] = v;
    o[6 + f] = dv;
  }
  o[5] = (i <= d.nx && j <= d.ny) ? (float)d.liga[n] : 0.f;
}

__global__ void __launch_bounds__(WT) k_ws_target(const CaseDev* __restrict__ dc, const CaseCtl* __restrict__ dk,
                                                  const WsCase* __restrict__ dw, int H, int W,
                                                  const double* __restrict__ sc, float* __restrict__ T,
                                                  float* __restrict__ Wt) {
  const int c = blockIdx.y;
  const int q = blockIdx.x * WT + threadIdx.x;
  if (q >= H * W) return;
  const CaseDev& d = dc[c];
  const CaseCtl& k = dk[c];
  const WsCase& w = dw[c];
  const int x = q % W, y = q / W, i = x + 1, j = y + 1;
  const long long o = ((long long)c * H * W + q) * WS_OUT;
  const long long n = (i <= d.nx + 1 && j <= d.ny + 1) ? lin(i, j, d.pitch) : 0;
#pragma unroll
  for (int f = 0; f < WS_OUT; ++f) {
    float t = 0.f, m = 0.f;
    if (f < WS_FIELDS && in_field(d, f, i, j)) {
      t = (float)(((phys_field(d, k, f)[n] - w.prev[f][n]) - w.inc[f][n]) / sc[c * WS_OUT + f]);
      m = 1.f;
    }
    T[o + f] = t;
    Wt[o + f] = m;
  }
}

// extrapolated (yy null): x + inc (order 1) or x + (2 inc - incp) (order 2);
// learned: x + scale[8+f] * inc + s[f] * scale[f] * Y
__device__ inline double start_value(const CaseDev& d, const CaseCtl& k, const WsCase& w, const double* sc,
                                     const float* yy, const float* scale, int order, int c, int f, long long n) {
  if (!yy) {
    if (order == 2) return phys_field(d, k, f)[n] + (2.0 * w.inc[f][n] - w.incp[f][n]);
    return phys_field(d, k, f)[n] + w.inc[f][n];
  }
  const double corr = sc[c * WS_OUT + f] * (double)scale[f] * (double)yy[f];
  return phys_field(d, k, f)[n] + (double)scale[WS_OUT + f] * w.inc[f][n] + corr;
}

// u, v, p of a candidate start into S[0], S[1], S[2]
__global__ void __launch_bounds__(WT) k_ws_candidate(const CaseDev* __restrict__ dc, const CaseCtl* __restrict__ dk,
                                                     const WsCase* __restrict__ dw, int H, int W,
                                                     const double* __restrict__ sc, const float* __restrict__ Y,
                                                     int ldy, const float* __restrict__ scale, int order) {
  const int c = blockIdx.y;
  const int q = blockIdx.x * WT + threadIdx.x;
  if (q >= H * W) return;
  const CaseDev& d = dc[c];
  const CaseCtl& k = dk[c];
  const int i = q % W + 1, j = q / W + 1;
  if (i > d.nx + 1 || j > d.ny + 1) return;
  const long long n = lin(i, j, d.pitch);
  const float* yy = Y ? Y + ((long long)c * H * W + q) * ldy : nullptr;
#pragma unroll
  for (int f = 0; f < 3; ++f)
    if (in_field(d, f, i, j)) d.S[f][n] = start_value(d, k, dw[c], sc, yy, scale, order, c, f, n);
}

__global__ void k_ws_bc_candidate(const CaseDev* __restrict__ dc) {
  const CaseDev& d = dc[blockIdx.x];
  bc_uv_block(d, d.S[0], d.S[1]);
  __syncthreads();
  bc_cell_block(d, d.S[2], true, 0.0);
}

// initial residuals: of the plain start into res[3c + slot_plain] (slot_plain >= 0) and of the
// candidate in S[0..2] into res[3c + slot_cand]
__global__ void __launch_bounds__(WT) k_ws_probe(const CaseDev* __restrict__ dc, const CaseCtl* __restrict__ dk, int H,
                                                 int W, int slot_plain, int slot_cand,
                                                 unsigned long long* __restrict__ res) {
  const int c = blockIdx.y;
  const int q = blockIdx.x * WT + threadIdx.x;
  const CaseDev& d = dc[c];
  const CaseCtl& k = dk[c];
  const G g(d);
  double a[2] = {0.0, 0.0};
  if (q < H * W) {
    const int i = q % W + 1, j = q / W + 1;
    const double* um = d.U[k.ru[R_PHYS]];
    const double* vm = d.V[k.rv[R_PHYS]];
    const double* T = d.T[k.rt[R_PHYS]];
    for (int s = slot_plain >= 0 ? 0 : 1; s < 2; ++s) {
      const double* ut = s ? d.S[0] : d.U[k.ru[R_TAU]];
      const double* vt = s ? d.S[1] : d.V[k.rv[R_TAU]];
      const double* pn = s ? d.S[2] : d.P[k.rp_read];
      if (i >= 3 && i <= d.nx - 1 && j >= 2 && j <= d.ny - 1) {
        const bool quick = d.scheme == 0 && j >= 3 && j <= d.ny - 2;
        const double RU = quick ? resu_quick(d, g, ut, vt, pn, i, j) : resu_upwind(d, g, ut, vt, pn, i, j);
        const long long o = g.o(i, j);
        acc_max(a[s], fabs(((um[o] - ut[o]) + RU * d.dt) * d.dtau));
      }
      if (i >= 2 && i <= d.nx - 1 && j >= 3 && j <= d.ny - 1) {
        const bool quick = d.scheme == 0 && i >= 3 && i <= d.nx - 2;
        const double RV = quick ? resv_quick(d, g, ut, vt, pn, T, i, j) : resv_upwind(d, g, ut, vt, pn, T, i, j);
        const long long o = g.o(i, j);
        acc_max(a[s], fabs(((vm[o] - vt[o]) + RV * d.dt) * d.dtau));
      }
      if (i >= 2 && i <= d.nx - 1 && j >= 2 && j <= d.ny - 1) {
        const double Aew = g.ym[j + 1] - g.ym[j], Ans = g.xm[i + 1] - g.xm[i];
        const double dudx = ut[g.o(i + 1, j)] * Aew - ut[g.o(i, j)] * Aew;
        const double dvdy = vt[g.o(i, j + 1)] * Ans - vt[g.o(i, j)] * Ans;
        double RP = -(dudx + dvdy);
        if (d.continuity == 1) RP = RP / ((g.ym[j + 1] - g.ym[j]) * (g.xm[i + 1] - g.xm[i]));
        acc_max(a[s], fabs(d.dtau * RP * d.beta));
      }
    }
  }
  if (slot_plain >= 0) {
    block_max_to(&res[3 * c + slot_plain], a[0]);
    __syncthreads();
  }
  block_max_to(&res[3 * c + slot_cand], a[1]);
}

// 0 = plain, 1 = extrapolated, 2 = learned (residual bits compare like the non-negative values,
// NaN above everything; ties keep the earlier candidate)
__device__ inline int pick(int policy, bool have_y, const unsigned long long* r) {
  if (policy == 2) return 0;
  if (policy == 1) return have_y ? 2 : 1;
  int best = 0;
  if (r[1] < r[best]) best = 1;
  if (have_y && r[2] < r[best]) best = 2;
  return best;
}

__global__ void __launch_bounds__(WT) k_ws_commit(const CaseDev* __restrict__ dc, CaseCtl* __restrict__ dk,
                                                  const WsCase* __restrict__ dw, int H, int W,
                                                  const double* __restrict__ sc, const float* __restrict__ Y, int ldy,
                                                  const float* __restrict__ scale, int policy, int order,
                                                  const unsigned long long* __restrict__ res, int* __restrict__ choice) {
  const int c = blockIdx.y;
  const int q = blockIdx.x * WT + threadIdx.x;
  const int which = pick(policy, Y != nullptr, res + 3 * c);
  const CaseDev& d = dc[c];
  const CaseCtl k = dk[c];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    choice[c] = which;
    if (which) dk[c].tau_dirty = 1;
  }
  if (!which || q >= H * W) return;
  const int i = q % W + 1, j = q / W + 1;
  if (i > d.nx + 1 || j > d.ny + 1) return;
  const long long n = lin(i, j, d.pitch);
  const float* yy = which == 2 ? Y + ((long long)c * H * W + q) * ldy : nullptr;
  const WsCase& w = dw[c];
  if (in_field(d, 0, i, j)) d.U[k.ru[R_TAU]][n] = start_value(d, k, w, sc, yy, scale, order, c, 0, n);
  if (in_field(d, 1, i, j)) d.V[k.rv[R_TAU]][n] = start_value(d, k, w, sc, yy, scale, order, c, 1, n);
  if (in_field(d, 2, i, j)) {
    const double pv = start_value(d, k, w, sc, yy, scale, order, c, 2, n);
    if (k.scalars) {
      d.T[k.rt[R_TAU]][n] = start_value(d, k, w, sc, yy, scale, order, c, 3, n);
      d.C[k.rc[R_TAU]][n] = start_value(d, k, w, sc, yy, scale, order, c, 4, n);
    }
    // p and pn both hold the start (the reads above went through P[rp_read] first)
    d.P[0][n] = pv;
    d.P[1][n] = pv;
  }
}

__global__ void k_ws_bc_commit(const CaseDev* __restrict__ dc, const CaseCtl* __restrict__ dk,
                               const int* __restrict__ choice) {
  const int c = blockIdx.x;
  const CaseDev& d = dc[c];
  const CaseCtl& k = dk[c];
  if (!choice[c]) return;
  bc_uv_block(d, d.U[k.ru[R_TAU]], d.V[k.rv[R_TAU]]);
  __syncthreads();
  bc_cell_block(d, d.P[0], true, 0.0);
  __syncthreads();
  bc_cell_block(d, d.P[1], true, 0.0);
  if (!k.scalars) return;
  __syncthreads();
  bc_cell_block(d, d.T[k.rt[R_TAU]], false, d.T_in);
  __syncthreads();
  bc_cell_block(d, d.C[k.rc[R_TAU]], false, d.C_in);
}

inline dim3 canvas_grid(int n, int H, int W) { return dim3((unsigned)((H * W + WT - 1) / WT), (unsigned)n); }

}  // namespace

void launch_ws_features(const CaseDev* dc, const CaseCtl* dk, const WsCase* dw, int n, int H, int W, int has_prev,
                        double* ss, double* sc, float* X, float* scale_out, cudaStream_t s) {
  cudaMemsetAsync(ss, 0, sizeof(double) * WS_OUT * n, s);
  const dim3 g = canvas_grid(n, H, W);
  k_ws_history<<<g, WT, 0, s>>>(dc, dk, dw, H, W, has_prev, ss);
  k_ws_scale<<<n, 32, 0, s>>>(dc, ss, sc, scale_out);
  k_ws_features<<<g, WT, 0, s>>>(dc, dk, dw, H, W, sc, X);
}

void launch_ws_target(const CaseDev* dc, const CaseCtl* dk, const WsCase* dw, int n, int H, int W, const double* sc,
                      float* T, float* Wt, cudaStream_t s) {
  k_ws_target<<<canvas_grid(n, H, W), WT, 0, s>>>(dc, dk, dw, H, W, sc, T, Wt);
}

void launch_ws_start(const CaseDev* dc, CaseCtl* dk, const WsCase* dw, int n, int H, int W, const double* sc,
                     const float* Y, int ldy, const float* scale, int policy, int order, unsigned long long* res,
                     int* choice, cudaStream_t s) {
  cudaMemsetAsync(res, 0, sizeof(unsigned long long) * 3 * n, s);
  const dim3 g = canvas_grid(n, H, W);
  k_ws_candidate<<<g, WT, 0, s>>>(dc, dk, dw, H, W, sc, nullptr, ldy, scale, order);
  k_ws_bc_candidate<<<n, 128, 0, s>>>(dc);
  k_ws_probe<<<g, WT, 0, s>>>(dc, dk, H, W, 0, 1, res);
  if (Y) {
    k_ws_candidate<<<g, WT, 0, s>>>(dc, dk, dw, H, W, sc, Y, ldy, scale, order);
    k_ws_bc_candidate<<<n, 128, 0, s>>>(dc);
    k_ws_probe<<<g, WT, 0, s>>>(dc, dk, H, W, -1, 2, res);
  }
  k_ws_commit<<<g, WT, 0, s>>>(dc, dk, dw, H, W, sc, Y, ldy, scale, policy, order, res, choice);
  k_ws_bc_commit<<<n, 128, 0, s>>>(dc, dk, choice);
}

}  // namespace acs
