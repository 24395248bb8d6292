// acs_dev.cuh -- device data model shared by the solver kernels and the host orchestration.
//
// Every case lives in its own set of pitched FP64 buffers.  A node (i,j) of the reference's
// 1-based Fortran arrays is stored at (i-1) + (j-1)*pitch for every field of the case, so um,
// vm and the cell fields share one index and one row pitch (pitch >= imax+1, a multiple of 4
// doubles so rows start on 32-byte boundaries).  The u family (um, um_tau, um_n_tau) rotates
// through three buffers by role instead of being copied (main.f90:145-157 copies); the same
// holds for v, T and C, and p/pn rotate through two.
#pragma once
#include <cstdint>

namespace acs {

enum Role { R_PHYS = 0, R_TAU = 1, R_NTAU = 2 };
enum CaseFlags {
  F_BUOY = 1,      // buoyancy term active (InvFr2 != 0 and T not identically 1)
  F_BART = 2,      // b_art != 0
  F_POROUS = 4,    // some cell has liga != 0
  F_BINARY = 8,    // epsilon1/liga take only (1,0) and (phi,1): fast path may use a byte mask
};

// per-case constants of the FAST arithmetic (CaseDev::fc)
enum FastConst { FC_IPHI = 0, FC_IRE, FC_IREDA, FC_CFS, FC_IRESC, FC_IPE, FC_DTB, FC_N };

struct CaseDev {
  int nx, ny, pitch, flags;
  int scheme, bc, solve_scalars, itc_max;
  int continuity, pad0;
  double Re, Pe, Sc, Da, Cf, g, InvFr2, v_in, T_in, C_in, b_art, beta, dt, dtau, eps;
  double phi;                         // porosity of flagged cells when F_BINARY
  const double *x, *y, *xm, *ym;      // 1-based: x[1..nx], y[1..ny], xm[1..nx+1], ym[1..ny+1]
  const double *epsf, *liga;          // pitched cell fields
  const uint8_t* mask;                // pitched porous mask (1 = porous), F_BINARY only
  // FAST arithmetic (engine_fast.cu): per-column / per-row metric tables of 4 doubles each,
  // indexed like x and y, and per-case constants
  const double* mx;
  const double* my;
  double fc[8];
  double* U[3];
  double* V[3];
  double* P[2];
  double* T[3];
  double* C[3];
  double* S[4];                       // stage scratch (largest field shape)
  double* S2[4];                      // stage scratch of T and C in the persistent engine, where
                                      // their stages overlap the next iteration's U and V stages
  long long n_elems;                  // pitch * (ny+1): doubles per buffer
};

// Mutable per-case control word (device).  Roles index into CaseDev::U/V/T/C/P.
struct CaseCtl {
  int ru[3], rv[3], rt[3], rc[3], rp[2];
  // Buffer holding the pressure that the momentum routines read (the reference's pn).  After a
  // non-exit iteration the reference copies p = pn and keeps reading pn, so the latest pressure
  // lives in both arrays; with swapped roles it lives only in the p-role buffer, rp[0].  After
  // an exit (no copy) it is the pn-role buffer, rp[1].
  int rp_read;
  // What the reference's n_tau arrays hold after the last control pass: 0 = their own buffer,
  // 1 = the same values as phys (after an exit, um = um_n_tau), 2 = the same values as tau
  // (after a non-exit iteration, um_tau = um_n_tau).  The loop never reads n_tau before
  // rewriting it, so this only matters when the state is read back.
  int ntau_alias;
  int itc;          // the reference's pseudo counter (main.f90:77,150,182)
  int step;         // physical steps completed in this run
  int n_steps;      // physical steps requested
  int k;            // pseudo-iterations in the current step
  int active;       // 1 while the case still iterates
  int status;       // acs_case_status
  int copy_phys;    // 1: copy tau -> phys at the next control pass (itc_max exit)
  int scalars;      // 1: the T and C kernels run for this case
  unsigned long long res_u, res_v, res_p;  // max |res| as IEEE bits (non-negative doubles)
  long long total_iters;
  // 1 while um_tau / vm_tau may not satisfy the boundary passes (after an upload): the next
  // iteration must run U and V in the reference's order with the full bcUV side effects
  int tau_dirty, pad1;
  unsigned long long slot[2][3];  // residual maxima of the persistent engine, by iteration parity
};

// Tile of the launch grid: case id and the 1-based origin of a 32 x 8 node block.
struct Tile { int c, i0, j0, pad; };

constexpr int TILE_X = 32;
constexpr int TILE_Y = 8;

__host__ __device__ inline long long lin(int i, int j, int pitch) {
  return (long long)(i - 1) + (long long)(j - 1) * pitch;
}

// max of non-negative doubles through their bit patterns (NaN bits compare above +inf, so a
// NaN residual wins and is reported).
__device__ inline void atomic_max_nonneg(unsigned long long* slot, double v) {
  atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

// Block-wide max of non-negative values, then one atomic per block.
__device__ inline void block_max_to(unsigned long long* slot, double v) {
  __shared__ double red[32];
  unsigned m = 0xffffffffu;
  for (int o = 16; o > 0; o >>= 1) {
    double w = __shfl_xor_sync(m, v, o);
    v = (w > v || w != w) ? w : v;
  }
  int tid = threadIdx.x + threadIdx.y * blockDim.x;
  int nw = (blockDim.x * blockDim.y + 31) / 32;
  if ((tid & 31) == 0) red[tid >> 5] = v;
  __syncthreads();
  if (tid < 32) {
    v = tid < nw ? red[tid] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      double w = __shfl_xor_sync(m, v, o);
      v = (w > v || w != w) ? w : v;
    }
    if (tid == 0 && v != 0.0) atomic_max_nonneg(slot, v);
  }
}

// Block-wide max of two sets of non-negative values, one atomic each per block (one barrier).
__device__ inline void block_max2_to(unsigned long long* slot_a, double a, unsigned long long* slot_b, double b) {
  __shared__ double red2[2][32];
  unsigned m = 0xffffffffu;
  for (int o = 16; o > 0; o >>= 1) {
    const double wa = __shfl_xor_sync(m, a, o), wb = __shfl_xor_sync(m, b, o);
    a = (wa > a || wa != wa) ? wa : a;
    b = (wb > b || wb != wb) ? wb : b;
  }
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nw = (blockDim.x * blockDim.y + 31) / 32;
  if ((tid & 31) == 0) {
    red2[0][tid >> 5] = a;
    red2[1][tid >> 5] = b;
  }
  __syncthreads();
  if (tid < 32) {
    a = tid < nw ? red2[0][tid] : 0.0;
    b = tid < nw ? red2[1][tid] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      const double wa = __shfl_xor_sync(m, a, o), wb = __shfl_xor_sync(m, b, o);
      a = (wa > a || wa != wa) ? wa : a;
      b = (wb > b || wb != wb) ? wb : b;
    }
    if (tid == 0) {
      if (a != 0.0) atomic_max_nonneg(slot_a, a);
      if (b != 0.0) atomic_max_nonneg(slot_b, b);
    }
  }
}

}  // namespace acs
