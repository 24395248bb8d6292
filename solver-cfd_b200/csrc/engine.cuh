// engine.cuh -- persistent thread-block-cluster engine: one cluster per case runs whole physical
// steps of the pseudo-time loop (main.f90:116-186) inside a single launch.
//
// Layout: a case is split into K horizontal strips of node rows (rows 1..jmax+1), one CTA per
// strip; K <= 16 CTAs form a thread-block cluster, so every CTA of a case is co-resident and the
// stages are separated by hardware cluster barriers (barrier.cluster.arrive.release /
// wait.acquire).  Fields live in global memory (each case is a few MB and stays in L2); reads of
// arrays written by other CTAs of the cluster use ld.global.cg.
//
// Schedule of one pseudo-iteration (the reference runs solve_U, solve_V, solve_P, solve_Z,
// solve_C one after the other; V reads um_tau, not um_n_tau, so U and V are independent, and
// P, Z, C all read the new velocities only):
//   phase 1..3: U stage s and V stage s side by side, each followed by its boundary pass; in
//               phases 1 and 2 also T, C stages 2 and 3 of the previous iteration
//   phase 4   : P (the three stages fuse pointwise) and T, C stage 1
//   control   : every CTA reads the case's residual maxima and takes the same decision; on
//               exit the pending T, C stages 2 and 3 run on their own first
// The boundary passes bcUV(u_stage, vm_tau) and bcUV(um_tau, v_stage) also rewrite the boundary
// of vm_tau / um_tau (boundary.f90:1-49).  Those arrays come from earlier boundary passes, so the
// rewrite changes nothing -- except right after the state was uploaded.  An iteration with
// CaseCtl::tau_dirty set therefore runs U and V in the reference's sequential order with the
// full boundary passes.  The one array element the rewrite does change in steady state,
// vm(imax, jmax+1), is never read by the loop.
//
// Termination: every CTA of a cluster makes the same decisions from the same residuals, each
// physical step ends after at most itc_max iterations and the launch after n_steps steps, so
// every cluster barrier is reached by all CTAs and the kernel always ends.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "acs_dev.cuh"

namespace acs {
namespace cg = cooperative_groups;

constexpr int ENGINE_THREADS = 256;  // CTA width of the EXACT engine (the FAST engine also has 512)

struct EngineArgs {
  const CaseDev* cs;
  CaseCtl* ctl;
  const int* cases;  // case id per cluster
  int* iters;        // [case * n_steps + step]
  double* err;
  int stage_elems;   // staged engine: doubles per shared-memory slot (>= (strip rows + 4) * pitch)
};

// Staged engine: each phase first copies the rows [r0-2, r1+2) of the arrays it reads with a
// stencil into shared-memory slots (cp.async, 16-byte chunks through L2), then computes from
// them.  One L2 round trip per phase replaces the dependent L2 loads of every node.
constexpr int STAGE_SLOTS = 7;

// Issues the copy of rows [ra, rb) of a case array into `slot` and returns a pointer that indexes
// like the global array for those rows.  Rows start on 32-byte boundaries (the pitch is a
// multiple of 4 doubles), so every 16-byte chunk is aligned on both sides.
__device__ __forceinline__ const double* stage_rows(const double* g, double* slot, int ra, int rb, int P) {
  const long long o = (long long)(ra - 1) * P;
  const int n16 = ((rb - ra) * P) >> 1;
  const char* src = reinterpret_cast<const char*>(g + o);
  const unsigned dst = (unsigned)__cvta_generic_to_shared(slot);
  for (int q = threadIdx.x; q < n16; q += blockDim.x)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst + 16u * (unsigned)q),
                 "l"(src + 16 * (long long)q)
                 : "memory");
  return slot - o;
}
// Completes this thread's copies, then makes every thread's copies visible to the CTA.
__device__ __forceinline__ void stage_wait() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
}

struct LocalCtl {
  int ru[3], rv[3], rt[3], rc[3], rp[2];
  int rp_read, ntau_alias, itc, step, n_steps, k, active, status, scalars, tau_dirty;
  long long total;
};

__device__ __forceinline__ void swap_l(int& a, int& b) { int t = a; a = b; b = t; }

// Strip of node rows [r0, r1) owned by one CTA.
struct Strip {
  int r0, r1;
  __device__ bool has(int j) const { return j >= r0 && j < r1; }
  __device__ int lo(int a) const { return a > r0 ? a : r0; }
  __device__ int hi(int b) const { return b < r1 - 1 ? b : r1 - 1; }  // inclusive
};

// Calls f(i, j) for i in [ia, ib], j in [ja, jb] intersected with the strip, spread over the
// CTA's threads with consecutive threads on consecutive i.
template <class F>
__device__ __forceinline__ void for_nodes(const Strip& s, int ia, int ib, int ja, int jb, F f) {
  const int j0 = s.lo(ja), j1 = s.hi(jb);
  const int w = ib - ia + 1;
  if (j1 < j0 || w <= 0) return;
  const int n = w * (j1 - j0 + 1);
  for (int q = threadIdx.x; q < n; q += blockDim.x) f(ia + q % w, j0 + q / w);
}

// Same node set, two nodes per thread and trip: g(i, j) (loads and arithmetic only) runs for both
// nodes before h(i, j, g) stores either result, so the loads of the two nodes are in flight
// together.  The second node repeats the first when the count is odd (g has no side effects).
template <class G, class H>
__device__ __forceinline__ void for_nodes_pair(const Strip& s, int ia, int ib, int ja, int jb, G g, H h) {
  const int j0 = s.lo(ja), j1 = s.hi(jb);
  const int w = ib - ia + 1;
  if (j1 < j0 || w <= 0) return;
  const int n = w * (j1 - j0 + 1);
  const int bd = blockDim.x;
  for (int q = threadIdx.x; q < n; q += 2 * bd) {
    const int q2 = q + bd;
    const bool two = q2 < n;
    const int i1 = ia + q % w, jj1 = j0 + q / w;
    const int i2 = two ? ia + q2 % w : i1, jj2 = two ? j0 + q2 / w : jj1;
    const double a1 = g(i1, jj1);
    const double a2 = g(i2, jj2);
    h(i1, jj1, a1);
    if (two) h(i2, jj2, a2);
  }
}

template <class F>
__device__ __forceinline__ void for_range(int a, int b, F f) {
  for (int q = a + threadIdx.x; q <= b; q += blockDim.x) f(q);
}

// ---- boundary passes restricted to a strip (boundary.f90; channel variant as in the oracle) ----
// u part of bcUV.  Both variants need row 2 / row ny-1 next to the rows they set, which the
// first / last strip own (strips have at least 4 rows).
__device__ inline void strip_bc_u(const CaseDev& d, const Strip& s, double* um) {
  const int nx = d.nx, ny = d.ny, P = d.pitch;
  if (d.bc == 0) {
    if (s.has(1)) for_range(2, nx, [&](int i) { um[lin(i, 1, P)] = 0.0; });
    if (s.has(ny)) for_range(2, nx, [&](int i) { um[lin(i, ny, P)] = um[lin(i, ny - 1, P)]; });
    __syncthreads();
    for_range(s.lo(1), s.hi(ny), [&](int j) {
      um[lin(2, j, P)] = 0.0; um[lin(1, j, P)] = 0.0;
      um[lin(nx, j, P)] = 0.0; um[lin(nx + 1, j, P)] = 0.0;
    });
  } else {
    for_range(s.lo(1), s.hi(ny), [&](int j) {
      um[lin(1, j, P)] = d.v_in; um[lin(2, j, P)] = d.v_in;
      um[lin(nx, j, P)] = um[lin(nx - 1, j, P)];
      um[lin(nx + 1, j, P)] = um[lin(nx, j, P)];
    });
    __syncthreads();
    if (s.has(1)) for_range(1, nx + 1, [&](int i) { um[lin(i, 1, P)] = -um[lin(i, 2, P)]; });
    if (s.has(ny)) for_range(1, nx + 1, [&](int i) { um[lin(i, ny, P)] = -um[lin(i, ny - 1, P)]; });
  }
}

// v part of bcUV
__device__ inline void strip_bc_v(const CaseDev& d, const Strip& s, double* vm) {
  const int nx = d.nx, ny = d.ny, P = d.pitch;
  if (d.bc == 0) {
    if (s.has(1)) for_range(1, nx, [&](int i) { vm[lin(i, 1, P)] = d.v_in; vm[lin(i, 2, P)] = vm[lin(i, 1, P)]; });
    if (s.has(ny)) for_range(2, nx, [&](int i) {
      vm[lin(i, ny, P)] = 2.0 * vm[lin(i, ny - 2, P)] - vm[lin(i, ny - 1, P)];
      vm[lin(i, ny + 1, P)] = 2.0 * vm[lin(i, ny - 1, P)] - vm[lin(i, ny, P)];
    });
    __syncthreads();
    for_range(s.lo(1), s.hi(ny + 1), [&](int j) {
      vm[lin(1, j, P)] = vm[lin(2, j, P)];
      if (j >= 2 && j <= ny) vm[lin(nx, j, P)] = vm[lin(nx - 1, j, P)];
    });
  } else {
    for_range(s.lo(1), s.hi(ny + 1), [&](int j) {
      vm[lin(1, j, P)] = -vm[lin(2, j, P)];
      vm[lin(nx, j, P)] = vm[lin(nx - 1, j, P)];
    });
    __syncthreads();
    if (s.has(1)) for_range(1, nx, [&](int i) { vm[lin(i, 2, P)] = 0.0; vm[lin(i, 1, P)] = -vm[lin(i, 3, P)]; });
    if (s.has(ny)) for_range(1, nx, [&](int i) { vm[lin(i, ny, P)] = 0.0; vm[lin(i, ny + 1, P)] = -vm[lin(i, ny - 1, P)]; });
  }
}

// bcP / bcZ / bcC
__device__ inline void strip_bc_cell(const CaseDev& d, const Strip& s, double* z, bool neumann_in, double zin) {
  const int nx = d.nx, ny = d.ny, P = d.pitch;
  if (d.bc == 0) {
    if (s.has(1)) for_range(1, nx, [&](int i) { z[lin(i, 1, P)] = neumann_in ? z[lin(i, 2, P)] : zin; });
    if (s.has(ny)) for_range(1, nx, [&](int i) {
      z[lin(i, ny, P)] = z[lin(i, ny - 1, P)] + 1.0 * (z[lin(i, ny - 1, P)] - z[lin(i, ny - 2, P)]);
    });
    __syncthreads();
    for_range(s.lo(1), s.hi(ny), [&](int j) {
      z[lin(1, j, P)] = z[lin(2, j, P)];
      z[lin(nx, j, P)] = z[lin(nx - 1, j, P)];
    });
  } else {
    for_range(s.lo(1), s.hi(ny), [&](int j) {
      z[lin(1, j, P)] = neumann_in ? z[lin(2, j, P)] : zin;
      z[lin(nx, j, P)] = z[lin(nx - 1, j, P)] + 1.0 * (z[lin(nx - 1, j, P)] - z[lin(nx - 2, j, P)]);
    });
    __syncthreads();
    if (s.has(1)) for_range(1, nx, [&](int i) { z[lin(i, 1, P)] = z[lin(i, 2, P)]; });
    if (s.has(ny)) for_range(1, nx, [&](int i) { z[lin(i, ny, P)] = z[lin(i, ny - 1, P)]; });
  }
}

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = (w > v || w != w) ? w : v;
  }
  return v;
}

// block max of three values, one atomic per value per CTA
__device__ inline void block_max3(double a, double b, double c, unsigned long long* slot) {
  __shared__ double red[3][32];
  a = warp_max(a); b = warp_max(b); c = warp_max(c);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (l == 0) { red[0][w] = a; red[1][w] = b; red[2][w] = c; }
  __syncthreads();
  if (w == 0) {
    a = l < nw ? red[0][l] : 0.0;
    b = l < nw ? red[1][l] : 0.0;
    c = l < nw ? red[2][l] : 0.0;
    a = warp_max(a); b = warp_max(b); c = warp_max(c);
    if (l == 0) {
      if (a != 0.0) atomic_max_nonneg(slot + 0, a);
      if (b != 0.0) atomic_max_nonneg(slot + 1, b);
      if (c != 0.0) atomic_max_nonneg(slot + 2, c);
    }
  }
  __syncthreads();
}

// ---- the engine --------------------------------------------------------------------------------
// PT provides the per-node residuals: ru(d, uin, vt, pn, i, j), rv(d, ut, vin, pn, T, i, j),
// rs<IS_C>(d, un, vn, z, i, j), p_update(d, p0, un, vn, i, j, &r), and ld(ptr, q), the load used
// for arrays that other CTAs of the cluster write.
template <class PT, int NT, int MINB = 1, bool STG = false>
__global__ void __launch_bounds__(NT, MINB) k_engine(EngineArgs a) {
  extern __shared__ __align__(16) double stg_smem[];
  cg::cluster_group cl = cg::this_cluster();
  const int K = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int c = a.cases[blockIdx.x / K];
  // the case's constants and buffer pointers in shared memory: reads of them neither go to L1/L2
  // nor have to be repeated after every global store (a global store cannot alias them)
  __shared__ CaseDev d_sh;
  if (threadIdx.x == 0) d_sh = a.cs[c];
  __syncthreads();
  const CaseDev& d = d_sh;
  CaseCtl* gk = a.ctl + c;

  LocalCtl k;
  for (int r = 0; r < 3; ++r) { k.ru[r] = gk->ru[r]; k.rv[r] = gk->rv[r]; k.rt[r] = gk->rt[r]; k.rc[r] = gk->rc[r]; }
  k.rp[0] = gk->rp[0]; k.rp[1] = gk->rp[1];
  k.rp_read = gk->rp_read; k.ntau_alias = gk->ntau_alias; k.itc = gk->itc; k.step = gk->step;
  k.n_steps = gk->n_steps; k.k = gk->k; k.active = gk->active; k.status = gk->status;
  k.scalars = gk->scalars; k.tau_dirty = gk->tau_dirty; k.total = gk->total_iters;
  if (!k.active) return;

  const int R = d.ny + 1;
  const Strip s{1 + (rank * R) / K, 1 + ((rank + 1) * R) / K};
  const int nx = d.nx, ny = d.ny;
  const bool scal = k.scalars && d.solve_scalars;
  unsigned long long* slots = gk->slot[0];
  const int ra = s.r0 - 2 > 1 ? s.r0 - 2 : 1;
  const int rb = s.r1 + 2 < R + 1 ? s.r1 + 2 : R + 1;
  auto stage = [&](int slot, const double* g) -> const double* {
    if constexpr (STG) return stage_rows(g, stg_smem + (long long)slot * a.stage_elems, ra, rb, d.pitch);
    else return g;
  };
  auto stage_done = [&]() {
    if constexpr (STG) stage_wait();
  };

  // T and C of iteration k read only the new velocities of iteration k, and U, V read only the
  // physical-step T, so T/C stages 2 and 3 of iteration k run during the U/V stages 1 and 2 of
  // iteration k+1 (four cluster barriers per pseudo-iteration instead of six).  `tb` holds the
  // buffers of the pending T/C work; on exit (or at itc_max) the pending stages run first.
  struct TcBufs { const double* un; const double* vn; const double* tau[2]; const double* phys[2]; double* out[2]; };
  TcBufs tb{};
  bool pend = false;
  // zs[v] / us / vs: staged copies of the stage input and of the velocities (null: global arrays)
  auto tc_stage = [&](const TcBufs& b, int st, const double* const* zs, const double* us, const double* vs) {
    const double* un = us ? us : b.un;
    const double* vn = vs ? vs : b.vn;
    for (int v = 0; v < 2; ++v) {
      const bool isc = v == 1;
      const double* zin = zs && zs[v] ? zs[v] : (st == 1 ? b.tau[v] : d.S2[2 * v + st - 2]);
      double* zout = st == 3 ? b.out[v] : d.S2[2 * v + st - 1];
      const double* ztau = b.tau[v];
      const double* z = b.phys[v];
      for_nodes_pair(s, 2, nx - 1, 2, ny - 1, [&](int i, int j) {
        return isc ? PT::template rs<true>(d, un, vn, zin, i, j) : PT::template rs<false>(d, un, vn, zin, i, j);
      }, [&](int i, int j, double Rz) {
        const long long q = lin(i, j, d.pitch);
        const double r = ((PT::ld(z, q) - PT::ld(ztau, q)) + Rz * d.dt) * d.dtau;
        if (st == 1) zout[q] = PT::ld(ztau, q) + r;
        else if (st == 2) zout[q] = 0.75 * PT::ld(ztau, q) + 0.25 * (PT::ld(zin, q) + r);
        else zout[q] = 1.0 / 3.0 * PT::ld(ztau, q) + 2.0 / 3.0 * (PT::ld(zin, q) + r);
      });
    }
  };
  // boundary passes of T/C stage st (callers put a __syncthreads before)
  auto tc_bc = [&](const TcBufs& b, int st) {
    strip_bc_cell(d, s, st == 3 ? b.out[0] : d.S2[st - 1], false, d.T_in);
    __syncthreads();
    strip_bc_cell(d, s, st == 3 ? b.out[1] : d.S2[2 + st - 1], false, d.C_in);
  };
  // the pending stages 2 and 3 on their own (end of a physical step)
  auto tc_tail = [&]() {
    for (int st = 2; st <= 3; ++st) {
      tc_stage(tb, st, nullptr, nullptr, nullptr);
      __syncthreads();
      tc_bc(tb, st);
      cl.sync();
    }
    pend = false;
  };

  for (int it = 0;; ++it) {
    unsigned long long* slot = slots + 3 * (it & 1);
    double mu = 0.0, mv = 0.0, mp = 0.0;
    const double* pn_read = d.P[k.rp_read];
    // ---- U and V, three stages (with T/C stages 2, 3 of the previous iteration) ----
    const bool seq = k.tau_dirty;
    if (seq && pend) tc_tail();
    for (int pass = 0; pass < (seq ? 2 : 1); ++pass) {
      const bool doU = !seq || pass == 0, doV = !seq || pass == 1;
      for (int st = 1; st <= 3; ++st) {
        const bool tc = pend && st <= 2;
        // arrays read with a stencil in this phase, staged (or the global arrays themselves)
        const double* g_ut = d.U[k.ru[R_TAU]];
        const double* g_vt = d.V[k.rv[R_TAU]];
        const double* s_ut = stage(0, g_ut);
        const double* s_vt = stage(1, g_vt);
        const double* s_pn = stage(2, pn_read);
        const double* s_uin = st == 1 ? s_ut : stage(3, d.S[st - 2]);
        const double* s_vin = st == 1 ? s_vt : stage(4, d.S[2 + st - 2]);
        const double* s_z[2] = {nullptr, nullptr};
        if (tc) {
          s_z[0] = stage(5, d.S2[st - 1]);
          s_z[1] = stage(6, d.S2[2 + st - 1]);
        }
        stage_done();
        if (doU) {
          const double* uin = s_uin;
          double* uout = st == 3 ? d.U[k.ru[R_NTAU]] : d.S[st - 1];
          const double* utau = g_ut;
          const double* um = d.U[k.ru[R_PHYS]];
          const double* vt = s_vt;
          for_nodes_pair(s, 3, nx - 1, 2, ny - 1, [&](int i, int j) { return PT::ru(d, uin, vt, s_pn, i, j); },
                         [&](int i, int j, double RU) {
            const long long q = lin(i, j, d.pitch);
            const double r = ((PT::ld(um, q) - PT::ld(utau, q)) + RU * d.dt) * d.dtau;
            if (st == 1) uout[q] = PT::ld(utau, q) + r;
            else if (st == 2) uout[q] = 0.75 * PT::ld(utau, q) + 0.25 * (PT::ld(uin, q) + r);
            else {
              uout[q] = 1.0 / 3.0 * PT::ld(utau, q) + 2.0 / 3.0 * (PT::ld(uin, q) + r);
              const double ar = fabs(r);
              mu = (ar > mu || ar != ar) ? ar : mu;
            }
          });
        }
        if (doV) {
          const double* vin = s_vin;
          double* vout = st == 3 ? d.V[k.rv[R_NTAU]] : d.S[2 + st - 1];
          const double* vtau = g_vt;
          const double* vm = d.V[k.rv[R_PHYS]];
          const double* ut = s_ut;
          const double* T = d.T[k.rt[R_PHYS]];
          for_nodes_pair(s, 2, nx - 1, 3, ny - 1, [&](int i, int j) { return PT::rv(d, ut, vin, s_pn, T, i, j); },
                         [&](int i, int j, double RV) {
            const long long q = lin(i, j, d.pitch);
            const double r = ((PT::ld(vm, q) - PT::ld(vtau, q)) + RV * d.dt) * d.dtau;
            if (st == 1) vout[q] = (PT::ld(vtau, q) + r);
            else if (st == 2) vout[q] = (0.75 * PT::ld(vtau, q) + 0.25 * (PT::ld(vin, q) + r));
            else {
              vout[q] = 1.0 / 3.0 * PT::ld(vtau, q) + 2.0 / 3.0 * (PT::ld(vin, q) + r);
              const double ar = fabs(r);
              mv = (ar > mv || ar != ar) ? ar : mv;
            }
          });
        }
        // the pending T/C work reads the previous iteration's new velocities, which after the
        // role swap are this iteration's tau arrays
        if (tc) tc_stage(tb, st + 1, s_z, tb.un == g_ut ? s_ut : nullptr, tb.vn == g_vt ? s_vt : nullptr);
        __syncthreads();
        if (doU) strip_bc_u(d, s, st == 3 ? d.U[k.ru[R_NTAU]] : d.S[st - 1]);
        if (doV) strip_bc_v(d, s, st == 3 ? d.V[k.rv[R_NTAU]] : d.S[2 + st - 1]);
        if (tc) {
          __syncthreads();
          tc_bc(tb, st + 1);
        }
        if (seq) {
          // bcUV(u_stage, vm_tau) / bcUV(um_tau, v_stage) also rewrite vm_tau / um_tau, which
          // other CTAs may still be reading for this stage: wait for the whole cluster first
          cl.sync();
          if (doU) strip_bc_v(d, s, d.V[k.rv[R_TAU]]);
          else strip_bc_u(d, s, d.U[k.ru[R_TAU]]);
        }
        cl.sync();
        if (tc && st == 2) pend = false;
        // the residual slot of the next iteration is free once every CTA is past the control
        // step of the previous one, i.e. after the first barrier of this iteration
        if (st == 1 && pass == 0 && rank == 0 && threadIdx.x == 0) {
          unsigned long long* nxt = slots + 3 * ((it + 1) & 1);
          nxt[0] = nxt[1] = nxt[2] = 0ull;
        }
      }
    }
    // ---- P, and T / C stage 1 ----
    const double* un = d.U[k.ru[R_NTAU]];
    const double* vn = d.V[k.rv[R_NTAU]];
    const double* s_un = stage(0, un);
    const double* s_vn = stage(1, vn);
    const double* s_z4[2] = {nullptr, nullptr};
    if (scal) {
      s_z4[0] = stage(2, d.T[k.rt[R_TAU]]);
      s_z4[1] = stage(3, d.C[k.rc[R_TAU]]);
    }
    stage_done();
    {
      const double* p0 = d.P[k.rp[0]];
      double* pn = d.P[k.rp[1]];
      for_nodes(s, 2, nx - 1, 2, ny - 1, [&](int i, int j) {
        double r;
        pn[lin(i, j, d.pitch)] = PT::p_update(d, p0, s_un, s_vn, i, j, &r);
        const double ar = fabs(r);
        mp = (ar > mp || ar != ar) ? ar : mp;
      });
    }
    if (scal) {
      tb.un = un;
      tb.vn = vn;
      tb.tau[0] = d.T[k.rt[R_TAU]]; tb.phys[0] = d.T[k.rt[R_PHYS]]; tb.out[0] = d.T[k.rt[R_NTAU]];
      tb.tau[1] = d.C[k.rc[R_TAU]]; tb.phys[1] = d.C[k.rc[R_PHYS]]; tb.out[1] = d.C[k.rc[R_NTAU]];
      tc_stage(tb, 1, s_z4, s_un, s_vn);
    }
    __syncthreads();
    strip_bc_cell(d, s, d.P[k.rp[1]], true, 0.0);
    if (scal) {
      __syncthreads();
      tc_bc(tb, 1);
      pend = true;
    }
    block_max3(mu, mv, mp, slot);
    cl.sync();
    // ---- control (main.f90:139-157), identical in every CTA ----
    const double ru = __longlong_as_double((long long)__ldcg(slot + 0));
    const double rv = __longlong_as_double((long long)__ldcg(slot + 1));
    const double rpv = __longlong_as_double((long long)__ldcg(slot + 2));
    double e = ru;
    if (rv > e || rv != rv) e = rv;
    if (rpv > e || rpv != rpv) e = rpv;
    k.k += 1;
    k.total += 1;
    bool step_done = false, copy = false;
    if (e != e || e > 1.0e300) {
      k.status = 2;
      k.active = 0;
      step_done = true;
    } else if (k.itc != 1 && e < d.eps) {
      if (pend) tc_tail();
      k.rp_read = k.rp[1];
      k.ntau_alias = 1;
      swap_l(k.ru[R_PHYS], k.ru[R_NTAU]);
      swap_l(k.rv[R_PHYS], k.rv[R_NTAU]);
      if (d.solve_scalars) { swap_l(k.rt[R_PHYS], k.rt[R_NTAU]); swap_l(k.rc[R_PHYS], k.rc[R_NTAU]); }
      step_done = true;
    } else {
      swap_l(k.ru[R_TAU], k.ru[R_NTAU]);
      swap_l(k.rv[R_TAU], k.rv[R_NTAU]);
      swap_l(k.rp[0], k.rp[1]);
      k.rp_read = k.rp[0];
      k.ntau_alias = 2;
      k.tau_dirty = 0;
      if (d.solve_scalars) { swap_l(k.rt[R_TAU], k.rt[R_NTAU]); swap_l(k.rc[R_TAU], k.rc[R_NTAU]); }
      k.itc += 1;
      if (k.itc >= d.itc_max) { copy = true; step_done = true; }
    }
    if (copy) {  // loop condition failed after the copies: phys = latest iterate (main.f90:154-157)
      if (pend) tc_tail();
      const int nf = d.solve_scalars ? 4 : 2;
      for (int f = 0; f < nf; ++f) {
        const double* src = f == 0 ? d.U[k.ru[R_TAU]] : f == 1 ? d.V[k.rv[R_TAU]] : f == 2 ? d.T[k.rt[R_TAU]] : d.C[k.rc[R_TAU]];
        double* dst = f == 0 ? d.U[k.ru[R_PHYS]] : f == 1 ? d.V[k.rv[R_PHYS]] : f == 2 ? d.T[k.rt[R_PHYS]] : d.C[k.rc[R_PHYS]];
        const long long q0 = lin(1, s.r0, d.pitch), q1 = lin(1, s.r1, d.pitch);
        for (long long q = q0 + threadIdx.x; q < q1; q += blockDim.x) dst[q] = PT::ld(src, q);
      }
      cl.sync();
    }
    if (step_done) {
      if (rank == 0 && threadIdx.x == 0 && k.step < k.n_steps) {
        if (a.iters) a.iters[(long long)c * k.n_steps + k.step] = k.k;
        if (a.err) a.err[(long long)c * k.n_steps + k.step] = e;
      }
      if (k.status != 2) {
        k.step += 1;
        k.itc = 0;
        k.k = 0;
        if (k.step >= k.n_steps) { k.active = 0; k.status = 1; }
      }
    }
    if (!k.active) break;
  }
  if (rank == 0 && threadIdx.x == 0) {
    for (int r = 0; r < 3; ++r) { gk->ru[r] = k.ru[r]; gk->rv[r] = k.rv[r]; gk->rt[r] = k.rt[r]; gk->rc[r] = k.rc[r]; }
    gk->rp[0] = k.rp[0]; gk->rp[1] = k.rp[1];
    gk->rp_read = k.rp_read; gk->ntau_alias = k.ntau_alias; gk->itc = k.itc; gk->step = k.step;
    gk->k = k.k; gk->active = k.active; gk->status = k.status; gk->tau_dirty = k.tau_dirty;
    gk->total_iters = k.total;
  }
}

}  // namespace acs
