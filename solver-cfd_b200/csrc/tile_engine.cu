// tile_engine.cu -- the tile engine: one pseudo-iteration of every active case as four stage
// kernels over 32 x 32-node tiles whose inputs are loaded into shared memory by TMA.
//
//   k_te_uv<1..3>: Runge-Kutta stage s of solve_U and of solve_V (equations.f90:244-301 and
//                  :546-603) side by side: the stage inputs (u_in, v_in) and the arrays read with
//                  a stencil (um_tau, vm_tau, pn) arrive as 36 x 36 boxes (the tile plus the
//                  two-node QUICK halo) through cp.async.bulk.tensor; the pointwise arrays (um,
//                  vm, T, the porous mask, the 1-D metric tables) are read from global memory.
//                  The stage of every interior node of the tile is computed into a shared tile,
//                  bcUV (boundary.f90:1-49) is applied to that tile, and the whole tile is
//                  stored.  Stage 3 also reduces residual_u / residual_v (stage-3 max |res|).
//   k_te_ptc:      solve_P (:607-665; with RP frozen the three stages give pn = p + dtau*beta*RP)
//                  and bcP on the tile, then the three stages of solve_Z (:669-719) and of
//                  solve_C (:769-819) fused over one 40 x 40 box (tile plus four): stage 1 on
//                  the tile grown by two nodes, stage 2 grown by one, stage 3 on the tile, each
//                  followed by bcZ / bcC on the nodes it computed, so the intermediate stages
//                  never leave shared memory.
//
// Why a tile can finish its own boundary: the tile table (te_case_tiles) puts every boundary node
// in a tile that also holds the nodes its boundary pass reads (at most two nodes further in,
// toward the interior), so the stored arrays are complete after every launch -- interior and
// boundary -- exactly like the reference's arrays after each bc* call.  Inside the fused T/C
// stages a grown region may hold boundary nodes whose sources lie outside it; those are left
// unset, and no node the next stage reads depends on one of them (a node read by the five-point
// stencil of an interior node of the next region has its sources within the current region).
//
// The first pseudo-iteration after the state was uploaded reads um_tau / vm_tau before their
// boundary passes: solve_U's stage 1 reads both as they are, solve_V's stage 1 reads vm_tau after
// solve_U's bcUV rewrote its boundary, and stages 2 and 3 read both rewritten.  Stage 1 therefore
// gives V a copy of the vm_tau box with the boundary pass applied (identical to the box once the
// arrays satisfy the passes), and k_te_tau_bc applies the passes to um_tau / vm_tau before stage 2
// for the cases that were uploaded.  Every iteration runs the same kernels and arithmetic.
//
// TMA: 2-D tensor maps over each case buffer (dims pitch x (ny+1), FP64, no swizzle, zero fill
// outside), non-multicast loads into 128-byte aligned shared memory, one mbarrier per CTA with the
// expected byte count; every wait is bounded (about a second), after which the CTA sets the
// error word, waits once more (bounded) so no copy lands after it has left, and returns.
#include "tile_engine.h"

#include <cudaTypedefs.h>

#include <algorithm>

#include "bc_exact.cuh"
#include "points_fast.cuh"

namespace acs {

void te_case_tiles(int c, int pitch, int ny, std::vector<Tile>& out) {
  std::vector<int> xs, ys;
  for (int x = 0;; x += TE_TILE) {
    if (x + TE_TILE >= pitch) { xs.push_back(std::max(0, pitch - TE_TILE)); break; }
    xs.push_back(x);
  }
  for (int y = 0;; y += TE_TILE) {
    if (y + TE_TILE >= ny + 1) { ys.push_back(std::max(0, ny + 1 - TE_TILE)); break; }
    ys.push_back(y);
  }
  for (int y : ys)
    for (int x : xs) out.push_back({c, x + 1, y + 1, 0});
}

int te_encode_maps(const std::vector<CaseDev>& cases, TeMaps* maps) {
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q{};
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
      q != cudaDriverEntryPointSuccess)
    return 1;
  auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  for (size_t c = 0; c < cases.size(); ++c) {
    const CaseDev& d = cases[c];
    const double* bufs[TE_NBUF] = {d.U[0], d.U[1], d.U[2], d.V[0], d.V[1], d.V[2], d.P[0], d.P[1], d.T[0],
                                   d.T[1], d.T[2], d.C[0], d.C[1], d.C[2], d.S[0], d.S[1], d.S[2], d.S[3]};
    const cuuint64_t dims[2] = {(cuuint64_t)d.pitch, (cuuint64_t)(d.ny + 1)};
    const cuuint64_t strides[1] = {(cuuint64_t)d.pitch * sizeof(double)};
    const cuuint32_t estr[2] = {1, 1};
    auto make = [&](CUtensorMap* m, const double* base, cuuint32_t bw, cuuint32_t bh) {
      const cuuint32_t box[2] = {bw, bh};
      return encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    bool ok = true;
    for (int b = 0; b < TE_NBUF; ++b) {
      ok = ok && make(&maps[c].uv[b], bufs[b], TE_BOX_UV, TE_BOX_UV);
      ok = ok && make(&maps[c].ptc[b], bufs[b], TE_BOX_PTC, TE_BOX_PTC);
      ok = ok && make(&maps[c].pt[b], bufs[b], TE_TILE, TE_TILE);
    }
    for (int b = 0; b < 3; ++b) ok = ok && make(&maps[c].t33[b], d.T[b], TE_TILE, TE_TILE + 1);
    ok = ok && make(&maps[c].liga32, d.liga, TE_TILE, TE_TILE);
    ok = ok && make(&maps[c].liga36, d.liga, TE_BOX_UV, TE_BOX_UV);
    ok = ok && make(&maps[c].buoyw, d.S2[3], TE_TILE, TE_TILE);
    if (!ok) return 2;
  }
  return 0;
}

namespace {

using PT = PtFastT<LdGen>;
constexpr int NT = TE_TILE;
constexpr int BU = TE_BOX_UV;
constexpr int BP = TE_BOX_PTC;
constexpr uint32_t BOX_UV_BYTES = BU * BU * 8;
constexpr uint32_t BOX_PTC_BYTES = BP * BP * 8;
constexpr long long kWaitCycles = 2000000000ll;  // about one second at the B200's clocks

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned long long* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned long long* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ bool mbar_wait_bounded(unsigned long long* bar, uint32_t parity) {
  const long long t0 = clock64();
  for (long long it = 0; it < (1ll << 26); ++it) {
    if (mbar_try(bar, parity)) return true;
    if (clock64() - t0 > kWaitCycles) break;
  }
  return false;
}
// 2-D tiled TMA load of the box at (x, y) into dst, completing on `bar`; x is even (16-byte
// aligned in FP64), y may be negative (rows outside the array read as zero).
__device__ __forceinline__ void tma_load(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(saddr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(saddr(bar))
      : "memory");
}
// Thread 0 waits (bounded) and the CTA takes the outcome together.  On a timeout the copies may
// still be in flight: one more bounded wait, so none lands after the CTA has returned.
__device__ bool cta_wait(unsigned long long* bar, uint32_t parity, int* flag, int* err) {
  if (threadIdx.x == 0) {
    bool ok = mbar_wait_bounded(bar, parity);
    if (!ok) {
      atomicExch(err, 1);
      mbar_wait_bounded(bar, parity);
    }
    *flag = ok ? 1 : 0;
  }
  __syncthreads();
  const bool ok = *flag != 0;
  __syncthreads();
  return ok;
}

// Copies the case descriptor into shared memory (8-byte words, all threads).
__device__ __forceinline__ void load_case(CaseDev* dst, const CaseDev* src) {
  static_assert(sizeof(CaseDev) % 8 == 0, "case descriptor size");
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
  unsigned long long* o = reinterpret_cast<unsigned long long*>(dst);
  for (int q = threadIdx.x; q < (int)(sizeof(CaseDev) / 8); q += blockDim.x) o[q] = s[q];
}

// A window of a shared-memory tile: node (i, j) at a[(i-i0) + (j-j0)*P] for i in [i0, i0+w),
// j in [j0, j0+h).
struct Win {
  double* a;
  int i0, j0, w, h, P;
  __device__ bool in(int i, int j) const { return i >= i0 && i < i0 + w && j >= j0 && j < j0 + h; }
  __device__ double& at(int i, int j) const { return a[(i - i0) + (j - j0) * P]; }
  // thread-strided loops over the window's columns in [ia, ib] / rows in [ja, jb]
  template <class F>
  __device__ void cols(int ia, int ib, F f) const {
    const int lo = max(ia, i0), hi = min(ib, i0 + w - 1);
    for (int i = lo + (int)threadIdx.x; i <= hi; i += blockDim.x) f(i);
  }
  template <class F>
  __device__ void rows(int ja, int jb, F f) const {
    const int lo = max(ja, j0), hi = min(jb, j0 + h - 1);
    for (int j = lo + (int)threadIdx.x; j <= hi; j += blockDim.x) f(j);
  }
};

// The two passes of each boundary routine on a window, in the reference's order (pass 0 first,
// a __syncthreads between them).  An assignment runs only where the node and every node it reads
// lie in the window.  Reference variant (bc = 0): rows first, then columns; channel variant
// (bc = 1): columns first, then rows -- as in bc_exact.cuh.
__device__ void bc_u_pass(const CaseDev& d, const Win& w, int pass) {
  const int nx = d.nx, ny = d.ny;
  if (d.bc == 0) {
    if (pass == 0) {
      w.cols(2, nx, [&](int i) {
        if (w.in(i, 1)) w.at(i, 1) = 0.0;
        if (w.in(i, ny) && w.in(i, ny - 1)) w.at(i, ny) = w.at(i, ny - 1);
      });
    } else {
      w.rows(1, ny, [&](int j) {
        if (w.in(2, j)) w.at(2, j) = 0.0;
        if (w.in(1, j)) w.at(1, j) = 0.0;
        if (w.in(nx, j)) w.at(nx, j) = 0.0;
        if (w.in(nx + 1, j)) w.at(nx + 1, j) = 0.0;
      });
    }
  } else {
    if (pass == 0) {
      w.rows(1, ny, [&](int j) {
        if (w.in(1, j)) w.at(1, j) = d.v_in;
        if (w.in(2, j)) w.at(2, j) = d.v_in;
        if (w.in(nx, j) && w.in(nx - 1, j)) w.at(nx, j) = w.at(nx - 1, j);
        if (w.in(nx + 1, j) && w.in(nx, j)) w.at(nx + 1, j) = w.at(nx, j);
      });
    } else {
      w.cols(1, nx + 1, [&](int i) {
        if (w.in(i, 1) && w.in(i, 2)) w.at(i, 1) = -w.at(i, 2);
        if (w.in(i, ny) && w.in(i, ny - 1)) w.at(i, ny) = -w.at(i, ny - 1);
      });
    }
  }
}

__device__ void bc_v_pass(const CaseDev& d, const Win& w, int pass) {
  const int nx = d.nx, ny = d.ny;
  if (d.bc == 0) {
    if (pass == 0) {
      w.cols(1, nx, [&](int i) {
        if (w.in(i, 1)) w.at(i, 1) = d.v_in;
        if (w.in(i, 2)) w.at(i, 2) = d.v_in;
        if (i >= 2) {
          if (w.in(i, ny) && w.in(i, ny - 2) && w.in(i, ny - 1))
            w.at(i, ny) = 2.0 * w.at(i, ny - 2) - w.at(i, ny - 1);
          if (w.in(i, ny + 1) && w.in(i, ny - 1) && w.in(i, ny))
            w.at(i, ny + 1) = 2.0 * w.at(i, ny - 1) - w.at(i, ny);
        }
      });
    } else {
      w.rows(1, ny + 1, [&](int j) {
        if (w.in(1, j) && w.in(2, j)) w.at(1, j) = w.at(2, j);
        if (j >= 2 && j <= ny && w.in(nx, j) && w.in(nx - 1, j)) w.at(nx, j) = w.at(nx - 1, j);
      });
    }
  } else {
    if (pass == 0) {
      w.rows(1, ny + 1, [&](int j) {
        if (w.in(1, j) && w.in(2, j)) w.at(1, j) = -w.at(2, j);
        if (w.in(nx, j) && w.in(nx - 1, j)) w.at(nx, j) = w.at(nx - 1, j);
      });
    } else {
      w.cols(1, nx, [&](int i) {
        if (w.in(i, 2)) w.at(i, 2) = 0.0;
        if (w.in(i, ny)) w.at(i, ny) = 0.0;
        if (w.in(i, 1) && w.in(i, 3)) w.at(i, 1) = -w.at(i, 3);
        if (w.in(i, ny + 1) && w.in(i, ny - 1)) w.at(i, ny + 1) = -w.at(i, ny - 1);
      });
    }
  }
}

// bcP (neumann_in = true) / bcZ, bcC (inflow value zin)
__device__ void bc_cell_pass(const CaseDev& d, const Win& w, int pass, bool neumann_in, double zin) {
  const int nx = d.nx, ny = d.ny;
  if (d.bc == 0) {
    if (pass == 0) {
      w.cols(1, nx, [&](int i) {
        if (w.in(i, 1)) {
          if (!neumann_in) w.at(i, 1) = zin;
          else if (w.in(i, 2)) w.at(i, 1) = w.at(i, 2);
        }
        if (w.in(i, ny) && w.in(i, ny - 1) && w.in(i, ny - 2))
          w.at(i, ny) = w.at(i, ny - 1) + 1.0 * (w.at(i, ny - 1) - w.at(i, ny - 2));
      });
    } else {
      w.rows(1, ny, [&](int j) {
        if (w.in(1, j) && w.in(2, j)) w.at(1, j) = w.at(2, j);
        if (w.in(nx, j) && w.in(nx - 1, j)) w.at(nx, j) = w.at(nx - 1, j);
      });
    }
  } else {
    if (pass == 0) {
      w.rows(1, ny, [&](int j) {
        if (w.in(1, j)) {
          if (!neumann_in) w.at(1, j) = zin;
          else if (w.in(2, j)) w.at(1, j) = w.at(2, j);
        }
        if (w.in(nx, j) && w.in(nx - 1, j) && w.in(nx - 2, j))
          w.at(nx, j) = w.at(nx - 1, j) + 1.0 * (w.at(nx - 1, j) - w.at(nx - 2, j));
      });
    } else {
      w.cols(1, nx, [&](int i) {
        if (w.in(i, 1) && w.in(i, 2)) w.at(i, 1) = w.at(i, 2);
        if (w.in(i, ny) && w.in(i, ny - 1)) w.at(i, ny) = w.at(i, ny - 1);
      });
    }
  }
}

__device__ __forceinline__ double nanmax(double m, double a) { return (a > m || a != a) ? a : m; }

// Metric-table slice: entries k0 .. k0+N-1 of a case table (4 doubles each) into shared memory,
// component c of entry k0+m at sl[m + c*N] (entries outside the table left unset); returns the
// pointer that LdShared<N>::met indexes by table entry.
template <int N>
__device__ __forceinline__ const double* met_slice(double* sl, const double* table, int k0, int kmax) {
  for (int e = threadIdx.x; e < 4 * N; e += blockDim.x) {
    const int m = e >> 2, c = e & 3, k = k0 + m;
    if (k >= 0 && k <= kmax) sl[m + c * N] = __ldg(table + 4 * k + c);
  }
  return sl - k0;
}

// ---- U and V, Runge-Kutta stage ST ------------------------------------------------------------
// Shared memory (doubles): um_tau, vm_tau, pn boxes (36 x 36, the tile plus two nodes), for ST > 1
// the stage inputs u_in, v_in (36 x 36); um and vm (32 x 32, overwritten in place by the stage
// outputs), T (32 x 33, rows j0-1 .. j0+31), liga (32 x 32) and the metric slices.
constexpr int MS_UV = 34;  // metric entries i0-1 .. i0+32
template <int ST>
constexpr size_t smem_uv() {
  return (size_t)(ST == 1 ? 4 : 5) * BOX_UV_BYTES + 3 * NT * NT * 8 + NT * (NT + 1) * 8 + 2 * MS_UV * 32;
}

template <int ST>
__global__ void __launch_bounds__(TE_THREADS, 2) k_te_uv(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                       const Tile* __restrict__ tiles,
                                                       const TeMaps* __restrict__ maps, int* err) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ CaseDev d;
  __shared__ unsigned long long bar;
  __shared__ int flag;
  const Tile t = tiles[blockIdx.x];
  const CaseCtl* kc = ctl + t.c;
  // after a TMA timeout anywhere in the run every later CTA leaves at once (the host reports it)
  if (!kc->active || *(volatile int*)err) return;
  const int ru_tau = kc->ru[R_TAU], ru_phys = kc->ru[R_PHYS], ru_ntau = kc->ru[R_NTAU];
  const int rv_tau = kc->rv[R_TAU], rv_phys = kc->rv[R_PHYS], rv_ntau = kc->rv[R_NTAU];
  const int rt_phys = kc->rt[R_PHYS], rp_read = kc->rp_read;
  const bool buoy = (cs[t.c].flags & F_BUOY) != 0;
  // the buoyancy factor w = 1 - 2/(T(i,j) + T(i,j-1)) of the physical-step temperature: stage 1 of
  // a step's first pseudo-iteration computes it from T and stores it, every other launch loads it
  const bool fresh = ST == 1 && kc->k == 0;

  double* Ub = reinterpret_cast<double*>(sm);  // um_tau box
  double* Vb = Ub + BU * BU;                   // vm_tau box
  double* Pb = Vb + BU * BU;                   // pn box
  double* Ui = ST == 1 ? Ub : Pb + BU * BU;    // stage inputs
  double* Vi = ST == 1 ? Vb : Ui + BU * BU;
  double* Um = (ST == 1 ? Pb + BU * BU : Vi) + BU * BU;  // um, then the U stage output (stage 1:
                                                         // after the vm_tau copy for V)
  double* Vm = Um + NT * NT;                   // vm, then the V stage output
  double* Lg = Vm + NT * NT;                   // liga
  double* Tb = Lg + NT * NT;                   // T, rows j0-1 .. j0+31 (or w, rows j0 .. j0+31)
  double* Ms = Tb + NT * (NT + 1);             // metric slices
  double* Mt = Ms + 4 * MS_UV;

  const TeMaps* M = maps + t.c;
  const int x0 = t.i0 - 1, y0 = t.j0 - 1;
  if (threadIdx.x == 0) mbar_init(&bar);
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_expect(&bar, (ST == 1 ? 3u : 5u) * BOX_UV_BYTES + 3u * NT * NT * 8 +
                          (buoy ? (fresh ? NT * (NT + 1) * 8u : NT * NT * 8u) : 0u));
    tma_load(Ub, &M->uv[TE_U + ru_tau], x0 - 2, y0 - 2, &bar);
    tma_load(Vb, &M->uv[TE_V + rv_tau], x0 - 2, y0 - 2, &bar);
    tma_load(Pb, &M->uv[TE_P + rp_read], x0 - 2, y0 - 2, &bar);
    if (ST > 1) {
      tma_load(Ui, &M->uv[TE_S + ST - 2], x0 - 2, y0 - 2, &bar);
      tma_load(Vi, &M->uv[TE_S + 2 + ST - 2], x0 - 2, y0 - 2, &bar);
    }
    tma_load(Um, &M->pt[TE_U + ru_phys], x0, y0, &bar);
    tma_load(Vm, &M->pt[TE_V + rv_phys], x0, y0, &bar);
    tma_load(Lg, &M->liga32, x0, y0, &bar);
    if (buoy && fresh) tma_load(Tb, &M->t33[rt_phys], x0, y0 - 1, &bar);
    if (buoy && !fresh) tma_load(Tb, &M->buoyw, x0, y0, &bar);
  }
  load_case(&d, cs + t.c);
  const CaseDev& dg = cs[t.c];
  const double* mxs = met_slice<MS_UV>(Ms, dg.mx, t.i0 - 1, dg.nx + 1);
  const double* mys = met_slice<MS_UV>(Mt, dg.my, t.j0 - 1, dg.ny + 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    d.mx = mxs;
    d.my = mys;
  }
  if (!cta_wait(&bar, 0, &flag, err)) return;

  using PS = PtFastT<LdShared<MS_UV>>;
  const int nx = d.nx, ny = d.ny;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const double* Vs = Vi;  // the vm_tau (stage 1) or stage input V reads with its stencil
  if (ST == 1 && (t.i0 - 2 <= 1 || t.i0 + NT + 1 >= nx || t.j0 - 2 <= 2 || t.j0 + NT + 1 >= ny)) {
    // Stage 1 reads vm_tau twice: solve_U as it is (the reference's bcUV then rewrites its
    // boundary as a side effect), solve_V after that rewrite.  The two differ only right after an
    // upload; a box that holds v boundary nodes gets a copy with bcUV's v part applied for V, and U
    // keeps the box as loaded.
    double* Vc = Pb + BU * BU;
    for (int q = threadIdx.x; q < BU * BU; q += blockDim.x) Vc[q] = Vb[q];
    __syncthreads();
    const Win wc{Vc, t.i0 - 2, t.j0 - 2, BU, BU, BU};
    bc_v_pass(d, wc, 0);
    __syncthreads();
    bc_v_pass(d, wc, 1);
    __syncthreads();
    Vs = Vc;
  }
  double mu = 0.0, mv = 0.0;
#pragma unroll 1
  for (int r = 0; r < NT / 8; ++r) {
    const int li = tx, lj = ty + 8 * r;
    const int i = t.i0 + li, j = t.j0 + lj;
    const int qs = (li + 2) + (lj + 2) * BU;
    const int qo = li + lj * NT;
    const bool por = Lg[qo] != 0.0;
    // both residuals for every node of the tile (the boxes hold every neighbour), kept only at
    // interior nodes: no branch separates the two chains
    const double RU = PS::ru_at(d, Ui, Vb, Pb, BU, qs, por, i, j);
    double w = 0.0;
    if (buoy) {
      if (fresh) {
        w = 1.0 - 2.0 / (Tb[li + (lj + 1) * NT] + Tb[li + lj * NT]);
        if (i <= nx && j <= ny + 1) d.S2[3][lin(i, j, d.pitch)] = w;  // v nodes only: inside the buffer
      } else {
        w = Tb[li + lj * NT];
      }
    }
    const double RV = PS::rv_at_w(d, Ub, Vs, Pb, w, BU, qs, por, i, j);
    const double ut = Ub[qs], vt = Vb[qs];
    const double ru = ((Um[qo] - ut) + RU * d.dt) * d.dtau;
    const double rv = ((Vm[qo] - vt) + RV * d.dt) * d.dtau;
    double ou, ov;
    if (ST == 1) {
      ou = ut + ru;
      ov = vt + rv;
    } else if (ST == 2) {
      ou = 0.75 * ut + 0.25 * (Ui[qs] + ru);
      ov = 0.75 * vt + 0.25 * (Vi[qs] + rv);
    } else {
      ou = 1.0 / 3.0 * ut + 2.0 / 3.0 * (Ui[qs] + ru);
      ov = 1.0 / 3.0 * vt + 2.0 / 3.0 * (Vi[qs] + rv);
    }
    if (i >= 3 && i <= nx - 1 && j >= 2 && j <= ny - 1) {
      Um[qo] = ou;
      if (ST == 3) mu = nanmax(mu, fabs(ru));
    }
    if (i >= 2 && i <= nx - 1 && j >= 3 && j <= ny - 1) {
      Vm[qo] = ov;
      if (ST == 3) mv = nanmax(mv, fabs(rv));
    }
  }
  if (ST == 3) block_max2_to(&ctl[t.c].res_u, mu, &ctl[t.c].res_v, mv);
  __syncthreads();
  // boundary passes, only where the tile holds boundary nodes (u: i in {1,2,nx,nx+1} or
  // j in {1,ny}; v: i in {1,nx} or j in {1,2,ny,ny+1})
  if (!(t.i0 >= 3 && t.i0 + NT - 1 <= nx - 1 && t.j0 >= 3 && t.j0 + NT - 1 <= ny - 1)) {
    const Win wu{Um, t.i0, t.j0, NT, NT, NT}, wv{Vm, t.i0, t.j0, NT, NT, NT};
    bc_u_pass(d, wu, 0);
    bc_v_pass(d, wv, 0);
    __syncthreads();
    bc_u_pass(d, wu, 1);
    bc_v_pass(d, wv, 1);
    __syncthreads();
  }
  double* uo_g = ST == 3 ? d.U[ru_ntau] : d.S[ST - 1];
  double* vo_g = ST == 3 ? d.V[rv_ntau] : d.S[2 + ST - 1];
  for (int r = 0; r < NT / 8; ++r) {
    const int li = tx, lj = ty + 8 * r;
    const int i = t.i0 + li, j = t.j0 + lj;
    const int qo = li + lj * NT;
    if (i <= nx + 1 && j <= ny) uo_g[lin(i, j, d.pitch)] = Um[qo];
    if (i <= nx && j <= ny + 1) vo_g[lin(i, j, d.pitch)] = Vm[qo];
  }
}

// ---- P, then T and C (three stages each) -------------------------------------------------------
// Shared memory (doubles): un, vn, T_tau, C_tau boxes (40 x 40, the tile plus four nodes); liga
// (36 x 36, the tile plus two); two stage buffers per scalar (36 x 36); p (32 x 32, overwritten in
// place by pn); the metric slices.  The physical-step T and C, read once per node and stage, come
// through the read-only cache.  Stage s of T and C covers the tile grown by g = 3 - s nodes, i.e.
// positions [2-g, 34+g) of the 36 x 36 layout; one pass computes both scalars at each node, so the
// two share their loads of un, vn, liga and the metrics, and the stages of T and C share barriers.
constexpr int MS_PTC = 38;  // metric entries i0-2 .. i0+35
constexpr size_t SMEM_PTC2 = 4 * (size_t)BOX_PTC_BYTES + 5 * (size_t)BOX_UV_BYTES + NT * NT * 8 + 2 * MS_PTC * 32;

struct ScalarSet {
  const double* Z;    // the tau box (40 x 40)
  const double* Zp;   // the physical-step array (global, pitched)
  double* S1;         // stage buffers (36 x 36)
  double* S2;
  double zin;         // inflow value
};

// stage ST (1..3) of T and of C on the tile grown by 3 - ST nodes, then bcZ and bcC there (only
// where the region holds boundary cells: `edge`)
template <int ST>
__device__ __forceinline__ void scalar_stage2(const CaseDev& d, const Tile& t, const double* Un, const double* Vn,
                                              const double* Lg, const ScalarSet& T, const ScalarSet& C, bool edge) {
  using PS = PtFastT<LdShared<MS_PTC>>;
  constexpr int g = 3 - ST, e = NT + 2 * g, o36 = 2 - g, o40 = 4 - g;
  constexpr int Pz = ST == 1 ? BP : BU;
  const double* tin = ST == 1 ? T.Z : ST == 2 ? T.S1 : T.S2;
  const double* cin = ST == 1 ? C.Z : ST == 2 ? C.S1 : C.S2;
  double* tout = ST == 2 ? T.S2 : T.S1;
  double* cout = ST == 2 ? C.S2 : C.S1;
  const int nx = d.nx, ny = d.ny;
  for (int q = threadIdx.x; q < e * e; q += blockDim.x) {
    const int a = q % e, b = q / e;
    const int i = t.i0 - g + a, j = t.j0 - g + b;
    if (i >= 2 && i <= nx - 1 && j >= 2 && j <= ny - 1) {
      const int q36 = (o36 + a) + (o36 + b) * BU, q40 = (o40 + a) + (o40 + b) * BP;
      const int qz = ST == 1 ? q40 : q36;
      const bool por = Lg[q36] != 0.0;
      const long long qg = lin(i, j, d.pitch);
      const double Rt = PS::template rs_at<false>(d, Un, Vn, BP, q40, tin, Pz, qz, por, i, j);
      const double Rc = PS::template rs_at<true>(d, Un, Vn, BP, q40, cin, Pz, qz, por, i, j);
      const double tt = T.Z[q40], ct = C.Z[q40];
      const double rt = ((__ldg(T.Zp + qg) - tt) + Rt * d.dt) * d.dtau;
      const double rc = ((__ldg(C.Zp + qg) - ct) + Rc * d.dt) * d.dtau;
      if (ST == 1) {
        tout[q36] = tt + rt;
        cout[q36] = ct + rc;
      } else if (ST == 2) {
        tout[q36] = 0.75 * tt + 0.25 * (T.S1[q36] + rt);
        cout[q36] = 0.75 * ct + 0.25 * (C.S1[q36] + rc);
      } else {
        tout[q36] = 1.0 / 3.0 * tt + 2.0 / 3.0 * (T.S2[q36] + rt);
        cout[q36] = 1.0 / 3.0 * ct + 2.0 / 3.0 * (C.S2[q36] + rc);
      }
    }
  }
  __syncthreads();
  if (edge) {
    const Win wt{tout + o36 + o36 * BU, t.i0 - g, t.j0 - g, e, e, BU};
    const Win wc{cout + o36 + o36 * BU, t.i0 - g, t.j0 - g, e, e, BU};
    bc_cell_pass(d, wt, 0, false, T.zin);
    bc_cell_pass(d, wc, 0, false, C.zin);
    __syncthreads();
    bc_cell_pass(d, wt, 1, false, T.zin);
    bc_cell_pass(d, wc, 1, false, C.zin);
    __syncthreads();
  }
}

__device__ void te_scalars(const CaseDev& d, const Tile& t, const double* Un, const double* Vn, const double* Lg,
                           const ScalarSet& T, const ScalarSet& C, double* to_g, double* co_g, bool edge) {
  scalar_stage2<1>(d, t, Un, Vn, Lg, T, C, edge);
  scalar_stage2<2>(d, t, Un, Vn, Lg, T, C, edge);
  scalar_stage2<3>(d, t, Un, Vn, Lg, T, C, edge);
  const int nx = d.nx, ny = d.ny;
  for (int q = threadIdx.x; q < NT * NT; q += blockDim.x) {
    const int a = q % NT, b = q / NT;
    const int i = t.i0 + a, j = t.j0 + b;
    if (i <= nx && j <= ny) {
      const int q36 = (2 + a) + (2 + b) * BU;
      to_g[lin(i, j, d.pitch)] = T.S1[q36];
      co_g[lin(i, j, d.pitch)] = C.S1[q36];
    }
  }
}

__global__ void __launch_bounds__(TE_THREADS, 2) k_te_ptc(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                        const Tile* __restrict__ tiles,
                                                        const TeMaps* __restrict__ maps, int* err) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ CaseDev d;
  __shared__ unsigned long long bar;
  __shared__ int flag;
  const Tile t = tiles[blockIdx.x];
  const CaseCtl* kc = ctl + t.c;
  if (!kc->active || *(volatile int*)err) return;
  const int ru_ntau = kc->ru[R_NTAU], rv_ntau = kc->rv[R_NTAU];
  const int rt_tau = kc->rt[R_TAU], rt_phys = kc->rt[R_PHYS], rt_ntau = kc->rt[R_NTAU];
  const int rc_tau = kc->rc[R_TAU], rc_phys = kc->rc[R_PHYS], rc_ntau = kc->rc[R_NTAU];
  const int rp0 = kc->rp[0], rp1 = kc->rp[1];
  const bool scal = kc->scalars != 0 && cs[t.c].solve_scalars != 0;

  double* Un = reinterpret_cast<double*>(sm);
  double* Vn = Un + BP * BP;
  double* Zt = Vn + BP * BP;  // T_tau
  double* Zc = Zt + BP * BP;  // C_tau
  double* Lg = Zc + BP * BP;  // liga
  double* S1t = Lg + BU * BU;  // stage buffers of T and C
  double* S2t = S1t + BU * BU;
  double* S1c = S2t + BU * BU;
  double* S2c = S1c + BU * BU;
  double* P0 = S2c + BU * BU;  // p, then pn
  double* Ms = P0 + NT * NT;
  double* Mt = Ms + 4 * MS_PTC;
  const TeMaps* M = maps + t.c;
  const int x0 = t.i0 - 1, y0 = t.j0 - 1;
  if (threadIdx.x == 0) mbar_init(&bar);
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_expect(&bar, 2u * BOX_PTC_BYTES + NT * NT * 8u + (scal ? 2u * BOX_PTC_BYTES + BOX_UV_BYTES : 0u));
    tma_load(Un, &M->ptc[TE_U + ru_ntau], x0 - 4, y0 - 4, &bar);
    tma_load(Vn, &M->ptc[TE_V + rv_ntau], x0 - 4, y0 - 4, &bar);
    tma_load(P0, &M->pt[TE_P + rp0], x0, y0, &bar);
    if (scal) {
      tma_load(Zt, &M->ptc[TE_T + rt_tau], x0 - 4, y0 - 4, &bar);
      tma_load(Zc, &M->ptc[TE_C + rc_tau], x0 - 4, y0 - 4, &bar);
      tma_load(Lg, &M->liga36, x0 - 2, y0 - 2, &bar);
    }
  }
  load_case(&d, cs + t.c);
  const CaseDev& dg = cs[t.c];
  const double* mxs = met_slice<MS_PTC>(Ms, dg.mx, t.i0 - 2, dg.nx + 1);
  const double* mys = met_slice<MS_PTC>(Mt, dg.my, t.j0 - 2, dg.ny + 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    d.mx = mxs;
    d.my = mys;
  }
  if (!cta_wait(&bar, 0, &flag, err)) return;

  // P: pn = p + dtau*beta*RP at the interior cells of the tile, then bcP, then store
  using PS = PtFastT<LdShared<MS_PTC>>;
  const int nx = d.nx, ny = d.ny;
  double mp = 0.0;
  for (int q = threadIdx.x; q < NT * NT; q += blockDim.x) {
    const int a = q % NT, b = q / NT;
    const int i = t.i0 + a, j = t.j0 + b;
    if (i >= 2 && i <= nx - 1 && j >= 2 && j <= ny - 1) {
      double rr;
      const double inc = PS::p_incr_at(d, Un, Vn, BP, (4 + a) + (4 + b) * BP, i, j, &rr);
      P0[q] = P0[q] + inc;
      mp = nanmax(mp, fabs(rr));
    }
  }
  block_max_to(&ctl[t.c].res_p, mp);
  __syncthreads();
  // boundary passes only where a region holds boundary cells (i in {1,nx} or j in {1,ny}); the
  // test uses the largest region, the tile grown by two nodes
  const bool edge = !(t.i0 - 2 >= 2 && t.i0 + NT + 1 <= nx - 1 && t.j0 - 2 >= 2 && t.j0 + NT + 1 <= ny - 1);
  {
    if (edge) {
      const Win w{P0, t.i0, t.j0, NT, NT, NT};
      bc_cell_pass(d, w, 0, true, 0.0);
      __syncthreads();
      bc_cell_pass(d, w, 1, true, 0.0);
      __syncthreads();
    }
    double* pn = d.P[rp1];
    for (int q = threadIdx.x; q < NT * NT; q += blockDim.x) {
      const int a = q % NT, b = q / NT;
      const int i = t.i0 + a, j = t.j0 + b;
      if (i <= nx && j <= ny) pn[lin(i, j, d.pitch)] = P0[q];
    }
  }
  if (!scal) return;
  const ScalarSet T{Zt, d.T[rt_phys], S1t, S2t, d.T_in}, C{Zc, d.C[rc_phys], S1c, S2c, d.C_in};
  te_scalars(d, t, Un, Vn, Lg, T, C, d.T[rt_ntau], d.C[rc_ntau], edge);
}

}  // namespace

// The bcUV side effects of the first iteration after an upload: solve_U's boundary passes rewrite
// vm_tau's boundary, solve_V's rewrite um_tau's (boundary.f90:1-49); stage 1 has read both arrays
// as they were, stages 2 and 3 read them rewritten.  One block per case; cases whose tau arrays
// already satisfy the passes (CaseCtl::tau_dirty == 0) are left alone.
__global__ void k_te_tau_bc(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl) {
  const CaseCtl& k = ctl[blockIdx.x];
  if (!k.active || !k.tau_dirty) return;
  const CaseDev& d = cs[blockIdx.x];
  bc_uv_block(d, d.U[k.ru[R_TAU]], d.V[k.rv[R_TAU]]);
}

void te_launch_tau_bc(const CaseDev* cs, CaseCtl* ctl, int ncases, cudaStream_t s) {
  k_te_tau_bc<<<ncases, 256, 0, s>>>(cs, ctl);
}

cudaError_t te_prepare() {
  cudaError_t e = cudaFuncSetAttribute(k_te_uv<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_uv<1>());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_te_uv<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_uv<2>());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_te_uv<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_uv<3>());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_te_ptc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_PTC2);
  return e;
}

void te_launch_uv(int stage, const CaseDev* cs, CaseCtl* ctl, const Tile* tiles, int ntiles, const TeMaps* maps,
                  int* err, cudaStream_t s) {
  if (stage == 1) k_te_uv<1><<<ntiles, TE_THREADS, smem_uv<1>(), s>>>(cs, ctl, tiles, maps, err);
  else if (stage == 2) k_te_uv<2><<<ntiles, TE_THREADS, smem_uv<2>(), s>>>(cs, ctl, tiles, maps, err);
  else k_te_uv<3><<<ntiles, TE_THREADS, smem_uv<3>(), s>>>(cs, ctl, tiles, maps, err);
}

void te_launch_ptc(const CaseDev* cs, CaseCtl* ctl, const Tile* tiles, int ntiles, const TeMaps* maps, int* err,
                   cudaStream_t s) {
  k_te_ptc<<<ntiles, TE_THREADS, SMEM_PTC2, s>>>(cs, ctl, tiles, maps, err);
}

}  // namespace acs
