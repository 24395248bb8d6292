// solver.cu -- host orchestration and the C ABI (include/acs.h).
//
// A batch owns one device allocation holding, per case, the metric arrays, the porous fields and
// the rotating field buffers (see acs_dev.cuh), plus the case table, the control words and a
// tile table covering every case.  One pseudo-iteration is a fixed sequence of launches over the
// tile table (U stages, V stages, P, T stages, C stages, control).  acs_batch_run captures that
// sequence once as the body of a CUDA graph WHILE node whose condition kernel keeps looping
// while any case is active, so a whole multi-step run is one graph launch with no host round
// trip.  A single case (acs_handle) is a batch of one.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/acs.h"
#include "acs_dev.cuh"
#include "fast.h"
#include "engine_api.h"
#include "kernels.h"
#include "tile_engine.h"
#include "warmstart.h"

namespace acs {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CU(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) return fail(ACS_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {

constexpr int kMinN = 6;
constexpr long long kMaxStageBytes = 220 * 1024;  // dynamic shared memory for the staged engine
constexpr int kMaxN = 1 << 15;

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct FieldLoc { int family; int role; };  // family: 0 U, 1 V, 2 P, 3 T, 4 C
FieldLoc field_loc(int f) {
  switch (f) {
    case ACS_UM: return {0, R_PHYS};
    case ACS_UM_TAU: return {0, R_TAU};
    case ACS_UM_N_TAU: return {0, R_NTAU};
    case ACS_VM: return {1, R_PHYS};
    case ACS_VM_TAU: return {1, R_TAU};
    case ACS_VM_N_TAU: return {1, R_NTAU};
    case ACS_P: return {2, 0};
    case ACS_PN: return {2, 1};
    case ACS_T: return {3, R_PHYS};
    case ACS_T_TAU: return {3, R_TAU};
    case ACS_T_N_TAU: return {3, R_NTAU};
    case ACS_C: return {4, R_PHYS};
    case ACS_C_TAU: return {4, R_TAU};
    case ACS_C_N_TAU: return {4, R_NTAU};
  }
  return {-1, -1};
}

}  // namespace

struct Batch {
  int n = 0;
  std::vector<acs_params> prm;
  std::vector<CaseDev> hc;    // host copy of the case table
  std::vector<CaseCtl> hk;    // host copy of the control words
  std::vector<char> t_unity;  // T known to be identically 1 (the buoyancy term vanishes)
  char* pool = nullptr;
  size_t pool_bytes = 0;
  CaseDev* dc = nullptr;
  CaseCtl* dk = nullptr;
  Tile* dtiles = nullptr;
  int ntiles = 0;
  int* d_nactive = nullptr;
  long long* d_iter = nullptr;
  int* d_iters = nullptr;
  double* d_err = nullptr;
  long long stats_cap = 0;
  int* h_flag = nullptr;  // mapped host word for the host-polled loop
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  bool graph_conditional = true;
  bool use_fast = false;
  FastPlan* fast = nullptr;
  long long launches = 0;
  long long body_kernels = 0;
  int graph_steps = -1;  // n_steps the graph's loop bound was built for
  int engine = 0;        // 0 = persistent cluster engine, 1 = graph of per-stage kernels,
                         // 2 = graph of TMA-tiled kernels (tile_engine.cu)
  // tile engine: tile table, tensor maps, TMA timeout word (set up on first use)
  Tile* d_tetiles = nullptr;
  int n_tetiles = 0;
  TeMaps* d_temaps = nullptr;
  int* d_te_err = nullptr;
  int nodes_per_cta = 1536;
  int l1_loads = 1;      // FAST engine: load cluster-written arrays through L1
  int threads = 512;     // FAST engine: threads per CTA (256 or 512)
  int ctas_per_sm = 1;   // FAST engine with 256 threads: 1 or 2 resident CTAs per SM
  int staged = 1;        // FAST engine: stage stencil arrays in shared memory where they fit
  int last_staged = 0;   // the last engine launch used the staged kernel
  std::vector<int> cluster_override;  // per case: CTAs of its cluster (0 = from nodes_per_cta)
  int* d_cases = nullptr;
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> ev;
  // learned warm start (warmstart.cu): canvas size, per-case previous fields and increments
  int ws_H = 0, ws_W = 0;
  int ws_has_prev = 0;
  int ws_calls = 0;   // feature calls since acs_batch_ws_enable (3 give two increments)
  int ws_order = 1;   // ACS_OPT_EXTRAP_ORDER
  char* ws_pool = nullptr;
  WsCase* d_ws = nullptr;
  unsigned long long* d_ws_res = nullptr;
  int* d_ws_choice = nullptr;
  double* d_ws_ss = nullptr;  // per case and field: sum of inc^2, then the RMS of inc
  double* d_ws_sc = nullptr;

  ~Batch() {
    if (ws_pool) cudaFree(ws_pool);
    if (d_ws) cudaFree(d_ws);
    if (d_ws_res) cudaFree(d_ws_res);
    if (d_ws_choice) cudaFree(d_ws_choice);
    if (d_ws_ss) cudaFree(d_ws_ss);
    if (d_ws_sc) cudaFree(d_ws_sc);
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    if (fast) fast_destroy(fast);
    if (pool) cudaFree(pool);
    if (d_iters) cudaFree(d_iters);
    if (d_err) cudaFree(d_err);
    if (h_flag) cudaFreeHost(h_flag);
    if (d_cases) cudaFree(d_cases);
    if (d_tetiles) cudaFree(d_tetiles);
    if (d_temaps) cudaFree(d_temaps);
    if (d_te_err) cudaFree(d_te_err);
    for (auto s : side) cudaStreamDestroy(s);
    for (auto e : ev) cudaEventDestroy(e);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }

  double* buf(int c, int family, int idx) const {
    const CaseDev& d = hc[c];
    switch (family) {
      case 0: return d.U[idx];
      case 1: return d.V[idx];
      case 2: return d.P[idx];
      case 3: return d.T[idx];
      case 4: return d.C[idx];
    }
    return nullptr;
  }
  int role_index(int c, FieldLoc L) const {
    const CaseCtl& k = hk[c];
    if (L.role == R_NTAU && k.ntau_alias && (L.family <= 1 || hc[c].solve_scalars))
      L.role = k.ntau_alias == 1 ? R_PHYS : R_TAU;
    switch (L.family) {
      case 0: return k.ru[L.role];
      case 1: return k.rv[L.role];
      case 2: return L.role == 1 ? k.rp_read : k.rp[0];
      case 3: return k.rt[L.role];
      case 4: return k.rc[L.role];
    }
    return 0;
  }
};

// Checks of the parameter block that every entry point taking an acs_params shares (sizes are
// checked by the caller, whose limits differ).
int validate_params(const acs_params& p) {
  if (p.scheme != 0 && p.scheme != 1) return fail(ACS_E_ARG, "scheme must be 0 or 1");
  if (p.bc != 0 && p.bc != 1) return fail(ACS_E_ARG, "bc must be 0 or 1");
  if (p.arith != ACS_ARITH_EXACT && p.arith != ACS_ARITH_FAST) return fail(ACS_E_ARG, "arith must be 0 or 1");
  if (p.itc_max < 2) return fail(ACS_E_ARG, "itc_max must be at least 2");
  if (p.continuity != 0 && p.continuity != 1) return fail(ACS_E_ARG, "continuity must be 0 or 1");
  if (!(p.Re > 0) || !(p.Pe > 0) || !(p.Sc > 0) || !(p.Da > 0)) return fail(ACS_E_ARG, "Re, Pe, Sc, Da must be positive");
  return ACS_OK;
}

namespace {

int validate(const acs_grid& g, const acs_params& p) {
  if (!g.x || !g.y || !g.xm || !g.ym || !g.epsilon1 || !g.liga_poros) return fail(ACS_E_ARG, "null grid array");
  if (g.imax != p.imax || g.jmax != p.jmax) return fail(ACS_E_ARG, "grid and params disagree on imax/jmax");
  if (p.imax < kMinN || p.jmax < kMinN || p.imax > kMaxN || p.jmax > kMaxN)
    return fail(ACS_E_SIZE, "imax and jmax must lie in [6, 32768]");
  return validate_params(p);
}

// Binary porous structure (eps, liga) in {(1,0), (phi,1)} for one phi.
bool binary_porosity(const acs_grid& g, double* phi) {
  const size_t nc = (size_t)g.imax * g.jmax;
  double ph = -1.0;
  for (size_t q = 0; q < nc; ++q) {
    const double e = g.epsilon1[q], l = g.liga_poros[q];
    if (l == 0.0) {
      if (e != 1.0) return false;
    } else if (l == 1.0) {
      if (ph < 0.0) ph = e;
      if (e != ph || !(e > 0.0)) return false;
    } else {
      return false;
    }
  }
  *phi = ph < 0.0 ? 1.0 : ph;
  return true;
}

int push_ctl(Batch& b);

int field_dims(const CaseDev& d, int family, int* w, int* h) {
  *w = family == 0 ? d.nx + 1 : d.nx;
  *h = family == 1 ? d.ny + 1 : d.ny;
  return 0;
}

int put(Batch& b, int c, int family, int idx, const double* host) {
  const CaseDev& d = b.hc[c];
  int w, h;
  field_dims(d, family, &w, &h);
  CU(cudaMemcpy2DAsync(b.buf(c, family, idx), (size_t)d.pitch * 8, host, (size_t)w * 8, (size_t)w * 8, h,
                       cudaMemcpyHostToDevice, b.stream));
  return ACS_OK;
}

int get(Batch& b, int c, int family, int idx, double* host) {
  const CaseDev& d = b.hc[c];
  int w, h;
  field_dims(d, family, &w, &h);
  CU(cudaMemcpy2DAsync(host, (size_t)w * 8, b.buf(c, family, idx), (size_t)d.pitch * 8, (size_t)w * 8, h,
                       cudaMemcpyDeviceToHost, b.stream));
  return ACS_OK;
}

bool all_ones(const double* a, size_t n) {
  for (size_t q = 0; q < n; ++q)
    if (a[q] != 1.0) return false;
  return true;
}

int upload_field(Batch& b, int c, int field, const double* host) {
  FieldLoc L = field_loc(field);
  if (L.family < 0) return fail(ACS_E_ARG, "unknown field id");
  if (field == ACS_UM_TAU || field == ACS_VM_TAU) {
    b.hk[c].tau_dirty = 1;
    int r = push_ctl(b);
    if (r) return r;
  }
  if (L.role == R_NTAU && L.family != 2 && b.hk[c].ntau_alias) {
    // give every n_tau array its own values again before one of them is overwritten
    CaseCtl& k = b.hk[c];
    const CaseDev& d = b.hc[c];
    const int nfam = d.solve_scalars ? 4 : 2;
    const int fams[4] = {0, 1, 3, 4};
    for (int q = 0; q < nfam; ++q) {
      const int f = fams[q];
      const int src = b.role_index(c, FieldLoc{f, R_NTAU});
      const int* roles = f == 0 ? k.ru : f == 1 ? k.rv : f == 3 ? k.rt : k.rc;
      CU(cudaMemcpyAsync(b.buf(c, f, roles[R_NTAU]), b.buf(c, f, src), sizeof(double) * d.n_elems,
                         cudaMemcpyDeviceToDevice, b.stream));
    }
    k.ntau_alias = 0;
    int r = push_ctl(b);
    if (r) return r;
  }
  if (L.family == 2) {
    // p and pn share one buffer after a non-exit iteration; give pn its own buffer first
    CaseCtl& k = b.hk[c];
    if (k.rp_read == k.rp[0]) {
      const CaseDev& d = b.hc[c];
      CU(cudaMemcpyAsync(d.P[k.rp[1]], d.P[k.rp[0]], sizeof(double) * d.n_elems, cudaMemcpyDeviceToDevice, b.stream));
      k.rp_read = k.rp[1];
      int r = push_ctl(b);
      if (r) return r;
    }
  }
  if (field == ACS_T) b.t_unity[c] = all_ones(host, (size_t)b.hc[c].nx * b.hc[c].ny);
  return put(b, c, L.family, b.role_index(c, L), host);
}

int download_field(Batch& b, int c, int field, double* host) {
  FieldLoc L = field_loc(field);
  if (L.family < 0) return fail(ACS_E_ARG, "unknown field id");
  int r = get(b, c, L.family, b.role_index(c, L), host);
  if (r) return r;
  CU(cudaStreamSynchronize(b.stream));
  return ACS_OK;
}

int refresh_flags(Batch& b) {
  for (int c = 0; c < b.n; ++c) {
    CaseDev& d = b.hc[c];
    const acs_params& p = b.prm[c];
    int f = d.flags & ~F_BUOY;
    if (p.InvFr2 != 0.0 && (p.solve_scalars || !b.t_unity[c])) f |= F_BUOY;
    if (f != d.flags) {
      d.flags = f;
      CU(cudaMemcpyAsync(b.dc + c, &d, sizeof(CaseDev), cudaMemcpyHostToDevice, b.stream));
    }
  }
  return ACS_OK;
}

int push_ctl(Batch& b) {
  CU(cudaMemcpyAsync(b.dk, b.hk.data(), sizeof(CaseCtl) * b.n, cudaMemcpyHostToDevice, b.stream));
  return ACS_OK;
}
int pull_ctl(Batch& b) {
  CU(cudaMemcpyAsync(b.hk.data(), b.dk, sizeof(CaseCtl) * b.n, cudaMemcpyDeviceToHost, b.stream));
  CU(cudaStreamSynchronize(b.stream));
  return ACS_OK;
}

void reset_roles(CaseCtl& k) {
  for (int r = 0; r < 3; ++r) k.ru[r] = k.rv[r] = k.rt[r] = k.rc[r] = r;
  k.rp[0] = 0;
  k.rp[1] = 1;
  k.rp_read = 1;
  k.ntau_alias = 0;
  k.tau_dirty = 1;
}

// Grid arrays may be host or device pointers (acs_mesh_channel_device writes device arrays): a
// grid with any array in device memory is copied to host storage before the pool is built.
int host_grids(const acs_grid* grids, int n, std::vector<acs_grid>& hg, std::vector<std::vector<double>>& store) {
  hg.assign(grids, grids + n);
  for (int c = 0; c < n; ++c) {
    acs_grid& g = hg[c];
    const double** arr[6] = {&g.x, &g.y, &g.xm, &g.ym, &g.epsilon1, &g.liga_poros};
    const size_t len[6] = {(size_t)g.imax, (size_t)g.jmax, (size_t)g.imax + 1, (size_t)g.jmax + 1,
                           (size_t)g.imax * g.jmax, (size_t)g.imax * g.jmax};
    for (int k = 0; k < 6; ++k) {
      cudaPointerAttributes a{};
      if (cudaPointerGetAttributes(&a, *arr[k]) != cudaSuccess) {
        cudaGetLastError();
        continue;  // not known to CUDA: host memory
      }
      if (a.type != cudaMemoryTypeDevice) continue;
      store.emplace_back(len[k]);
      if (cudaMemcpy(store.back().data(), *arr[k], sizeof(double) * len[k], cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(ACS_E_CUDA, "copying a device grid array");
      *arr[k] = store.back().data();
    }
  }
  return ACS_OK;
}

int create_batch(const acs_grid* grids_in, const acs_params* params, int n, Batch** out) {
  if (!grids_in || !params || n <= 0 || !out) return fail(ACS_E_ARG, "null argument or n <= 0");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(ACS_E_CUDA, "no CUDA device");
  for (int c = 0; c < n; ++c) {
    int r = validate(grids_in[c], params[c]);
    if (r) return r;
  }
  std::vector<acs_grid> hg;
  std::vector<std::vector<double>> grid_store;
  if (int r = host_grids(grids_in, n, hg, grid_store)) return r;
  const acs_grid* grids = hg.data();
  const bool fast = params[0].arith == ACS_ARITH_FAST;
  for (int c = 1; c < n; ++c)
    if ((params[c].arith == ACS_ARITH_FAST) != fast) return fail(ACS_E_ARG, "all cases of a batch must use one arith mode");

  // Layout of the pool: [case table][control][tiles][counters] then per case
  // [metrics][eps][liga][mask][U x3][V x3][P x2][T x3][C x3][S x4].
  std::vector<size_t> off(n);
  std::vector<size_t> sizes(n);
  size_t total = 0;
  for (int c = 0; c < n; ++c) {
    const int nx = params[c].imax, ny = params[c].jmax;
    const size_t ne = align_up(nx + 1, 4) * (size_t)(ny + 1);
    size_t sz = align_up(sizeof(double) * (2 * nx + 2 * ny + 6), 256) + 2 * align_up(8 * ne, 256) +
                align_up(ne, 256) + 22 * align_up(8 * ne, 256);
    off[c] = total;
    sizes[c] = sz;
    total += align_up(sz, 256);
  }
  std::vector<Tile> tiles;
  for (int c = 0; c < n; ++c)
    for (int j0 = 1; j0 <= params[c].jmax + 1; j0 += TILE_Y)
      for (int i0 = 1; i0 <= params[c].imax + 1; i0 += TILE_X) tiles.push_back({c, i0, j0, 0});
  const size_t a_case = align_up(sizeof(CaseDev) * n, 256);
  const size_t a_ctl = align_up(sizeof(CaseCtl) * n, 256);
  const size_t a_tile = align_up(sizeof(Tile) * tiles.size(), 256);
  const size_t head = a_case + a_ctl + a_tile + 256;

  Batch* b = new Batch();
  b->n = n;
  b->prm.assign(params, params + n);
  b->hc.resize(n);
  b->hk.assign(n, CaseCtl{});
  b->t_unity.assign(n, 0);
  b->use_fast = fast;
  b->pool_bytes = head + total;
  cudaError_t e = cudaMalloc(&b->pool, b->pool_bytes);
  if (e != cudaSuccess) {
    delete b;
    return fail(ACS_E_NOMEM, std::string("cudaMalloc of the case pool: ") + cudaGetErrorString(e));
  }
  e = cudaMemset(b->pool, 0, b->pool_bytes);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete b;
    return fail(ACS_E_CUDA, std::string("batch set-up: ") + cudaGetErrorString(e));
  }
  b->own_stream = true;
  char* p = b->pool;
  b->dc = (CaseDev*)p;
  b->dk = (CaseCtl*)(p + a_case);
  b->dtiles = (Tile*)(p + a_case + a_ctl);
  b->d_nactive = (int*)(p + a_case + a_ctl + a_tile);
  b->d_iter = (long long*)(p + a_case + a_ctl + a_tile + 64);
  b->ntiles = (int)tiles.size();
  char* base = p + head;
  std::vector<double> stage;
  for (int c = 0; c < n; ++c) {
    const acs_grid& g = grids[c];
    const acs_params& pr = params[c];
    const int nx = pr.imax, ny = pr.jmax;
    const int pitch = (int)align_up(nx + 1, 4);
    const size_t ne = (size_t)pitch * (ny + 1);
    char* q = base + off[c];
    CaseDev& d = b->hc[c];
    std::memset(&d, 0, sizeof(d));
    d.nx = nx; d.ny = ny; d.pitch = pitch;
    d.scheme = pr.scheme; d.bc = pr.bc; d.solve_scalars = pr.solve_scalars; d.itc_max = pr.itc_max;
    d.continuity = pr.continuity;
    d.Re = pr.Re; d.Pe = pr.Pe; d.Sc = pr.Sc; d.Da = pr.Da; d.Cf = pr.Cf; d.g = pr.g;
    d.InvFr2 = pr.InvFr2; d.v_in = pr.v_in; d.T_in = pr.T_in; d.C_in = pr.C_in; d.b_art = pr.b_art;
    d.beta = pr.beta; d.dt = pr.dt; d.dtau = pr.dtau; d.eps = pr.eps;
    d.n_elems = (long long)ne;
    stage.assign(2 * nx + 2 * ny + 6, 0.0);
    double* X = stage.data();
    double* Y = X + (nx + 1);
    double* XM = Y + (ny + 1);
    double* YM = XM + (nx + 2);
    for (int i = 1; i <= nx; ++i) X[i] = g.x[i - 1];
    for (int j = 1; j <= ny; ++j) Y[j] = g.y[j - 1];
    for (int i = 1; i <= nx + 1; ++i) XM[i] = g.xm[i - 1];
    for (int j = 1; j <= ny + 1; ++j) YM[j] = g.ym[j - 1];
    double* dm = (double*)q;
    d.x = dm; d.y = dm + (nx + 1); d.xm = d.y + (ny + 1); d.ym = d.xm + (nx + 2);
    CU(cudaMemcpy(dm, stage.data(), sizeof(double) * stage.size(), cudaMemcpyHostToDevice));
    q += align_up(sizeof(double) * (2 * nx + 2 * ny + 6), 256);
    double* deps = (double*)q; q += align_up(8 * ne, 256);
    double* dliga = (double*)q; q += align_up(8 * ne, 256);
    uint8_t* dmask = (uint8_t*)q; q += align_up(ne, 256);
    std::vector<double> pe(ne, 1.0), pl(ne, 0.0);
    std::vector<uint8_t> pm(ne, 0);
    bool porous = false;
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const size_t s = (size_t)(i - 1) + (size_t)(j - 1) * nx;
        const size_t t = (size_t)lin(i, j, pitch);
        pe[t] = g.epsilon1[s];
        pl[t] = g.liga_poros[s];
        pm[t] = g.liga_poros[s] != 0.0;
        porous |= g.liga_poros[s] != 0.0;
      }
    CU(cudaMemcpy(deps, pe.data(), 8 * ne, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(dliga, pl.data(), 8 * ne, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(dmask, pm.data(), ne, cudaMemcpyHostToDevice));
    d.epsf = deps; d.liga = dliga; d.mask = dmask;
    double phi = 1.0;
    if (binary_porosity(g, &phi)) d.flags |= F_BINARY;
    d.phi = phi;
    if (pr.b_art != 0.0) d.flags |= F_BART;
    if (porous) d.flags |= F_POROUS;
    if (pr.InvFr2 != 0.0 && pr.solve_scalars) d.flags |= F_BUOY;
    double** bufs[5] = {d.U, d.V, d.P, d.T, d.C};
    const int counts[5] = {3, 3, 2, 3, 3};
    for (int f = 0; f < 5; ++f)
      for (int r = 0; r < counts[f]; ++r) {
        bufs[f][r] = (double*)q;
        q += align_up(8 * ne, 256);
      }
    for (int r = 0; r < 4; ++r) { d.S[r] = (double*)q; q += align_up(8 * ne, 256); }
    for (int r = 0; r < 4; ++r) { d.S2[r] = (double*)q; q += align_up(8 * ne, 256); }
    reset_roles(b->hk[c]);
  }
  if (fast) {
    int r = fast_create(b->hc, grids, params, &b->fast);
    if (r) {
      delete b;
      return r;
    }
  }
  e = cudaMemcpy(b->dc, b->hc.data(), sizeof(CaseDev) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->dk, b->hk.data(), sizeof(CaseCtl) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->dtiles, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    delete b;
    return fail(ACS_E_CUDA, std::string("batch upload: ") + cudaGetErrorString(e));
  }
  *out = b;
  return ACS_OK;
}

// ---- launch sequences --------------------------------------------------------------------------
// solve_U: three stages, each followed by bcUV(stage array, vm_tau) (equations.f90:259-296)
void seq_u(Batch& b) {
  for (int s = 1; s <= 3; ++s) {
    (b.use_fast ? launch_u_stage_fast : launch_u_stage_exact)(s, b.dc, b.dk, b.dtiles, b.ntiles, b.stream);
    launch_bc_uv(b.dc, b.dk, b.n, s - 1, b.stream);
  }
  b.launches += 6;
}

// solve_V: three stages, each followed by bcUV(um_tau, stage array) (equations.f90:561-598)
void seq_v(Batch& b) {
  for (int s = 1; s <= 3; ++s) {
    (b.use_fast ? launch_v_stage_fast : launch_v_stage_exact)(s, b.dc, b.dk, b.dtiles, b.ntiles, b.stream);
    launch_bc_uv(b.dc, b.dk, b.n, 3 + s - 1, b.stream);
  }
  b.launches += 6;
}

// solve_P: the stages fuse pointwise; the intermediate bcP(pi) never reaches the interior
void seq_p(Batch& b) {
  (b.use_fast ? launch_p_fast : launch_p_exact)(b.dc, b.dk, b.dtiles, b.ntiles, b.stream);
  launch_bc_cell(b.dc, b.dk, b.n, 0, b.stream);
  b.launches += 2;
}

// solve_Z / solve_C: three stages, each followed by bcZ / bcC
void seq_s(Batch& b, bool is_c) {
  const int w0 = is_c ? 4 : 1;
  for (int s = 1; s <= 3; ++s) {
    (b.use_fast ? launch_s_stage_fast : launch_s_stage_exact)(is_c, s, b.dc, b.dk, b.dtiles, b.ntiles, b.stream);
    launch_bc_cell(b.dc, b.dk, b.n, w0 + s - 1, b.stream);
  }
  b.launches += 6;
}

// one launch of the timed kernel (acs_batch_time_kernel)
void launch_timed_kernel(Batch& b, int kernel) {
  switch (kernel) {
    case 0: (b.use_fast ? launch_u_stage_fast : launch_u_stage_exact)(1, b.dc, b.dk, b.dtiles, b.ntiles, b.stream); break;
    case 1: (b.use_fast ? launch_v_stage_fast : launch_v_stage_exact)(1, b.dc, b.dk, b.dtiles, b.ntiles, b.stream); break;
    case 2: (b.use_fast ? launch_p_fast : launch_p_exact)(b.dc, b.dk, b.dtiles, b.ntiles, b.stream); break;
    case 3: (b.use_fast ? launch_s_stage_fast : launch_s_stage_exact)(false, 1, b.dc, b.dk, b.dtiles, b.ntiles, b.stream); break;
    case 4: (b.use_fast ? launch_s_stage_fast : launch_s_stage_exact)(true, 1, b.dc, b.dk, b.dtiles, b.ntiles, b.stream); break;
    case 5: te_launch_uv(2, b.dc, b.dk, b.d_tetiles, b.n_tetiles, b.d_temaps, b.d_te_err, b.stream); break;
    case 6: te_launch_ptc(b.dc, b.dk, b.d_tetiles, b.n_tetiles, b.d_temaps, b.d_te_err, b.stream); break;
  }
}

bool any_scalars(const Batch& b) {
  for (auto& p : b.prm)
    if (p.solve_scalars) return true;
  return false;
}

// Tile engine set-up: tile table over every case, a tensor map per case buffer and box size.
int te_setup(Batch& b) {
  if (b.d_temaps) return ACS_OK;
  if (!b.use_fast) return fail(ACS_E_UNSUPPORTED, "the tile engine computes in the FAST arithmetic only");
  std::vector<Tile> tiles;
  for (int c = 0; c < b.n; ++c) te_case_tiles(c, b.hc[c].pitch, b.hc[c].ny, tiles);
  std::vector<TeMaps> maps(b.n);
  const int er = te_encode_maps(b.hc, maps.data());
  if (er) return fail(ACS_E_CUDA, er == 1 ? "cuTensorMapEncodeTiled is not available from the driver"
                                           : "cuTensorMapEncodeTiled rejected a case buffer");
  CU(te_prepare());
  CU(cudaMalloc(&b.d_tetiles, sizeof(Tile) * tiles.size()));
  CU(cudaMalloc(&b.d_temaps, sizeof(TeMaps) * b.n));
  CU(cudaMalloc(&b.d_te_err, sizeof(int)));
  CU(cudaMemcpy(b.d_tetiles, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(b.d_temaps, maps.data(), sizeof(TeMaps) * b.n, cudaMemcpyHostToDevice));
  CU(cudaMemset(b.d_te_err, 0, sizeof(int)));
  b.n_tetiles = (int)tiles.size();
  return ACS_OK;
}

// one pseudo-iteration of the tile engine: U/V stages 1-3, P + T/C, control
void te_iteration(Batch& b) {
  for (int s = 1; s <= 3; ++s) {
    te_launch_uv(s, b.dc, b.dk, b.d_tetiles, b.n_tetiles, b.d_temaps, b.d_te_err, b.stream);
    if (s == 1) te_launch_tau_bc(b.dc, b.dk, b.n, b.stream);
  }
  te_launch_ptc(b.dc, b.dk, b.d_tetiles, b.n_tetiles, b.d_temaps, b.d_te_err, b.stream);
  k_control<<<b.n, 256, 0, b.stream>>>(b.dc, b.dk, b.d_iters, b.d_err, b.d_nactive);
  b.launches += 6;
}

// one pseudo-iteration (main.f90:122-150) for every active case
void seq_iteration(Batch& b) {
  seq_u(b);
  seq_v(b);
  seq_p(b);
  if (any_scalars(b)) {
    seq_s(b, false);
    seq_s(b, true);
  }
  k_control<<<b.n, 256, 0, b.stream>>>(b.dc, b.dk, b.d_iters, b.d_err, b.d_nactive);
  b.launches += 1;
}

long long max_total_iterations(const Batch& b, int n_steps) {
  long long m = 0;
  for (auto& p : b.prm) m = std::max(m, (long long)p.itc_max * (long long)n_steps);
  return m + 2;
}

int build_graph(Batch& b, int n_steps) {
  if (b.gexec) { cudaGraphExecDestroy(b.gexec); b.gexec = nullptr; }
  if (b.graph) { cudaGraphDestroy(b.graph); b.graph = nullptr; }
  const long long saved = b.launches;
  // ACS_NO_CONDITIONAL_GRAPH=1 selects the host-polled loop below (profilers cannot look inside
  // a graph that holds conditional nodes)
  if (getenv("ACS_NO_CONDITIONAL_GRAPH")) b.graph_conditional = false;
  if (b.graph_conditional) {
    cudaGraph_t g;
    CU(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNode_t node;
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
    if (e == cudaSuccess) {
      cudaGraph_t body = np.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(b.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        const long long l0 = b.launches;
        if (b.engine == 2) te_iteration(b);
        else seq_iteration(b);
        k_loop_cond<<<1, 1, 0, b.stream>>>(b.d_nactive, b.d_iter, max_total_iterations(b, n_steps), h);
        b.body_kernels = b.launches - l0 + 1;
        e = cudaStreamEndCapture(b.stream, &body);
      }
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b.gexec, g, 0);
    if (e == cudaSuccess) {
      b.graph = g;
      b.launches = saved;
      return ACS_OK;
    }
    cudaGetLastError();
    cudaGraphDestroy(g);
    b.graph_conditional = false;  // fall back to the host-polled loop below
  }
  // host-polled: the graph holds one iteration plus a flag publish
  if (!b.h_flag) CU(cudaHostAlloc(&b.h_flag, sizeof(int), cudaHostAllocMapped));
  int* d_flag = nullptr;
  CU(cudaHostGetDevicePointer(&d_flag, b.h_flag, 0));
  cudaGraph_t g;
  CU(cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal));
  const long long l0 = b.launches;
  if (b.engine == 2) te_iteration(b);
  else seq_iteration(b);
  k_loop_flag<<<1, 1, 0, b.stream>>>(b.d_nactive, b.d_iter, d_flag);
  b.body_kernels = b.launches - l0 + 1;
  CU(cudaStreamEndCapture(b.stream, &g));
  CU(cudaGraphInstantiate(&b.gexec, g, 0));
  b.graph = g;
  b.launches = saved;
  return ACS_OK;
}

int run_engine(Batch& b);
int run_graph(Batch& b, int n_steps);

int run_batch(Batch& b, int n_steps, int* itc, int* iters, double* err, int* status) {
  if (n_steps <= 0) return fail(ACS_E_ARG, "n_steps must be positive");
  int r = refresh_flags(b);
  if (r) return r;
  const long long need = (long long)b.n * n_steps;
  if (need > b.stats_cap) {
    if (b.d_iters) cudaFree(b.d_iters);
    if (b.d_err) cudaFree(b.d_err);
    b.d_iters = nullptr;
    b.d_err = nullptr;
    CU(cudaMalloc(&b.d_iters, sizeof(int) * need));
    CU(cudaMalloc(&b.d_err, sizeof(double) * need));
    b.stats_cap = need;
    if (b.gexec) { cudaGraphExecDestroy(b.gexec); b.gexec = nullptr; }
    if (b.graph) { cudaGraphDestroy(b.graph); b.graph = nullptr; }
  }
  for (int c = 0; c < b.n; ++c) {
    CaseCtl& k = b.hk[c];
    k.itc = itc ? itc[c] : 1;
    k.step = 0;
    k.n_steps = n_steps;
    k.k = 0;
    k.active = 1;
    k.status = 0;
    k.copy_phys = 0;
    k.res_u = k.res_v = k.res_p = 0;
    k.total_iters = 0;
    k.scalars = b.prm[c].solve_scalars ? 1 : 0;
  }
  r = push_ctl(b);
  if (r) return r;
  CU(cudaMemsetAsync(b.d_nactive, 0, 256, b.stream));
  if (b.engine == 0) {
    r = run_engine(b);
    if (r) return r;
  } else {
    r = run_graph(b, n_steps);
    if (r) return r;
  }
  r = pull_ctl(b);
  if (r) return r;
  if (iters) CU(cudaMemcpy(iters, b.d_iters, sizeof(int) * need, cudaMemcpyDeviceToHost));
  if (err) CU(cudaMemcpy(err, b.d_err, sizeof(double) * need, cudaMemcpyDeviceToHost));
  bool failed = false;
  for (int c = 0; c < b.n; ++c) {
    if (itc) itc[c] = b.hk[c].itc;
    if (status) status[c] = b.hk[c].status;
    failed |= b.hk[c].status == ACS_CASE_FAILED;
    b.hk[c].active = 0;
  }
  CU(cudaMemsetAsync(b.d_iter, 0, sizeof(long long), b.stream));
  r = push_ctl(b);
  if (r) return r;
  CU(cudaStreamSynchronize(b.stream));
  if (failed) return fail(ACS_E_STATE, "a case failed: NaN or infinite residual");
  return ACS_OK;
}

int run_graph(Batch& b, int n_steps) {
  int r;
  if (b.engine == 2) {
    r = te_setup(b);
    if (r) return r;
  }
  // the graph bakes in the loop bound; rebuild when n_steps changes the bound
  if (!b.gexec || b.graph_steps != n_steps) {
    r = build_graph(b, n_steps);
    if (r) return r;
    b.graph_steps = n_steps;
  }
  if (b.graph_conditional) {
    CU(cudaGraphLaunch(b.gexec, b.stream));
    CU(cudaStreamSynchronize(b.stream));
  } else {
    const long long cap = max_total_iterations(b, n_steps);
    for (long long it = 0; it < cap; ++it) {
      CU(cudaGraphLaunch(b.gexec, b.stream));
      if ((it & 15) == 15) {
        CU(cudaStreamSynchronize(b.stream));
        if (*(volatile int*)b.h_flag == 0) break;
      }
    }
    CU(cudaStreamSynchronize(b.stream));
  }
  long long iters_done = 0;
  CU(cudaMemcpy(&iters_done, b.d_iter, sizeof(long long), cudaMemcpyDeviceToHost));
  b.launches = iters_done * b.body_kernels;
  if (b.engine == 2) {
    int te_err = 0;
    CU(cudaMemcpy(&te_err, b.d_te_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (te_err) return fail(ACS_E_CUDA, "tile engine: a TMA wait timed out (the results of this run are not valid)");
  }
  return ACS_OK;
}

// Cluster size for a case: about nodes_per_cta nodes per CTA, at most 16 CTAs, strips of at
// least 4 node rows.
int cluster_size(const Batch& b, int c) {
  const CaseDev& d = b.hc[c];
  const long long nodes = (long long)(d.nx + 1) * (d.ny + 1);
  int K = (int)((nodes + b.nodes_per_cta - 1) / b.nodes_per_cta);
  if (c < (int)b.cluster_override.size() && b.cluster_override[c] > 0) K = b.cluster_override[c];
  K = std::max(1, std::min(K, 16));
  K = std::min(K, std::max(1, (d.ny + 1) / 4));
  return K;
}

// One launch per cluster size, each on its own stream so the size classes run side by side.
int run_engine(Batch& b) {
  std::vector<std::vector<int>> groups(17);
  for (int c = 0; c < b.n; ++c) groups[cluster_size(b, c)].push_back(c);
  if (!b.d_cases) CU(cudaMalloc(&b.d_cases, sizeof(int) * b.n));
  std::vector<int> order;
  std::vector<std::pair<int, int>> launches;  // (K, offset)
  for (int K = 16; K >= 1; --K) {
    if (groups[K].empty()) continue;
    launches.push_back({K, (int)order.size()});
    order.insert(order.end(), groups[K].begin(), groups[K].end());
  }
  CU(cudaMemcpyAsync(b.d_cases, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice, b.stream));
  for (int c = 0; c < b.n; ++c) {
    std::memset(b.hk[c].slot, 0, sizeof(b.hk[c].slot));
  }
  int r = push_ctl(b);
  if (r) return r;
  while (b.side.size() < launches.size()) {
    cudaStream_t s;
    CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    b.side.push_back(s);
    cudaEvent_t e;
    CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b.ev.push_back(e);
  }
  cudaEvent_t fork;
  CU(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  CU(cudaEventRecord(fork, b.stream));
  b.launches = 0;
  for (size_t g = 0; g < launches.size(); ++g) {
    const int K = launches[g].first;
    const int off = launches[g].second;
    const int cnt = (int)groups[K].size();
    cudaStream_t s = g == 0 ? b.stream : b.side[g];
    if (g) CU(cudaStreamWaitEvent(s, fork, 0));
    // staging slot: the largest strip of the size class plus two halo rows on each side
    long long slot = 0;
    for (int q = 0; q < cnt; ++q) {
      const CaseDev& d = b.hc[order[off + q]];
      const long long rows = (d.ny + 1 + K - 1) / K + 4;
      slot = std::max(slot, (rows * d.pitch + 1) / 2 * 2);
    }
    const bool stg = b.use_fast && b.staged && b.ctas_per_sm == 1 &&
                     (long long)STAGE_SLOTS * slot * 8 <= kMaxStageBytes;
    EngineArgs a{b.dc, b.dk, b.d_cases + off, b.d_iters, b.d_err, stg ? (int)slot : 0};
    cudaError_t e = b.use_fast ? launch_engine_fast(a, K, cnt, s, b.l1_loads, b.threads, b.ctas_per_sm, stg ? 1 : 0)
                               : launch_engine_exact(a, K, cnt, s);
    b.last_staged = stg ? 1 : 0;
    if (e != cudaSuccess) {
      cudaEventDestroy(fork);
      return fail(ACS_E_CUDA, std::string("engine launch (cluster ") + std::to_string(K) + "): " + cudaGetErrorString(e));
    }
    b.launches += 1;
    if (g) {
      CU(cudaEventRecord(b.ev[g], s));
      CU(cudaStreamWaitEvent(b.stream, b.ev[g], 0));
    }
  }
  cudaEventDestroy(fork);
  CU(cudaStreamSynchronize(b.stream));
  CU(cudaGetLastError());
  return ACS_OK;
}

// Per-routine calls run one routine's launches on case 0 with identity roles.
int begin_routine(Batch& b) {
  CaseCtl& k = b.hk[0];
  reset_roles(k);
  k.active = 1;
  k.scalars = 1;
  k.res_u = k.res_v = k.res_p = 0;
  return push_ctl(b);
}

int end_routine(Batch& b) {
  CU(cudaStreamSynchronize(b.stream));
  CU(cudaGetLastError());
  int r = pull_ctl(b);
  b.hk[0].active = 0;
  if (!r) r = push_ctl(b);
  if (!r) CU(cudaStreamSynchronize(b.stream));
  return r;
}

double bits_to_double(unsigned long long v) {
  double d;
  std::memcpy(&d, &v, 8);
  return d;
}

}  // namespace
}  // namespace acs

using acs::Batch;
using acs::fail;

struct acs_batch { Batch* b; };
struct acs_handle { Batch* b; };

extern "C" {

const char* acs_last_error(void) { return acs::g_err.c_str(); }
const char* acs_version(void) { return "acs-b200 1.0 (sm_100a, FP64)"; }

int acs_device_count(int* n) {
  if (!n) return acs::fail(ACS_E_ARG, "null");
  if (cudaGetDeviceCount(n) != cudaSuccess) {
    *n = 0;
    cudaGetLastError();
  }
  return ACS_OK;
}

int acs_batch_create(const acs_grid* grids, const acs_params* params, int n_cases, acs_batch** out) {
  if (!out) return acs::fail(ACS_E_ARG, "null out");
  Batch* b = nullptr;
  int r = acs::create_batch(grids, params, n_cases, &b);
  if (r) return r;
  *out = new acs_batch{b};
  return ACS_OK;
}

int acs_batch_destroy(acs_batch* h) {
  if (!h) return ACS_OK;
  delete h->b;
  delete h;
  return ACS_OK;
}

int acs_batch_set_stream(acs_batch* h, void* s) {
  if (!h) return acs::fail(ACS_E_ARG, "null handle");
  Batch& b = *h->b;
  if (b.gexec) { cudaGraphExecDestroy(b.gexec); b.gexec = nullptr; }
  if (b.graph) { cudaGraphDestroy(b.graph); b.graph = nullptr; }
  if (s) {
    if (b.own_stream) cudaStreamDestroy(b.stream);
    b.stream = (cudaStream_t)s;
    b.own_stream = false;
  }
  return ACS_OK;
}

int acs_batch_set_field(acs_batch* h, int c, int field, const double* host) {
  if (!h || !host) return acs::fail(ACS_E_ARG, "null argument");
  if (c < 0 || c >= h->b->n) return acs::fail(ACS_E_ARG, "case id out of range");
  return acs::upload_field(*h->b, c, field, host);
}

int acs_batch_get_field(acs_batch* h, int c, int field, double* host) {
  if (!h || !host) return acs::fail(ACS_E_ARG, "null argument");
  if (c < 0 || c >= h->b->n) return acs::fail(ACS_E_ARG, "case id out of range");
  return acs::download_field(*h->b, c, field, host);
}

int acs_batch_cell_fields(acs_batch* h, int c, double* u, double* v, double* vel_mag) {
  if (!h || !u || !v || !vel_mag) return acs::fail(ACS_E_ARG, "null argument");
  Batch& b = *h->b;
  if (c < 0 || c >= b.n) return acs::fail(ACS_E_ARG, "case id out of range");
  const acs::CaseDev& d = b.hc[c];
  // the results go through the T/C stage scratch of the cluster engine, which no step keeps
  double* out[3] = {d.S2[0], d.S2[1], d.S2[2]};
  CU(acs::launch_cell_fields(b.buf(c, 0, b.role_index(c, acs::FieldLoc{0, acs::R_PHYS})),
                             b.buf(c, 1, b.role_index(c, acs::FieldLoc{1, acs::R_PHYS})), d.nx, d.ny, d.pitch,
                             out[0], out[1], out[2], b.stream));
  double* host[3] = {u, v, vel_mag};
  for (int f = 0; f < 3; ++f)
    CU(cudaMemcpy2DAsync(host[f], (size_t)d.nx * 8, out[f], (size_t)d.pitch * 8, (size_t)d.nx * 8, d.ny,
                         cudaMemcpyDeviceToHost, b.stream));
  CU(cudaStreamSynchronize(b.stream));
  return ACS_OK;
}

int acs_batch_run(acs_batch* h, int n_steps, int* itc, int* iters, double* err, int* status) {
  if (!h) return acs::fail(ACS_E_ARG, "null handle");
  return acs::run_batch(*h->b, n_steps, itc, iters, err, status);
}

int acs_batch_ws_enable(acs_batch* h, int H, int W) {
  if (!h) return acs::fail(ACS_E_ARG, "null handle");
  Batch& b = *h->b;
  for (int c = 0; c < b.n; ++c)
    if (b.hc[c].nx + 1 > W || b.hc[c].ny + 1 > H) return acs::fail(ACS_E_SIZE, "canvas smaller than (nx+1) x (ny+1)");
  if (H <= 0 || W <= 0 || (long long)H * W > (1LL << 30)) return acs::fail(ACS_E_ARG, "bad canvas size");
  if (!b.ws_pool) {
    size_t bytes = 0;
    for (int c = 0; c < b.n; ++c) bytes += 3 * acs::WS_FIELDS * acs::align_up(8 * b.hc[c].n_elems, 256);
    CU(cudaMalloc(&b.ws_pool, bytes));
    CU(cudaMemsetAsync(b.ws_pool, 0, bytes, b.stream));
    std::vector<acs::WsCase> hw(b.n);
    char* q = b.ws_pool;
    for (int c = 0; c < b.n; ++c)
      for (int f = 0; f < acs::WS_FIELDS; ++f) {
        hw[c].prev[f] = (double*)q; q += acs::align_up(8 * b.hc[c].n_elems, 256);
        hw[c].inc[f] = (double*)q; q += acs::align_up(8 * b.hc[c].n_elems, 256);
        hw[c].incp[f] = (double*)q; q += acs::align_up(8 * b.hc[c].n_elems, 256);
      }
    CU(cudaMalloc(&b.d_ws, sizeof(acs::WsCase) * b.n));
    CU(cudaMemcpyAsync(b.d_ws, hw.data(), sizeof(acs::WsCase) * b.n, cudaMemcpyHostToDevice, b.stream));
    CU(cudaMalloc(&b.d_ws_res, sizeof(unsigned long long) * 3 * b.n));
    CU(cudaMalloc(&b.d_ws_choice, sizeof(int) * b.n));
    CU(cudaMalloc(&b.d_ws_ss, sizeof(double) * acs::WS_OUT * b.n));
    CU(cudaMalloc(&b.d_ws_sc, sizeof(double) * acs::WS_OUT * b.n));
    CU(cudaMemsetAsync(b.d_ws_sc, 0, sizeof(double) * acs::WS_OUT * b.n, b.stream));
    CU(cudaStreamSynchronize(b.stream));
  }
  b.ws_H = H;
  b.ws_W = W;
  b.ws_has_prev = 0;
  b.ws_calls = 0;
  return ACS_OK;
}

int acs_batch_ws_features(acs_batch* h, float* X, float* inc_scale) {
  if (!h || !X) return acs::fail(ACS_E_ARG, "null argument");
  Batch& b = *h->b;
  if (!b.ws_pool) return acs::fail(ACS_E_STATE, "warm start not enabled");
  acs::launch_ws_features(b.dc, b.dk, b.d_ws, b.n, b.ws_H, b.ws_W, b.ws_has_prev, b.d_ws_ss, b.d_ws_sc, X, inc_scale,
                          b.stream);
  CU(cudaGetLastError());
  b.ws_has_prev = 1;
  ++b.ws_calls;
  return ACS_OK;
}

int acs_batch_ws_target(acs_batch* h, float* T, float* Wt) {
  if (!h || !T || !Wt) return acs::fail(ACS_E_ARG, "null argument");
  Batch& b = *h->b;
  if (!b.ws_pool) return acs::fail(ACS_E_STATE, "warm start not enabled");
  acs::launch_ws_target(b.dc, b.dk, b.d_ws, b.n, b.ws_H, b.ws_W, b.d_ws_sc, T, Wt, b.stream);
  CU(cudaGetLastError());
  return ACS_OK;
}

int acs_batch_set_start(acs_batch* h, const float* Y, int ldy, const float* scale, int policy, int* chosen,
                        double* res0) {
  if (!h) return acs::fail(ACS_E_ARG, "null handle");
  Batch& b = *h->b;
  if (!b.ws_pool) return acs::fail(ACS_E_STATE, "warm start not enabled");
  if (policy < 0 || policy > 2) return acs::fail(ACS_E_ARG, "policy must be 0, 1 or 2");
  if (Y && (!scale || ldy < acs::WS_FIELDS)) return acs::fail(ACS_E_ARG, "Y needs scale and ldy >= 5");
  // the quadratic candidate needs two increments, i.e. three feature calls; before that, linear
  const int order = (b.ws_order == 2 && b.ws_calls >= 3) ? 2 : 1;
  acs::launch_ws_start(b.dc, b.dk, b.d_ws, b.n, b.ws_H, b.ws_W, b.d_ws_sc, Y, ldy, scale, policy, order,
                       b.d_ws_res, b.d_ws_choice, b.stream);
  CU(cudaGetLastError());
  int r = acs::pull_ctl(b);  // the commit kernel set tau_dirty where the prediction was kept
  if (r) return r;
  if (chosen) CU(cudaMemcpy(chosen, b.d_ws_choice, sizeof(int) * b.n, cudaMemcpyDeviceToHost));
  if (res0) {
    std::vector<unsigned long long> bits(3 * b.n);
    CU(cudaMemcpy(bits.data(), b.d_ws_res, sizeof(unsigned long long) * 3 * b.n, cudaMemcpyDeviceToHost));
    for (int q = 0; q < 3 * b.n; ++q) res0[q] = acs::bits_to_double(bits[q]);
    if (!Y)
      for (int c = 0; c < b.n; ++c) res0[3 * c + 2] = std::nan("");
  }
  return ACS_OK;
}

int acs_batch_time_kernel(acs_batch* h, int kernel, int reps, double* ms_mean, long long* cells) {
  if (!h || !ms_mean || reps <= 0 || kernel < 0 || kernel > 6) return acs::fail(ACS_E_ARG, "bad argument");
  Batch& b = *h->b;
  if (kernel >= 5) {
    int r = acs::te_setup(b);
    if (r) return r;
  }
  std::vector<acs::CaseCtl> saved = b.hk;
  long long nc = 0;
  for (int c = 0; c < b.n; ++c) {
    b.hk[c].active = 1;
    b.hk[c].scalars = 1;
    const int nx = b.hc[c].nx, ny = b.hc[c].ny;
    nc += kernel == 0 ? (long long)(nx - 3) * (ny - 2) : kernel == 1 ? (long long)(nx - 2) * (ny - 3)
          : kernel >= 5 ? (long long)nx * ny : (long long)(nx - 2) * (ny - 2);
  }
  int r = acs::push_ctl(b);
  if (r) return r;
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  auto one = [&]() { acs::launch_timed_kernel(b, kernel); };
  // the pressure kernels write pn (and the tile engine's P/T/C kernel T and C of role n_tau): keep
  // copies in stage scratch
  auto save = [&](bool back) -> int {
    for (int c = 0; c < b.n; ++c) {
      const acs::CaseDev& d = b.hc[c];
      const acs::CaseCtl& k = b.hk[c];
      double* live[3] = {d.P[k.rp[1]], d.T[k.rt[acs::R_NTAU]], d.C[k.rc[acs::R_NTAU]]};
      const int nf = kernel == 6 ? 3 : 1;
      for (int f = 0; f < nf; ++f) {
        double* a = back ? live[f] : d.S[1 + f];
        double* z = back ? d.S[1 + f] : live[f];
        CU(cudaMemcpyAsync(a, z, 8 * d.n_elems, cudaMemcpyDeviceToDevice, b.stream));
      }
    }
    return ACS_OK;
  };
  if (kernel == 2 || kernel == 6) {
    r = save(false);
    if (r) return r;
  }
  one();  // warm
  CU(cudaEventRecord(e0, b.stream));
  for (int i = 0; i < reps; ++i) one();
  CU(cudaEventRecord(e1, b.stream));
  CU(cudaEventSynchronize(e1));
  float ms = 0.f;
  CU(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CU(cudaGetLastError());
  if (kernel == 2 || kernel == 6) {
    r = save(true);
    if (r) return r;
  }
  *ms_mean = ms / reps;
  if (cells) *cells = nc;
  for (int c = 0; c < b.n; ++c) {  // the residual slots were touched; restore the control words
    saved[c].res_u = saved[c].res_v = saved[c].res_p = 0;
  }
  b.hk = saved;
  r = acs::push_ctl(b);
  if (!r) CU(cudaStreamSynchronize(b.stream));
  return r;
}

int acs_batch_set_cluster_size(acs_batch* h, int c, int ctas) {
  if (!h) return acs::fail(ACS_E_ARG, "null handle");
  Batch& b = *h->b;
  if (c < 0 || c >= b.n) return acs::fail(ACS_E_ARG, "case id out of range");
  if (ctas < 0 || ctas > 16) return acs::fail(ACS_E_ARG, "cluster size must be 0..16");
  if ((int)b.cluster_override.size() < b.n) b.cluster_override.assign(b.n, 0);
  b.cluster_override[c] = ctas;
  return ACS_OK;
}

int acs_batch_set_tolerance(acs_batch* h, int c, double eps) {
  if (!h) return acs::fail(ACS_E_ARG, "null handle");
  Batch& b = *h->b;
  if (c < 0 || c >= b.n) return acs::fail(ACS_E_ARG, "case id out of range");
  if (!(eps > 0.0) || !std::isfinite(eps)) return acs::fail(ACS_E_ARG, "tolerance must be positive and finite");
  b.prm[c].eps = eps;
  b.hc[c].eps = eps;
  // stream-ordered: launches already queued keep the old value, the next ones see the new one
  CU(cudaMemcpyAsync(&b.dc[c].eps, &b.hc[c].eps, sizeof(double), cudaMemcpyHostToDevice, b.stream));
  CU(cudaStreamSynchronize(b.stream));
  return ACS_OK;
}

int acs_batch_set_option(acs_batch* h, int option, long long value) {
  if (!h) return acs::fail(ACS_E_ARG, "null handle");
  Batch& b = *h->b;
  switch (option) {
    case ACS_OPT_ENGINE: {
      if (value < 0 || value > 2) return acs::fail(ACS_E_ARG, "engine must be 0, 1 or 2");
      if (value == 2) {
        int r = acs::te_setup(b);
        if (r) return r;
      }
      if (b.engine != (int)value) {  // the captured loop body belongs to the previous engine
        if (b.gexec) { cudaGraphExecDestroy(b.gexec); b.gexec = nullptr; }
        if (b.graph) { cudaGraphDestroy(b.graph); b.graph = nullptr; }
        b.graph_steps = -1;
      }
      b.engine = (int)value;
      return ACS_OK;
    }
    case ACS_OPT_NODES_PER_CTA:
      if (value < 64 || value > (1 << 22)) return acs::fail(ACS_E_ARG, "nodes per CTA out of range");
      b.nodes_per_cta = (int)value;
      return ACS_OK;
    case ACS_OPT_L1_LOADS:
      b.l1_loads = value ? 1 : 0;
      return ACS_OK;
    case ACS_OPT_THREADS:
      if (value != 256 && value != 512) return acs::fail(ACS_E_ARG, "threads must be 256 or 512");
      b.threads = (int)value;
      return ACS_OK;
    case ACS_OPT_CTAS_PER_SM:
      if (value != 1 && value != 2) return acs::fail(ACS_E_ARG, "CTAs per SM must be 1 or 2");
      b.ctas_per_sm = (int)value;
      return ACS_OK;
    case ACS_OPT_STAGED:
      b.staged = value ? 1 : 0;
      return ACS_OK;
    case ACS_OPT_EXTRAP_ORDER:
      if (value != 1 && value != 2) return acs::fail(ACS_E_ARG, "extrapolation order must be 1 or 2");
      b.ws_order = (int)value;
      return ACS_OK;
  }
  return acs::fail(ACS_E_ARG, "unknown option");
}

int acs_set_option(acs_handle* h, int option, long long value) {
  if (!h) return acs::fail(ACS_E_ARG, "null handle");
  acs_batch tmp{h->b};
  return acs_batch_set_option(&tmp, option, value);
}

int acs_batch_launch_count(acs_batch* h, long long* n) {
  if (!h || !n) return acs::fail(ACS_E_ARG, "null");
  *n = h->b->launches;
  return ACS_OK;
}

int acs_create(const acs_grid* g, const acs_params* p, acs_handle** out) {
  if (!out) return acs::fail(ACS_E_ARG, "null out");
  Batch* b = nullptr;
  int r = acs::create_batch(g, p, 1, &b);
  if (r) return r;
  *out = new acs_handle{b};
  return ACS_OK;
}

int acs_destroy(acs_handle* h) {
  if (!h) return ACS_OK;
  delete h->b;
  delete h;
  return ACS_OK;
}

int acs_set_stream(acs_handle* h, void* s) {
  if (!h) return acs::fail(ACS_E_ARG, "null handle");
  acs_batch tmp{h->b};
  return acs_batch_set_stream(&tmp, s);
}

int acs_set_field(acs_handle* h, int field, const double* host) {
  if (!h || !host) return acs::fail(ACS_E_ARG, "null argument");
  return acs::upload_field(*h->b, 0, field, host);
}

int acs_get_field(acs_handle* h, int field, double* host) {
  if (!h || !host) return acs::fail(ACS_E_ARG, "null argument");
  return acs::download_field(*h->b, 0, field, host);
}

int acs_cell_fields(acs_handle* h, double* u, double* v, double* vel_mag) {
  if (!h) return acs::fail(ACS_E_ARG, "null handle");
  acs_batch tmp{h->b};
  return acs_batch_cell_fields(&tmp, 0, u, v, vel_mag);
}

int acs_physical_steps(acs_handle* h, int n_steps, int* itc, int* iters, double* err, int* status) {
  if (!h || !itc) return acs::fail(ACS_E_ARG, "null argument");
  int st = 0;
  int r = acs::run_batch(*h->b, n_steps, itc, iters, err, &st);
  if (status) *status = st;
  return r;
}

int acs_launch_count(acs_handle* h, long long* n) {
  if (!h || !n) return acs::fail(ACS_E_ARG, "null");
  *n = h->b->launches;
  return ACS_OK;
}

#define NEED(x) if (!(x)) return acs::fail(ACS_E_ARG, "null argument: " #x)

int acs_solve_u(acs_handle* h, const double* um, const double* um_tau, double* vm_tau, const double* p,
                double* um_n_tau, double* residual_u) {
  NEED(h); NEED(um); NEED(um_tau); NEED(vm_tau); NEED(p); NEED(um_n_tau); NEED(residual_u);
  Batch& b = *h->b;
  int r = acs::refresh_flags(b);
  if (!r) r = acs::begin_routine(b);
  if (!r) r = acs::put(b, 0, 0, acs::R_PHYS, um);
  if (!r) r = acs::put(b, 0, 0, acs::R_TAU, um_tau);
  if (!r) r = acs::put(b, 0, 1, acs::R_TAU, vm_tau);
  if (!r) r = acs::put(b, 0, 2, 1, p);
  if (r) return r;
  acs::seq_u(b);
  r = acs::end_routine(b);
  if (!r) r = acs::get(b, 0, 0, acs::R_NTAU, um_n_tau);
  if (!r) r = acs::get(b, 0, 1, acs::R_TAU, vm_tau);
  if (!r) { cudaStreamSynchronize(b.stream); *residual_u = acs::bits_to_double(b.hk[0].res_u); }
  return r;
}

int acs_solve_v(acs_handle* h, const double* vm, double* um_tau, const double* vm_tau, const double* p,
                const double* T, double* vm_n_tau, double* residual_v) {
  NEED(h); NEED(vm); NEED(um_tau); NEED(vm_tau); NEED(p); NEED(T); NEED(vm_n_tau); NEED(residual_v);
  Batch& b = *h->b;
  b.t_unity[0] = acs::all_ones(T, (size_t)b.hc[0].nx * b.hc[0].ny);
  int r = acs::refresh_flags(b);
  if (!r) r = acs::begin_routine(b);
  if (!r) r = acs::put(b, 0, 1, acs::R_PHYS, vm);
  if (!r) r = acs::put(b, 0, 0, acs::R_TAU, um_tau);
  if (!r) r = acs::put(b, 0, 1, acs::R_TAU, vm_tau);
  if (!r) r = acs::put(b, 0, 2, 1, p);
  if (!r) r = acs::put(b, 0, 3, acs::R_PHYS, T);
  if (r) return r;
  acs::seq_v(b);
  r = acs::end_routine(b);
  if (!r) r = acs::get(b, 0, 1, acs::R_NTAU, vm_n_tau);
  if (!r) r = acs::get(b, 0, 0, acs::R_TAU, um_tau);
  if (!r) { cudaStreamSynchronize(b.stream); *residual_v = acs::bits_to_double(b.hk[0].res_v); }
  return r;
}

int acs_solve_p(acs_handle* h, const double* p, const double* um_n_tau, const double* vm_n_tau, double* pn,
                double* residual_p) {
  NEED(h); NEED(p); NEED(um_n_tau); NEED(vm_n_tau); NEED(pn); NEED(residual_p);
  Batch& b = *h->b;
  int r = acs::begin_routine(b);
  if (!r) r = acs::put(b, 0, 2, 0, p);
  if (!r) r = acs::put(b, 0, 0, acs::R_NTAU, um_n_tau);
  if (!r) r = acs::put(b, 0, 1, acs::R_NTAU, vm_n_tau);
  if (r) return r;
  acs::seq_p(b);
  r = acs::end_routine(b);
  if (!r) r = acs::get(b, 0, 2, 1, pn);
  if (!r) { cudaStreamSynchronize(b.stream); *residual_p = acs::bits_to_double(b.hk[0].res_p); }
  return r;
}

static int solve_scalar(acs_handle* h, bool is_c, const double* um_n_tau, const double* vm_n_tau, const double* Z,
                        double* Z_n_tau, const double* Z_tau) {
  NEED(h); NEED(um_n_tau); NEED(vm_n_tau); NEED(Z); NEED(Z_n_tau); NEED(Z_tau);
  Batch& b = *h->b;
  const int fam = is_c ? 4 : 3;
  int r = acs::begin_routine(b);
  if (!r) r = acs::put(b, 0, 0, acs::R_NTAU, um_n_tau);
  if (!r) r = acs::put(b, 0, 1, acs::R_NTAU, vm_n_tau);
  if (!r) r = acs::put(b, 0, fam, acs::R_PHYS, Z);
  if (!r) r = acs::put(b, 0, fam, acs::R_TAU, Z_tau);
  if (r) return r;
  acs::seq_s(b, is_c);
  r = acs::end_routine(b);
  if (!r) r = acs::get(b, 0, fam, acs::R_NTAU, Z_n_tau);
  if (!r) { cudaError_t e = cudaStreamSynchronize(b.stream); if (e != cudaSuccess) return acs::fail(ACS_E_CUDA, cudaGetErrorString(e)); }
  return r;
}

int acs_solve_z(acs_handle* h, const double* um_n_tau, const double* vm_n_tau, const double* T, double* T_n_tau,
                const double* T_tau) {
  return solve_scalar(h, false, um_n_tau, vm_n_tau, T, T_n_tau, T_tau);
}

int acs_solve_c(acs_handle* h, const double* um_n_tau, const double* vm_n_tau, const double* Cc, double* C_n_tau,
                const double* C_tau) {
  return solve_scalar(h, true, um_n_tau, vm_n_tau, Cc, C_n_tau, C_tau);
}

}  // extern "C"
