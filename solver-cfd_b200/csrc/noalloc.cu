// noalloc.cu -- solve_U without any device allocation (acs_solve_u_static).
//
// Who needs it: callers that cannot call cudaMalloc -- a host application whose device memory is
// owned by another allocator (a pool that must not be fragmented, or a framework that pre-claims
// the GPU), or a loop that must not allocate while it runs.  acs_solve_u needs a handle, and
// acs_create allocates; this entry point uses none.
//
// The scratch it needs -- pitched copies of the input fields, the two Runge-Kutta stage arrays
// of solve_U (the reference's local array `ui`, equations.f90:249), the case descriptor, the
// control word holding the residual, and the tile table -- lives in one file-scope static device
// array of ACS_STATIC_SCRATCH_BYTES.  Every GPU that loads this library holds that array until
// the process exits.  Host code may not use the array's name as a device address: on the host the
// symbol is a stand-in, so the device address is fetched once per device with
// cudaGetSymbolAddress (on the first call made on that device; make that first call before any
// stream capture) and passed to the kernels.  That cached address belongs to the context it was
// taken in: after cudaDeviceReset the library's module is loaded again, so a caller that resets
// the device must not call this entry point again in the same process.  Every call rewrites the
// part of the array it uses (clearing it first), so calls that overlap on the GPU (two streams,
// two host threads) race and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/acs.h"
#include "acs_dev.cuh"
#include "kernels.h"

namespace acs {
int fail(int code, const std::string& msg);
int validate_params(const acs_params& p);  // solver.cu: the checks acs_create makes

namespace {

constexpr long long kMaxNodes = ACS_STATIC_MAX_NODES;  // (imax+1)*(jmax+1)
constexpr int kMaxDim = ACS_STATIC_MAX_DIM;            // imax, jmax
constexpr int kMaxTiles = 1024;
constexpr int kFields = 9;                             // eps liga um um_tau vm_tau p S0 S1 um_n_tau
constexpr size_t kHead = 4096;                         // CaseDev, CaseCtl
constexpr size_t kTileBytes = sizeof(Tile) * kMaxTiles;
constexpr size_t kMetricBytes = sizeof(double) * 4 * (kMaxDim + 3);
constexpr size_t kFieldBytes = sizeof(double) * kMaxNodes;
constexpr size_t kScratchBytes = kHead + kTileBytes + kMetricBytes + kFields * kFieldBytes;
static_assert(kScratchBytes <= ACS_STATIC_SCRATCH_BYTES, "scratch layout exceeds the stated size");
constexpr size_t kCtlOffset = 2048;                    // CaseDev at 0, CaseCtl at kCtlOffset
static_assert(sizeof(CaseDev) <= kCtlOffset, "case descriptor overlaps the control word");
static_assert(kCtlOffset + sizeof(CaseCtl) <= kHead, "control word overlaps the tile table");

__device__ __align__(256) unsigned char g_scratch[ACS_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
char* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_mutex;

// Device address of g_scratch on the current device (looked up once per device).
int scratch_address(char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(ACS_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(ACS_E_CUDA, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return fail(ACS_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<char*>(p);
  }
  *out = g_scratch_addr[dev];
  return ACS_OK;
}

// Sets n doubles at p to v (the porosity padding; cudaMemset cannot write 1.0).
__global__ void k_fill(double* p, long long n, double v) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    p[q] = v;
}

}  // namespace
}  // namespace acs

extern "C" int acs_solve_u_static(const acs_params* p, const acs_grid* g, const double* um, const double* um_tau,
                                  double* vm_tau, const double* pn, double* um_n_tau, double* residual_u,
                                  void* stream) {
  using namespace acs;
  if (!p || !g || !um || !um_tau || !vm_tau || !pn || !um_n_tau || !residual_u)
    return fail(ACS_E_ARG, "null argument");
  if (!g->x || !g->y || !g->xm || !g->ym || !g->epsilon1 || !g->liga_poros) return fail(ACS_E_ARG, "null grid array");
  const int nx = p->imax, ny = p->jmax;
  if (g->imax != nx || g->jmax != ny) return fail(ACS_E_ARG, "grid and params disagree on imax/jmax");
  if (nx < 6 || ny < 6) return fail(ACS_E_SIZE, "imax and jmax must be at least 6");
  const int pitch = (nx + 1 + 3) / 4 * 4;
  if (nx > kMaxDim || ny > kMaxDim || (long long)pitch * (ny + 1) > kMaxNodes)
    return fail(ACS_E_SIZE, "acs_solve_u_static: case too large for the static scratch (need imax, jmax <= " +
                                std::to_string(kMaxDim) + " and round_up(imax+1, 4)*(jmax+1) <= " +
                                std::to_string(kMaxNodes) + ")");
  int r = validate_params(*p);
  if (r) return r;
  if (p->arith != ACS_ARITH_EXACT)
    return fail(ACS_E_ARG, "acs_solve_u_static computes in the EXACT arithmetic only (arith must be 0)");
  char* base = nullptr;
  r = scratch_address(&base);
  if (r) return r;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  // carve the scratch
  CaseDev* dcase = reinterpret_cast<CaseDev*>(base);
  CaseCtl* dctl = reinterpret_cast<CaseCtl*>(base + kCtlOffset);
  Tile* dtiles = reinterpret_cast<Tile*>(base + kHead);
  double* metric = reinterpret_cast<double*>(base + kHead + kTileBytes);
  double* fld[kFields];
  for (int f = 0; f < kFields; ++f)
    fld[f] = reinterpret_cast<double*>(base + kHead + kTileBytes + kMetricBytes + f * kFieldBytes);
  double *eps = fld[0], *liga = fld[1], *f_um = fld[2], *f_utau = fld[3], *f_vtau = fld[4], *f_p = fld[5],
         *s0 = fld[6], *s1 = fld[7], *f_un = fld[8];

  // case descriptor: metric arrays 1-based (element 0 unused), fields pitched
  CaseDev d;
  std::memset(&d, 0, sizeof(d));
  d.nx = nx; d.ny = ny; d.pitch = pitch;
  d.scheme = p->scheme; d.bc = p->bc; d.solve_scalars = 0; d.itc_max = p->itc_max;
  d.continuity = p->continuity;
  d.Re = p->Re; d.Pe = p->Pe; d.Sc = p->Sc; d.Da = p->Da; d.Cf = p->Cf; d.g = p->g; d.InvFr2 = p->InvFr2;
  d.v_in = p->v_in; d.T_in = p->T_in; d.C_in = p->C_in; d.b_art = p->b_art; d.beta = p->beta;
  d.dt = p->dt; d.dtau = p->dtau; d.eps = p->eps;
  d.flags = F_POROUS | (p->b_art != 0.0 ? F_BART : 0);
  d.x = metric; d.y = metric + (kMaxDim + 3); d.xm = metric + 2 * (kMaxDim + 3); d.ym = metric + 3 * (kMaxDim + 3);
  d.epsf = eps; d.liga = liga;
  d.U[0] = f_um; d.U[1] = f_utau; d.U[2] = f_un;
  d.V[0] = f_vtau; d.V[1] = f_vtau; d.V[2] = f_vtau;  // solve_U reads only vm_tau
  d.P[0] = f_p; d.P[1] = f_p;
  d.S[0] = s0; d.S[1] = s1; d.S[2] = s0; d.S[3] = s1;
  d.n_elems = (long long)pitch * (ny + 1);
  CaseCtl k;
  std::memset(&k, 0, sizeof(k));
  for (int q = 0; q < 3; ++q) k.ru[q] = k.rv[q] = k.rt[q] = k.rc[q] = q;
  k.rv[0] = k.rv[1] = k.rv[2] = 0;
  k.rp[0] = 0; k.rp[1] = 1; k.rp_read = 1;
  k.active = 1;  // res_u starts at zero for this call

  const int ntx = (nx + 1 + TILE_X - 1) / TILE_X, nty = (ny + 1 + TILE_Y - 1) / TILE_Y;
  if (ntx * nty > kMaxTiles) return fail(ACS_E_SIZE, "acs_solve_u_static: too many tiles for the static table");
  Tile tiles[kMaxTiles];
  int nt = 0;
  for (int j0 = 1; j0 <= ny + 1; j0 += TILE_Y)
    for (int i0 = 1; i0 <= nx + 1; i0 += TILE_X) tiles[nt++] = {0, i0, j0, 0};

#define CUS(call)                                                                                  \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return fail(ACS_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)
  CUS(cudaMemcpyAsync(dcase, &d, sizeof(d), cudaMemcpyHostToDevice, s));
  CUS(cudaMemcpyAsync(dctl, &k, sizeof(k), cudaMemcpyHostToDevice, s));
  CUS(cudaMemcpyAsync(dtiles, tiles, sizeof(Tile) * nt, cudaMemcpyHostToDevice, s));
  const cudaMemcpyKind D2D = cudaMemcpyDeviceToDevice;
  CUS(cudaMemcpyAsync(const_cast<double*>(d.x) + 1, g->x, sizeof(double) * nx, D2D, s));
  CUS(cudaMemcpyAsync(const_cast<double*>(d.y) + 1, g->y, sizeof(double) * ny, D2D, s));
  CUS(cudaMemcpyAsync(const_cast<double*>(d.xm) + 1, g->xm, sizeof(double) * (nx + 1), D2D, s));
  CUS(cudaMemcpyAsync(const_cast<double*>(d.ym) + 1, g->ym, sizeof(double) * (ny + 1), D2D, s));
  // The scratch keeps the previous call's contents.  Clear every field region this call uses
  // (pitch padding, the row past jmax and the tail past the case included) so nothing of an
  // earlier, larger call survives, and give the porosity padding the values of a fluid node
  // (epsilon1 = 1, liga = 0).  None of this allocates.
  const long long ne = (long long)pitch * (ny + 1);
  for (int f = 1; f < kFields; ++f) CUS(cudaMemsetAsync(fld[f], 0, sizeof(double) * ne, s));
  k_fill<<<64, 256, 0, s>>>(eps, ne, 1.0);
  CUS(cudaGetLastError());
  // Fortran-layout inputs -> pitched scratch (leading dimension nx+1 for u, nx for v and cells)
  auto in2d = [&](double* dst, const double* src, int w, int h) {
    return cudaMemcpy2DAsync(dst, (size_t)pitch * 8, src, (size_t)w * 8, (size_t)w * 8, h, D2D, s);
  };
  CUS(in2d(eps, g->epsilon1, nx, ny));
  CUS(in2d(liga, g->liga_poros, nx, ny));
  CUS(in2d(f_um, um, nx + 1, ny));
  CUS(in2d(f_utau, um_tau, nx + 1, ny));
  CUS(in2d(f_vtau, vm_tau, nx, ny + 1));
  CUS(in2d(f_p, pn, nx, ny));
  // solve_U: three stages, each followed by bcUV(stage array, vm_tau) (equations.f90:259-296)
  for (int st = 1; st <= 3; ++st) {
    launch_u_stage_exact(st, dcase, dctl, dtiles, nt, s);
    launch_bc_uv(dcase, dctl, 1, st - 1, s);
  }
  CUS(cudaGetLastError());
  auto out2d = [&](double* dst, const double* src, int w, int h) {
    return cudaMemcpy2DAsync(dst, (size_t)w * 8, src, (size_t)pitch * 8, (size_t)w * 8, h, D2D, s);
  };
  CUS(out2d(um_n_tau, f_un, nx + 1, ny));
  CUS(out2d(vm_tau, f_vtau, nx, ny + 1));
  unsigned long long bits = 0;
  CUS(cudaMemcpyAsync(&bits, &dctl->res_u, sizeof(bits), cudaMemcpyDeviceToHost, s));
  CUS(cudaStreamSynchronize(s));
  std::memcpy(residual_u, &bits, sizeof(double));
#undef CUS
  return ACS_OK;
}
