// mesh_device.cu -- the channel mesh of the synthetic configurations generated on the device
// (acs_mesh_channel_device), for batches of many cases built without host arrays.
//
// The 1-D arrays x, y, xm, ym are O(nx + ny) and computed on the host exactly as acs_mesh_channel
// does (the same function), then copied; the O(nx * ny) part runs on the device in two kernels:
//   k_flag_dilate: a cell is "interior" (2) when its node lies in a porous box, else fluid (0);
//                  the first two sweeps of nonsymetric_mesh.f90:196-209 mark interior cells with a
//                  fluid neighbour as "boundary" (1) -- a sweep tests only for fluid neighbours and
//                  changes only interior cells, so every cell is decided from the classification
//                  of its neighbours, recomputed on the fly;
//   k_flag_side:   the third sweep (:210-218) marks fluid cells next to a boundary cell as
//                  "boundary side" (3), reading the previous kernel's flags (including the
//                  column-major word before each column, flag(0,j) = flag(nx,j-1), that the
//                  reference reads), and writes epsilon1 = porosity, liga = 1 on every
//                  non-fluid cell (1 and 0 elsewhere).
// Flags, epsilon1 and liga are bit-identical to acs_mesh_channel's (integer decisions and exact
// selections on identical coordinates).
#include <cuda_runtime.h>

#include <vector>

#include "../../include/acs.h"

void acs_channel_axes(int nx, int ny, double Lx, double Ly, double s, double* x, double* y, double* xm, double* ym);

namespace {

constexpr int kFluid = 0, kBoundary = 1, kInterior = 2, kBoundarySide = 3;  // comum.f90:75

struct Boxes {
  double b[2][4];  // x0, x1, y0, y1 of up to two porous boxes
  int nb;
};

__device__ __forceinline__ int classify(const double* X, const double* Y, const Boxes& B, int i, int j) {
  const double px = X[i - 1], py = Y[j - 1];
  for (int k = 0; k < B.nb; ++k) {
    const double* b = B.b[k];
    if (b[0] <= b[1] && px >= b[0] && px <= b[1] && py >= b[2] && py <= b[3]) return kInterior;
  }
  return kFluid;
}

__global__ void k_flag_dilate(const double* X, const double* Y, Boxes B, int nx, int ny, int* flag) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > nx || j > ny) return;
  int f = classify(X, Y, B, i, j);
  if (f == kInterior && j >= 2 && j <= ny - 1) {
    if (i >= 2 && i <= nx - 1) {
      if (classify(X, Y, B, i - 1, j) == kFluid || classify(X, Y, B, i, j - 1) == kFluid ||
          classify(X, Y, B, i + 1, j) == kFluid || classify(X, Y, B, i, j + 1) == kFluid)
        f = kBoundary;
    } else if (i == 1) {
      if (classify(X, Y, B, 1, j - 1) == kFluid || classify(X, Y, B, 1, j + 1) == kFluid) f = kBoundary;
    }
  }
  flag[(i - 1) + (long long)(j - 1) * nx] = f;
}

__global__ void k_flag_side(const int* flag_in, int nx, int ny, double porosity, int* flag, double* eps,
                            double* liga) {  // flag_in and flag may be the same array
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > nx || j > ny) return;
  const long long n = (long long)nx * ny;
  auto word = [&](int a, int b) -> int {
    const long long w = (long long)(a - 1) + (long long)(b - 1) * nx;
    return (w >= 0 && w < n) ? flag_in[w] : -1;
  };
  const long long q = (i - 1) + (long long)(j - 1) * nx;
  int f = flag_in[q];
  if (i <= nx - 1 && j <= ny - 1 && f == kFluid &&
      (word(i - 1, j) == kBoundary || word(i, j - 1) == kBoundary || word(i + 1, j) == kBoundary ||
       word(i, j + 1) == kBoundary))
    f = kBoundarySide;
  flag[q] = f;
  const bool porous = f != kFluid;
  eps[q] = porous ? porosity : 1.0;
  liga[q] = porous ? 1.0 : 0.0;
}

}  // namespace

extern "C" int acs_mesh_channel_device(int imax, int jmax, double Lx, double Ly, double s, const double* box1,
                                       const double* box2, double porosity, double* x, double* y, double* xm,
                                       double* ym, int* flag, double* epsilon1, double* liga_poros, void* stream) {
  if (imax < 6 || jmax < 6 || !x || !y || !xm || !ym || !flag || !epsilon1 || !liga_poros) return ACS_E_ARG;
  const int nx = imax, ny = jmax;
  std::vector<double> ax(nx), ay(ny), axm(nx + 1), aym(ny + 1);
  acs_channel_axes(nx, ny, Lx, Ly, s, ax.data(), ay.data(), axm.data(), aym.data());
  Boxes B{};
  for (const double* b : {box1, box2})
    if (b) {
      for (int k = 0; k < 4; ++k) B.b[B.nb][k] = b[k];
      ++B.nb;
    }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(x, ax.data(), sizeof(double) * nx, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(y, ay.data(), sizeof(double) * ny, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(xm, axm.data(), sizeof(double) * (nx + 1), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ym, aym.data(), sizeof(double) * (ny + 1), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return ACS_E_CUDA;
  // the third sweep runs in place on `flag`: it only turns fluid cells into boundary-side cells
  // and only asks whether a neighbour is a boundary cell, so a neighbour read before or after its
  // own update gives the same answer
  const dim3 block(32, 8), grid((nx + 31) / 32, (ny + 7) / 8);
  k_flag_dilate<<<grid, block, 0, st>>>(x, y, B, nx, ny, flag);
  k_flag_side<<<grid, block, 0, st>>>(flag, nx, ny, porosity, flag, epsilon1, liga_poros);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? ACS_OK : ACS_E_CUDA;
}
