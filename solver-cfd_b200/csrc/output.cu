// output.cu -- cell-centred output fields on the device (acs_batch_cell_fields, acs_cell_fields).
//
// comp_mean.f90:1-25: u(i,j) = (um(i+1,j) + um(i,j)) * 0.5 and v(i,j) = (vm(i,j+1) + vm(i,j)) * 0.5
// at every cell, and the velocity magnitude sqrt(u**2 + v**2) that transient.f90:69-74 writes to
// the ParaView file.  Compiled with -fmad=false: each product and sum is rounded on its own, as in
// the reference, so the fields equal the host's comp_mean bit for bit.
#include <cuda_runtime.h>

#include "acs_dev.cuh"

namespace acs {

__global__ void k_cell_fields(const double* __restrict__ um, const double* __restrict__ vm, int nx, int ny,
                              int pitch, double* __restrict__ u, double* __restrict__ v, double* __restrict__ mag) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > nx || j > ny) return;
  const long long q = lin(i, j, pitch);
  const double uc = (um[q + 1] + um[q]) * 0.5;
  const double vc = (vm[q + pitch] + vm[q]) * 0.5;
  u[q] = uc;
  v[q] = vc;
  mag[q] = sqrt(uc * uc + vc * vc);
}

cudaError_t launch_cell_fields(const double* um, const double* vm, int nx, int ny, int pitch, double* u, double* v,
                               double* mag, cudaStream_t s) {
  const dim3 block(32, 8), grid((nx + 31) / 32, (ny + 7) / 8);
  k_cell_fields<<<grid, block, 0, s>>>(um, vm, nx, ny, pitch, u, v, mag);
  return cudaGetLastError();
}

}  // namespace acs
