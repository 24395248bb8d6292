// bc_exact.cuh -- the boundary passes bcUV / bcP / bcZ / bcC, one thread block per case.
//
// Shared by the stage-kernel loop (kernels_exact.cu) and the warm-start kernels
// (warmstart.cu); both units are compiled with -fmad=false.  Reference (OpenMp_Multicore/):
// boundary.f90:1-159.
#pragma once
#include <cuda_runtime.h>
#include "acs_dev.cuh"

namespace acs {

// ---- boundary passes (boundary.f90), one block per case --------------------------------------
// which: 0..2 = u written by U stage s (S0, S1, U[ntau]) with vm = V[tau];
//        3..5 = um = U[tau] with v written by V stage s (S0, S1, V[ntau]).
__device__ inline void bc_uv_block(const CaseDev& d, double* um, double* vm) {
  const int nx = d.nx, ny = d.ny, P = d.pitch;
  const int tid = threadIdx.x, nt = blockDim.x;
  if (d.bc == 0) {
    // bottom, top rows (boundary.f90:9-26), per column i
    for (int i = 1 + tid; i <= nx; i += nt) {
      vm[lin(i, 1, P)] = d.v_in;
      vm[lin(i, 2, P)] = vm[lin(i, 1, P)];
      if (i >= 2) {
        um[lin(i, 1, P)] = 0.0;
        vm[lin(i, ny, P)] = 2.0 * vm[lin(i, ny - 2, P)] - vm[lin(i, ny - 1, P)];
        vm[lin(i, ny + 1, P)] = 2.0 * vm[lin(i, ny - 1, P)] - vm[lin(i, ny, P)];
        um[lin(i, ny, P)] = um[lin(i, ny - 1, P)];
      }
    }
    __syncthreads();
    // left (:29-36) and right (:39-46) columns
    for (int j = 1 + tid; j <= ny + 1; j += nt) {
      if (j <= ny) {
        um[lin(2, j, P)] = 0.0; um[lin(1, j, P)] = 0.0;
        um[lin(nx, j, P)] = 0.0; um[lin(nx + 1, j, P)] = 0.0;
      }
      vm[lin(1, j, P)] = vm[lin(2, j, P)];
      if (j >= 2 && j <= ny) vm[lin(nx, j, P)] = vm[lin(nx - 1, j, P)];
    }
  } else {
    // channel: inflow/outflow columns first, then the wall rows
    for (int j = 1 + tid; j <= ny + 1; j += nt) {
      if (j <= ny) {
        um[lin(1, j, P)] = d.v_in;
        um[lin(2, j, P)] = d.v_in;
        um[lin(nx, j, P)] = um[lin(nx - 1, j, P)];
        um[lin(nx + 1, j, P)] = um[lin(nx, j, P)];
      }
      vm[lin(1, j, P)] = -vm[lin(2, j, P)];
      vm[lin(nx, j, P)] = vm[lin(nx - 1, j, P)];
    }
    __syncthreads();
    for (int i = 1 + tid; i <= nx + 1; i += nt) {
      um[lin(i, 1, P)] = -um[lin(i, 2, P)];
      um[lin(i, ny, P)] = -um[lin(i, ny - 1, P)];
      if (i <= nx) {
        vm[lin(i, 2, P)] = 0.0;
        vm[lin(i, ny, P)] = 0.0;
        vm[lin(i, 1, P)] = -vm[lin(i, 3, P)];
        vm[lin(i, ny + 1, P)] = -vm[lin(i, ny - 1, P)];
      }
    }
  }
}

// bcP / bcZ / bcC (boundary.f90:52-159); `neumann_in` = true for p (inflow boundary copies the
// neighbour), false for scalars (inflow boundary takes zin).
__device__ inline void bc_cell_block(const CaseDev& d, double* z, bool neumann_in, double zin) {
  const int nx = d.nx, ny = d.ny, P = d.pitch;
  const int tid = threadIdx.x, nt = blockDim.x;
  if (d.bc == 0) {
    for (int i = 1 + tid; i <= nx; i += nt) {
      z[lin(i, 1, P)] = neumann_in ? z[lin(i, 2, P)] : zin;
      z[lin(i, ny, P)] = z[lin(i, ny - 1, P)] + 1.0 * (z[lin(i, ny - 1, P)] - z[lin(i, ny - 2, P)]);
    }
    __syncthreads();
    for (int j = 1 + tid; j <= ny; j += nt) {
      z[lin(1, j, P)] = z[lin(2, j, P)];
      z[lin(nx, j, P)] = z[lin(nx - 1, j, P)];
    }
  } else {
    for (int j = 1 + tid; j <= ny; j += nt) {
      z[lin(1, j, P)] = neumann_in ? z[lin(2, j, P)] : zin;
      z[lin(nx, j, P)] = z[lin(nx - 1, j, P)] + 1.0 * (z[lin(nx - 1, j, P)] - z[lin(nx - 2, j, P)]);
    }
    __syncthreads();
    for (int i = 1 + tid; i <= nx; i += nt) {
      z[lin(i, 1, P)] = z[lin(i, 2, P)];
      z[lin(i, ny, P)] = z[lin(i, ny - 1, P)];
    }
  }
}

}  // namespace acs
