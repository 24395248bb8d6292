// control.cu -- device-side pseudo-loop control (main.f90:116-186).
//
// After every pseudo-iteration one block per case evaluates
//     error = MAX(residual_u, residual_v, residual_p)                     (main.f90:139)
//     IF (itc .NE. 1 .AND. error .LT. eps) EXIT                            (main.f90:142)
// and applies the state updates of the reference by rotating buffer roles:
//   * no exit: um_tau=um_n_tau, vm_tau=vm_n_tau, p=pn, T_tau=T_n_tau, C_tau=C_n_tau, itc+=1
//     (main.f90:145-150) -> swap the tau and n_tau roles, swap p and pn; the momentum routines
//     then read the pressure from the p-role buffer (CaseCtl::rp_read), since after the copy
//     the reference's pn holds the same values;
//   * exit: the tau copies are skipped (the next step starts from the previous pseudo-iterate,
//     and p stays one iterate behind pn), then um=um_n_tau, vm=vm_n_tau, T=T_n_tau, C=C_n_tau
//     and itc=0 (main.f90:154-157,182) -> swap the phys and n_tau roles;
//   * the loop condition itc < itc_max fails after the copies (main.f90:120): the latest iterate
//     is then in the tau buffers and is copied into phys.
// A NaN or infinite residual marks the case FAILED and removes it from the launch (the reference
// would run on to itc_max).
#include <cuda_runtime.h>
#include "acs_dev.cuh"
#include "kernels.h"

namespace acs {

__device__ inline void swap_i(int& a, int& b) { int t = a; a = b; b = t; }

__global__ void k_control(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl, int* iters,
                          double* err, int* n_active) {
  const int c = blockIdx.x;
  CaseCtl& k = ctl[c];
  const CaseDev& d = cs[c];
  __shared__ int s_copy;
  if (threadIdx.x == 0) {
    s_copy = 0;
    if (k.active) {
      const double ru = __longlong_as_double((long long)k.res_u);
      const double rv = __longlong_as_double((long long)k.res_v);
      const double rp = __longlong_as_double((long long)k.res_p);
      double e = ru;
      if (rv > e || rv != rv) e = rv;
      if (rp > e || rp != rp) e = rp;
      k.res_u = k.res_v = k.res_p = 0ull;
      k.k += 1;
      k.total_iters += 1;
      const bool bad = (e != e) || (e > 1.0e300);
      bool step_done = false;
      if (bad) {
        k.status = 2;
        k.active = 0;
        step_done = true;
      } else if (k.itc != 1 && e < d.eps) {
        k.rp_read = k.rp[1];
        k.ntau_alias = 1;
        swap_i(k.ru[R_PHYS], k.ru[R_NTAU]);
        swap_i(k.rv[R_PHYS], k.rv[R_NTAU]);
        if (d.solve_scalars) {
          swap_i(k.rt[R_PHYS], k.rt[R_NTAU]);
          swap_i(k.rc[R_PHYS], k.rc[R_NTAU]);
        }
        step_done = true;
      } else {
        swap_i(k.ru[R_TAU], k.ru[R_NTAU]);
        swap_i(k.rv[R_TAU], k.rv[R_NTAU]);
        swap_i(k.rp[0], k.rp[1]);
        k.rp_read = k.rp[0];
        k.ntau_alias = 2;
        k.tau_dirty = 0;
        if (d.solve_scalars) {
          swap_i(k.rt[R_TAU], k.rt[R_NTAU]);
          swap_i(k.rc[R_TAU], k.rc[R_NTAU]);
        }
        k.itc += 1;
        if (k.itc >= d.itc_max) {
          s_copy = 1;
          step_done = true;
        }
      }
      if (step_done) {
        if (k.step < k.n_steps) {
          if (iters) iters[(long long)c * k.n_steps + k.step] = k.k;
          if (err) err[(long long)c * k.n_steps + k.step] = e;
        }
        if (k.status != 2) {
          k.step += 1;
          k.itc = 0;
          k.k = 0;
          if (k.step >= k.n_steps) {
            k.active = 0;
            k.status = 1;
          }
        }
      }
      if (k.active) atomicAdd(n_active, 1);
    }
  }
  __syncthreads();
  if (s_copy) {
    const long long n = d.n_elems;
    const double* src[4] = {d.U[k.ru[R_TAU]], d.V[k.rv[R_TAU]], d.T[k.rt[R_TAU]], d.C[k.rc[R_TAU]]};
    double* dst[4] = {d.U[k.ru[R_PHYS]], d.V[k.rv[R_PHYS]], d.T[k.rt[R_PHYS]], d.C[k.rc[R_PHYS]]};
    const int nf = d.solve_scalars ? 4 : 2;
    for (int f = 0; f < nf; ++f)
      for (long long q = threadIdx.x; q < n; q += blockDim.x) dst[f][q] = src[f][q];
  }
}

// Sets the WHILE condition of the graph: continue while any case is active, bounded by
// max_iters pseudo-iterations so the loop always ends.
__global__ void k_loop_cond(int* n_active, long long* iter_count, long long max_iters,
                            cudaGraphConditionalHandle handle) {
  const int a = *n_active;
  *n_active = 0;
  const long long it = ++(*iter_count);
  cudaGraphSetConditional(handle, (a > 0 && it < max_iters) ? 1u : 0u);
}

// Host-polled variant: publishes the number of active cases to a mapped host word.
__global__ void k_loop_flag(int* n_active, long long* iter_count, int* host_flag) {
  const int a = *n_active;
  *n_active = 0;
  ++(*iter_count);
  *(volatile int*)host_flag = a;
}

}  // namespace acs
