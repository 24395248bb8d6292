// engine_exact.cu -- the persistent cluster engine with the reference's exact arithmetic.
// Built with -fmad=false (see points_exact.cuh); results are bit-identical to the per-stage
// kernels and to the CPU oracle.
#include "engine.cuh"
#include "engine_api.h"
#include "points_exact.cuh"

namespace acs {

struct PtExact {
  static __device__ __forceinline__ double ld(const double* a, long long q) { return __ldcg(a + q); }
  static __device__ __forceinline__ double ru(const CaseDev& d, const double* uin, const double* vt,
                                              const double* pn, int i, int j) {
    const exact::G g(d);
    const bool quick = d.scheme == 0 && j >= 3 && j <= d.ny - 2;
    return quick ? exact::resu_quick(d, g, uin, vt, pn, i, j) : exact::resu_upwind(d, g, uin, vt, pn, i, j);
  }
  static __device__ __forceinline__ double rv(const CaseDev& d, const double* ut, const double* vin,
                                              const double* pn, const double* T, int i, int j) {
    const exact::G g(d);
    const bool quick = d.scheme == 0 && i >= 3 && i <= d.nx - 2;
    return quick ? exact::resv_quick(d, g, ut, vin, pn, T, i, j) : exact::resv_upwind(d, g, ut, vin, pn, T, i, j);
  }
  template <bool IS_C>
  static __device__ __forceinline__ double rs(const CaseDev& d, const double* un, const double* vn,
                                              const double* z, int i, int j) {
    const exact::G g(d);
    return exact::res_scalar<IS_C>(d, g, un, vn, z, i, j);
  }
  // solve_P's three stages at one node (equations.f90:620-662); *r = dtau*RP*beta
  static __device__ __forceinline__ double p_update(const CaseDev& d, const double* p, const double* un,
                                                    const double* vn, int i, int j, double* r) {
    const exact::G g(d);
    const double Aew = g.ym[j + 1] - g.ym[j], Ans = g.xm[i + 1] - g.xm[i];
    const double dudx = LD(un, g.o(i + 1, j)) * Aew - LD(un, g.o(i, j)) * Aew;
    const double dvdy = LD(vn, g.o(i, j + 1)) * Ans - LD(vn, g.o(i, j)) * Ans;
    double RP = -(dudx + dvdy);
    if (d.continuity == 1) RP = RP / ((g.ym[j + 1] - g.ym[j]) * (g.xm[i + 1] - g.xm[i]));
    const double p0 = LD(p, g.o(i, j));
    const double pi1 = p0 + d.dtau * RP * d.beta;
    const double pi2 = 0.75 * p0 + 0.25 * (pi1 + d.dtau * RP * d.beta);
    *r = d.dtau * RP * d.beta;
    return 1.0 / 3.0 * p0 + 2.0 / 3.0 * (pi2 + *r);
  }
};

cudaError_t launch_engine_exact(const EngineArgs& a, int cluster, int nclusters, cudaStream_t s) {
  auto kern = k_engine<PtExact, ENGINE_THREADS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cluster * nclusters);
  cfg.blockDim = dim3(ENGINE_THREADS);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, a);
}

int max_active_clusters_exact(int cluster) {
  auto kern = k_engine<PtExact, ENGINE_THREADS>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cluster);
  cfg.blockDim = dim3(ENGINE_THREADS);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

}  // namespace acs
