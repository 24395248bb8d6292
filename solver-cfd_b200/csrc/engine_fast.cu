// engine_fast.cu -- the persistent cluster engine with FAST arithmetic.
//
// The FAST arithmetic (points_fast.cuh) differs from the reference's in the last bits only; the
// loop's iteration counts and fields are checked against the oracle at 1e-10 relative.
#include "engine.cuh"
#include "engine_api.h"
#include "fast.h"
#include "points_fast.cuh"

namespace acs {

using PtFast = PtFastT<LdL2>;
using PtFastL1 = PtFastT<LdL1>;
using PtFastGen = PtFastT<LdGen>;

namespace {
template <class PT, int NT, int MINB, bool STG = false>
cudaError_t launch_fast_t(const EngineArgs& a, int cluster, int nclusters, cudaStream_t s) {
  auto kern = k_engine<PT, NT, MINB, STG>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  const size_t smem = STG ? (size_t)STAGE_SLOTS * a.stage_elems * sizeof(double) : 0;
  if (STG) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cluster * nclusters);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = smem;
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
}  // namespace

// threads: 256 or 512 per CTA; ctas_per_sm: 2 caps a 256-thread CTA at 128 registers so two
// CTAs of different clusters share an SM; l1: load cluster-written arrays through L1; staged:
// stage the stencil arrays in shared memory (a.stage_elems doubles per slot, one CTA per SM)
cudaError_t launch_engine_fast(const EngineArgs& a, int cluster, int nclusters, cudaStream_t s, int l1, int threads,
                               int ctas_per_sm, int staged) {
  if (staged) {
    if (threads == 512) return launch_fast_t<PtFastGen, 512, 1, true>(a, cluster, nclusters, s);
    return launch_fast_t<PtFastGen, 256, 1, true>(a, cluster, nclusters, s);
  }
  if (threads == 512)
    return l1 ? launch_fast_t<PtFastL1, 512, 1>(a, cluster, nclusters, s) : launch_fast_t<PtFast, 512, 1>(a, cluster, nclusters, s);
  if (ctas_per_sm == 2)
    return l1 ? launch_fast_t<PtFastL1, 256, 2>(a, cluster, nclusters, s) : launch_fast_t<PtFast, 256, 2>(a, cluster, nclusters, s);
  return l1 ? launch_fast_t<PtFastL1, 256, 1>(a, cluster, nclusters, s) : launch_fast_t<PtFast, 256, 1>(a, cluster, nclusters, s);
}

}  // namespace acs
