// engine_api.h -- host entry points of the persistent cluster engine (engine_*.cu).
#pragma once
#include <cuda_runtime.h>
#include "engine.cuh"

namespace acs {
// Launch `nclusters` clusters of `cluster` CTAs; cluster c handles case a.cases[c].
cudaError_t launch_engine_exact(const EngineArgs& a, int cluster, int nclusters, cudaStream_t s);
cudaError_t launch_engine_fast(const EngineArgs& a, int cluster, int nclusters, cudaStream_t s, int l1, int threads,
                               int ctas_per_sm, int staged);
// Clusters of this size that fit on the device at once (0 if the size cannot be launched).
int max_active_clusters_exact(int cluster);
}  // namespace acs
