// kernels_fast.cu -- fused FAST-arithmetic kernels (placeholder until the fused path lands).
#include "engine_api.h"
#include "fast.h"

namespace acs {

struct FastPlan { int dummy; };

int fast_create(std::vector<CaseDev>&, const acs_grid*, const acs_params*, FastPlan**) {
  return fail(ACS_E_UNSUPPORTED, "fast arithmetic is not built yet");
}
void fast_destroy(FastPlan* f) { delete f; }
void fast_u(FastPlan*, const CaseDev*, CaseCtl*, const Tile*, int, int, cudaStream_t) {}
void fast_v(FastPlan*, const CaseDev*, CaseCtl*, const Tile*, int, int, cudaStream_t) {}
void fast_p(FastPlan*, const CaseDev*, CaseCtl*, const Tile*, int, int, cudaStream_t) {}
void fast_s(FastPlan*, bool, const CaseDev*, CaseCtl*, const Tile*, int, int, cudaStream_t) {}
void fast_timed(FastPlan*, int, const CaseDev*, CaseCtl*, const Tile*, int, int, cudaStream_t) {}
int fast_u_launches(const FastPlan*) { return 0; }
cudaError_t launch_engine_fast(const EngineArgs&, int, int, cudaStream_t) { return cudaErrorNotSupported; }
int max_active_clusters_fast(int) { return 0; }
int fast_v_launches(const FastPlan*) { return 0; }
int fast_p_launches(const FastPlan*) { return 0; }
int fast_s_launches(const FastPlan*) { return 0; }

}  // namespace acs
