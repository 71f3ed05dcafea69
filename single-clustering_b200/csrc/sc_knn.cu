// sc_knn.cu — Gaussian kNN graph builder (neighborhood/mod.rs). Placeholder
// until the tcgen05 distance kernel lands: reports SC_E_UNSUPPORTED.
#include "sc_prims.cuh"

namespace sc {
void knn_gaussian(Ctx&, const float*, uint64_t, uint64_t, uint64_t, const sc_knn_opts&, uint32_t*, float*,
                  uint64_t*, uint32_t*, float*, uint64_t, uint64_t*, DevGraph**) {
    fail(SC_E_UNSUPPORTED, "kNN graph builder not built yet");
}
}  // namespace sc
