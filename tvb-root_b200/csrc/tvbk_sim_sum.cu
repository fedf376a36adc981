// Simulation kernel instantiation for the exact-propagation test model
// (dx = x + c, Linear coupling, Identity scheme).
#include "tvbk_sim_impl.cuh"

namespace tvbk {

int launch_sum(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes) {
    if (L.cfun != CF_LINEAR || L.scheme != TVBK_SCHEME_IDENTITY) return -2;
    if (L.ring_in_smem) {
        if (L.max_n > 256) return -1;
        return launch_deg<SumModel, CF_LINEAR, TVBK_SCHEME_IDENTITY, true, 256>(L, st, smem_bytes, L.max_degree);
    }
    return launch_one<SumModel, CF_LINEAR, TVBK_SCHEME_IDENTITY, false, 1024, 0>(L, st, 0);
}

}  // namespace tvbk
