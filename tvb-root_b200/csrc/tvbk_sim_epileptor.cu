// Simulation kernel instantiations for Epileptor.
#include "tvbk_sim_impl.cuh"

namespace tvbk {

int launch_epileptor(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes) {
    switch (L.cfun) {
        case CF_LINEAR: return launch_cfun<Epileptor, CF_LINEAR>(L, st, smem_bytes, L.max_degree);
        case CF_DIFFERENCE: return launch_cfun<Epileptor, CF_DIFFERENCE>(L, st, smem_bytes, L.max_degree);
        case CF_SIGMOIDAL_JR: return launch_cfun<Epileptor, CF_SIGMOIDAL_JR>(L, st, smem_bytes, L.max_degree);
        default: return -2;
    }
}

}  // namespace tvbk
