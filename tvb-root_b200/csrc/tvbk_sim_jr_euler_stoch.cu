// Simulation kernel instantiations for JansenRit with scheme TVBK_SCHEME_EULER_STOCH.
#include "tvbk_sim_lanes.cuh"

namespace tvbk {

int launch_jr_euler_stoch(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes) {
    switch (L.cfun) {
        case CF_LINEAR: return launch_all_scheme<JansenRit, CF_LINEAR, TVBK_SCHEME_EULER_STOCH>(L, st, smem_bytes);
        case CF_DIFFERENCE: return launch_all_scheme<JansenRit, CF_DIFFERENCE, TVBK_SCHEME_EULER_STOCH>(L, st, smem_bytes);
        case CF_SIGMOIDAL_JR: return launch_all_scheme<JansenRit, CF_SIGMOIDAL_JR, TVBK_SCHEME_EULER_STOCH>(L, st, smem_bytes);
        case TVBK_CFUN_SIGMOIDAL:
        case TVBK_CFUN_HYPERBOLIC_TANGENT:
        case TVBK_CFUN_KURAMOTO: return launch_all_scheme<JansenRit, CF_GENERIC, TVBK_SCHEME_EULER_STOCH>(L, st, smem_bytes);
        default: return -2;
    }
}

}  // namespace tvbk
