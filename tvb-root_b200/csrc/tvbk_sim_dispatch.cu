// Dispatch of tvbk_sim_run to the per-model, per-scheme kernel instantiations.
#include <cuda_runtime.h>

#include "tvbk.h"

namespace tvbk {

int launch_g2d_euler_det(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_g2d_euler_stoch(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_g2d_heun_det(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_g2d_heun_stoch(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_g2d_rk4(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_rww_euler_det(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_rww_euler_stoch(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_rww_heun_det(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_rww_heun_stoch(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_rww_rk4(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_jr_euler_det(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_jr_euler_stoch(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_jr_heun_det(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_jr_heun_stoch(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_jr_rk4(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_epileptor_euler_det(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_epileptor_euler_stoch(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_epileptor_heun_det(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_epileptor_heun_stoch(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);
int launch_epileptor_rk4(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes);

int launch_g2d(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes) {
    switch (L.scheme) {
        case TVBK_SCHEME_EULER_DET: return launch_g2d_euler_det(L, st, smem_bytes);
        case TVBK_SCHEME_EULER_STOCH: return launch_g2d_euler_stoch(L, st, smem_bytes);
        case TVBK_SCHEME_HEUN_DET: return launch_g2d_heun_det(L, st, smem_bytes);
        case TVBK_SCHEME_HEUN_STOCH: return launch_g2d_heun_stoch(L, st, smem_bytes);
        case TVBK_SCHEME_RK4: return launch_g2d_rk4(L, st, smem_bytes);
        default: return -2;
    }
}

int launch_rww(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes) {
    switch (L.scheme) {
        case TVBK_SCHEME_EULER_DET: return launch_rww_euler_det(L, st, smem_bytes);
        case TVBK_SCHEME_EULER_STOCH: return launch_rww_euler_stoch(L, st, smem_bytes);
        case TVBK_SCHEME_HEUN_DET: return launch_rww_heun_det(L, st, smem_bytes);
        case TVBK_SCHEME_HEUN_STOCH: return launch_rww_heun_stoch(L, st, smem_bytes);
        case TVBK_SCHEME_RK4: return launch_rww_rk4(L, st, smem_bytes);
        default: return -2;
    }
}

int launch_jr(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes) {
    switch (L.scheme) {
        case TVBK_SCHEME_EULER_DET: return launch_jr_euler_det(L, st, smem_bytes);
        case TVBK_SCHEME_EULER_STOCH: return launch_jr_euler_stoch(L, st, smem_bytes);
        case TVBK_SCHEME_HEUN_DET: return launch_jr_heun_det(L, st, smem_bytes);
        case TVBK_SCHEME_HEUN_STOCH: return launch_jr_heun_stoch(L, st, smem_bytes);
        case TVBK_SCHEME_RK4: return launch_jr_rk4(L, st, smem_bytes);
        default: return -2;
    }
}

int launch_epileptor(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes) {
    switch (L.scheme) {
        case TVBK_SCHEME_EULER_DET: return launch_epileptor_euler_det(L, st, smem_bytes);
        case TVBK_SCHEME_EULER_STOCH: return launch_epileptor_euler_stoch(L, st, smem_bytes);
        case TVBK_SCHEME_HEUN_DET: return launch_epileptor_heun_det(L, st, smem_bytes);
        case TVBK_SCHEME_HEUN_STOCH: return launch_epileptor_heun_stoch(L, st, smem_bytes);
        case TVBK_SCHEME_RK4: return launch_epileptor_rk4(L, st, smem_bytes);
        default: return -2;
    }
}

}  // namespace tvbk
