// Balloon-Windkessel haemodynamics: the BOLD signal of a neural-activity time
// series, in float64 (tvb_library/tvb/analyzers/fmri_balloon.py:198-364).
//
// One thread per series (an instance's region): from s = 0, f = v = q = 1 the
// thread integrates
//     ds/dt = x - s / tau_s - (f - 1) / tau_f
//     df/dt = s
//     dv/dt = (f - v^(1/alpha)) / tau_o
//     dq/dt = (f (1 - (1 - E0)^(1/f)) / E0 - v^(1/alpha) q / v) / tau_o
// with the Heun scheme the reference uses (HeunDeterministic, the input of
// step t held over both stages, integrators.py:296-318) and writes
//     nonlinear: V0 (k1 (1 - q) + k2 (1 - q / v) + k3 (1 - v))
//     linear:    V0 ((k1 + k2) (1 - q) + (k3 - k2) (1 - v))
// at every step, step 0 included.  Series are the fast index of the input
// and output ([T][nseries]), so a warp's loads and stores are coalesced.
#include <cuda_runtime.h>

#include "tvbk.h"

namespace {

struct Balloon {
    double inv_tau_s, inv_tau_f, inv_tau_o, inv_alpha, E0, V0, k1, k2, k3;
};

__device__ __forceinline__ void balloon_dfun(const Balloon& P, double x, const double* y, double* d) {
    const double s = y[0], f = y[1], v = y[2], q = y[3];
    const double va = pow(v, P.inv_alpha);
    d[0] = x - P.inv_tau_s * s - P.inv_tau_f * (f - 1.0);
    d[1] = s;
    d[2] = P.inv_tau_o * (f - va);
    d[3] = P.inv_tau_o * ((f * (1.0 - pow(1.0 - P.E0, 1.0 / f)) / P.E0) - va * (q / v));
}

__device__ __forceinline__ double balloon_bold(const Balloon& P, const double* y, bool nonlinear) {
    const double v = y[2], q = y[3];
    if (nonlinear) return P.V0 * (P.k1 * (1.0 - q) + P.k2 * (1.0 - q / v) + P.k3 * (1.0 - v));
    return P.V0 * ((P.k1 + P.k2) * (1.0 - q) + (P.k3 - P.k2) * (1.0 - v));
}

__global__ void balloon_kernel(const double* __restrict__ x, int T, int64_t ns, double dt, Balloon P, int nonlinear,
                               double* __restrict__ bold) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ns) return;
    double y[4] = {0.0, 1.0, 1.0, 1.0};
    bold[k] = balloon_bold(P, y, nonlinear != 0);
    const double hdt = dt / 2.0;
    for (int t = 1; t < T; ++t) {
        const double xt = x[(int64_t)t * ns + k];
        double m0[4], inter[4], m1[4];
        balloon_dfun(P, xt, y, m0);
#pragma unroll
        for (int j = 0; j < 4; ++j) inter[j] = y[j] + dt * (m0[j] + 0.0);
        balloon_dfun(P, xt, inter, m1);
#pragma unroll
        for (int j = 0; j < 4; ++j) y[j] = y[j] + (m0[j] + m1[j]) * hdt;
        bold[(int64_t)t * ns + k] = balloon_bold(P, y, nonlinear != 0);
    }
}

}  // namespace

namespace tvbk {
int set_error(int code, const char* msg);
}

extern "C" int tvbk_balloon(const double* x, int32_t T, int64_t nseries, double dt, const double* params,
                            int32_t nonlinear, double* bold, void* stream) {
    if (!x || !params || !bold || T < 1 || nseries < 1 || !(dt > 0.0))
        return tvbk::set_error(TVBK_ERR_INVALID, "tvbk_balloon: bad arguments");
    Balloon P;
    // params: tau_s, tau_f, tau_o, alpha, E0, V0, k1, k2, k3 (host memory)
    P.inv_tau_s = 1.0 / params[0];
    P.inv_tau_f = 1.0 / params[1];
    P.inv_tau_o = 1.0 / params[2];
    P.inv_alpha = 1.0 / params[3];
    P.E0 = params[4];
    P.V0 = params[5];
    P.k1 = params[6];
    P.k2 = params[7];
    P.k3 = params[8];
    const int threads = 128;
    const int64_t blocks = (nseries + threads - 1) / threads;
    if (blocks > 2147483647LL) return tvbk::set_error(TVBK_ERR_TOO_LARGE, "tvbk_balloon: too many series");
    balloon_kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(x, T, nseries, dt, P, nonlinear, bold);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return tvbk::set_error(TVBK_ERR_CUDA, cudaGetErrorString(e));
    return TVBK_OK;
}
