// Functional connectivity: Pearson correlation of each instance's region
// series over time, the numpy.corrcoef(data.T) of the framework's
// cross-correlation analyzer
// (tvb_framework/tvb/adapters/analyzers/cross_correlation_adapter.py:348-380).
//
// One CTA per instance.  The series (T x n float64) is staged in shared
// memory, centred per region, and the n x n products are accumulated in
// float64: corr_ij = S_ij / (sqrt(S_ii) sqrt(S_jj)) with S the centred
// cross-products, clipped to [-1, 1] like numpy.corrcoef.  At the sizes of a
// sweep (T ~ 30 Bold samples, n ~ 68) one instance is ~0.3 MFLOP, so the
// contraction stays on the float64 pipes.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "tvbk.h"

namespace {

constexpr int kFcThreads = 256;
constexpr int64_t kFcMaxSmem = 200 * 1024;

__global__ void __launch_bounds__(kFcThreads) fc_kernel(const double* __restrict__ x, int T, int n,
                                                        double* __restrict__ fc) {
    extern __shared__ __align__(16) double zs[];  // [T][n] centred series, then [n] norms
    const size_t inst = blockIdx.x;
    const double* xi = x + inst * (size_t)T * n;
    double* fi = fc + inst * (size_t)n * n;
    double* norm = zs + (size_t)T * n;
    for (int k = threadIdx.x; k < T * n; k += blockDim.x) zs[k] = xi[k];
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double m = 0.0;
        for (int t = 0; t < T; ++t) m += zs[t * n + j];
        m /= (double)T;
        double ss = 0.0;
        for (int t = 0; t < T; ++t) {
            const double v = zs[t * n + j] - m;
            zs[t * n + j] = v;
            ss = fma(v, v, ss);
        }
        norm[j] = sqrt(ss);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) {
        const int a = q / n, b = q - a * n;
        if (b < a) continue;
        double s = 0.0;
        for (int t = 0; t < T; ++t) s = fma(zs[t * n + a], zs[t * n + b], s);
        double r = s / (norm[a] * norm[b]);
        if (r > 1.0) r = 1.0;
        if (r < -1.0) r = -1.0;
        fi[(size_t)a * n + b] = r;
        fi[(size_t)b * n + a] = r;
    }
}

}  // namespace

namespace tvbk {

// Shared memory bytes of the float64 FC kernel, or 0 when the series does not fit.
int64_t fc_smem_bytes(int32_t T, int32_t n) {
    const int64_t bytes = ((int64_t)T * n + n) * (int64_t)sizeof(double);
    return bytes <= kFcMaxSmem ? bytes : 0;
}

int fc_launch(const double* x, int32_t n_inst, int32_t T, int32_t n, double* fc, cudaStream_t stream) {
    const size_t smem = (size_t)fc_smem_bytes(T, n);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(fc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    fc_kernel<<<n_inst, kFcThreads, smem, stream>>>(x, T, n, fc);
    return (int)cudaGetLastError();
}

}  // namespace tvbk
