// Sensor projection of the EEG / MEG / iEEG monitors: the lead-field product
// of tvb/simulator/monitors.py:602-614, applied to the period means that the
// simulation kernel streams out (the gain is linear, so gain . mean over a
// period equals the reference's per-step products summed and divided).
//
//     y[t][v][s] = sum_r gain[s][r] * x[t][voi[v]][r]      (float64)
//
// x is the float32 period-mean stream [T][nvoi][n] of one or many instances
// (rows of all instances stacked), gain the float64 region lead field [S][n].
// A float64 GEMM of (T * nvoi_m) x n by n x S: tcgen05 has no float64 kind,
// so it runs on the DFMA pipes.  Each CTA computes a 64 x 64 output tile with
// 256 threads (4 x 4 outputs each), staging 16-wide K slices of both
// operands in shared memory (the x slice converted to float64 and the voi
// rows gathered as it is loaded).  Every output is one sequential fma chain
// over r = 0..n-1, so a row's result does not depend on how many rows share
// the launch (a sweep's stacked instances give the same bits as one
// instance alone).
#include <cuda_runtime.h>

#include "tvbk.h"

namespace {

constexpr int kTileM = 64, kTileS = 64, kTileK = 16, kThreads = 256;

__global__ void __launch_bounds__(kThreads) project_kernel(const float* __restrict__ x, int64_t T, int nvoi, int n,
                                                           const int32_t* __restrict__ voi, int nvoi_m,
                                                           const double* __restrict__ gain, int S,
                                                           double* __restrict__ y) {
    __shared__ double As[kTileK][kTileM + 1];  // [k][row]
    __shared__ double Bs[kTileK][kTileS + 1];  // [k][sensor]
    const int64_t M = T * nvoi_m;
    const int64_t m0 = (int64_t)blockIdx.x * kTileM;
    const int s0 = blockIdx.y * kTileS;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;  // 16 x 16 threads, 4 x 4 outputs each
    double acc[4][4] = {};
    for (int k0 = 0; k0 < n; k0 += kTileK) {
        // A slice: rows m0..m0+63, regions k0..k0+15 (row m = t * nvoi_m + v reads x[t][voi[v]])
        for (int e = threadIdx.x; e < kTileM * kTileK; e += kThreads) {
            const int r = e / kTileK, k = e % kTileK;
            const int64_t m = m0 + r;
            double v = 0.0;
            if (m < M && k0 + k < n) {
                const int64_t t = m / nvoi_m;
                const int vv = (int)(m - t * nvoi_m);
                v = (double)x[(t * nvoi + voi[vv]) * (int64_t)n + k0 + k];
            }
            As[k][r] = v;
        }
        // B slice: sensors s0..s0+63, regions k0..k0+15
        for (int e = threadIdx.x; e < kTileS * kTileK; e += kThreads) {
            const int c = e / kTileK, k = e % kTileK;
            Bs[k][c] = (s0 + c < S && k0 + k < n) ? gain[(int64_t)(s0 + c) * n + k0 + k] : 0.0;
        }
        __syncthreads();
        const int kmax = min(kTileK, n - k0);
        for (int k = 0; k < kmax; ++k) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[k][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[k][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int64_t m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int s = s0 + tx * 4 + j;
            if (s < S) y[m * S + s] = acc[i][j];
        }
    }
}

}  // namespace

namespace tvbk {
int set_error(int code, const char* msg);
}

extern "C" int tvbk_project(const float* x, int64_t T, int32_t nvoi, int32_t n, const int32_t* voi, int32_t nvoi_m,
                            const double* gain, int32_t S, double* y, void* stream) {
    if (!x || !voi || !gain || !y || T < 0 || nvoi < 1 || n < 1 || nvoi_m < 1 || nvoi_m > nvoi || S < 1)
        return tvbk::set_error(TVBK_ERR_INVALID, "tvbk_project: bad arguments");
    const int64_t M = T * nvoi_m;
    if (M == 0) return TVBK_OK;
    const int64_t tiles = (M + kTileM - 1) / kTileM;
    if (tiles > 2147483647LL) return tvbk::set_error(TVBK_ERR_TOO_LARGE, "tvbk_project: too many samples");
    const dim3 grid((unsigned)tiles, (unsigned)((S + kTileS - 1) / kTileS));
    project_kernel<<<grid, kThreads, 0, (cudaStream_t)stream>>>(x, T, nvoi, n, voi, nvoi_m, gain, S, y);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return tvbk::set_error(TVBK_ERR_CUDA, cudaGetErrorString(e));
    return TVBK_OK;
}
