// Instance-group variant of the simulation kernel for parameter sweeps.
//
// A CTA advances a group of G instances that share connectome, ring length
// and step range.  Thread (region i, lane v) advances region i of instance
// g*G + v; the group's rings are interleaved [ring_len][n][ncvar][G] in
// global memory, G * ncvar * 4 = 32 bytes per (slot, region), so the G lanes
// of a region read one full 32-byte sector per edge and L2 / DRAM traffic
// equals the algorithmic gather bytes.  Rings stay out of shared memory
// (which holds the group's edge list and the gather staging buffers), so
// every instance of a sweep can be resident at once.
//
// Group g is instances [g*G, g*G + G) of the launch; the group's ring is the
// `ring` of its first instance.  Per-instance parameters, coupling
// parameters, noise streams, states and monitors stay per instance.
#pragma once
#include <cuda_pipeline.h>

#include "tvbk_sim_cluster.cuh"
#include "tvbk_sim_ws.cuh"
#include "tvbk_sim_impl.cuh"

namespace tvbk {

// Bytes of the group kernel's shared edge list (>= nnz of every instance).
__host__ __device__ inline size_t group_edge_bytes(int max_n, int max_degree) {
    return ((size_t)max_n * max_degree * sizeof(int2) + 15) & ~(size_t)15;
}

// Shared memory of the group kernel: edge list + two staging buffers of
// max_degree * ncvar floats per thread.
inline size_t group_smem_bytes(int max_n, int max_degree, int ncvar, int threads) {
    return group_edge_bytes(max_n, max_degree) + (size_t)2 * max_degree * ncvar * threads * sizeof(float);
}

// The delayed values of step s are copied global -> shared with cp.async
// (one 4-byte copy per edge and coupling variable, straight into this
// thread's staging slots, no registers held while in flight) and consumed
// after __pipeline_wait_prior.  With PIPE the copies for step s + 1 are
// issued before the wait for step s (they read times <= s - d_min), so the
// L2 latency overlaps a whole step; without it (some delay is 0) they are
// issued and awaited within the step.
template <class M, int CF, int SCHEME, int G, bool PIPE, int MAXT>
__global__ void __launch_bounds__(MAXT) sim_kernel_group(const tvbk_launch L) {
    constexpr int NCV = M::NCV;
    constexpr int W = NCV * G;  // floats per (slot, region)
    extern __shared__ __align__(16) unsigned char sm[];
    int2* esm = reinterpret_cast<int2*>(sm);  // the group's edges, staged once per launch
    float* stage = reinterpret_cast<float*>(sm + group_edge_bytes(L.max_n, L.max_degree));  // [2][maxdeg*NCV][T]
    const int SD = L.max_degree * NCV;  // staging slots per thread and buffer

    tvbk_inst* __restrict__ I0 = L.insts + (size_t)blockIdx.x * G;
    const int n = I0->n;
    const int T = blockDim.x;
    const int v = threadIdx.x % G;
    const int i = threadIdx.x / G;
    const bool act = i < n;
    tvbk_inst* __restrict__ Ip = I0 + v;
    const int RL = I0->ring_len;
    const int slot_floats = n * W;
    const int ring_floats = RL * slot_floats;
    const int64_t s0 = I0->step;
    const int64_t s_end = min(I0->step_end, s0 + L.max_steps);
    if (s0 >= s_end) return;  // uniform over the block
    const int nsteps = (int)(s_end - s0);
    const float* __restrict__ ring_r = I0->ring;
    float* __restrict__ ring = I0->ring;

    float cf[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) cf[k] = Ip->cfun[k];
    // edges in shared memory, offsets rescaled to the group layout: (d*n - j)*ncvar*G
    const int nnz = I0->nnz;
    {
        const int2* ed2 = reinterpret_cast<const int2*>(I0->edges);
        for (int e = threadIdx.x; e < nnz; e += T) {
            const int2 ed = __ldg(ed2 + e);
            esm[e] = make_int2(ed.x * G, ed.y);
        }
    }
    int e0 = 0, deg = 0;
    Node<M, SCHEME> node;
    if (act) {
        e0 = I0->row_ptr[i];
        deg = I0->row_ptr[i + 1] - e0;
        if (deg > L.max_degree) atomicOr(L.status + (size_t)blockIdx.x * G + v, TVBK_STATUS_DEGREE);
        deg = min(deg, L.max_degree);
        node.init(L, Ip, i, n, s0);
        if (Ip->aff != nullptr) atomicOr(L.status + (size_t)blockIdx.x * G + v, TVBK_STATUS_UNSUPPORTED);
    }
    __syncthreads();

    // copy the delayed values of row i's edges for the step whose time s - 1 is in `slot` into buffer `buf`
    auto issue = [&](int slot, int buf) {
        const int base_off = slot * slot_floats + v;
        float* dst = stage + (size_t)buf * SD * T + threadIdx.x;
        const int2* ed = esm + e0;
#pragma unroll 4
        for (int k = 0; k < deg; ++k) {
            const int a = gather_addr(base_off, ed[k].x, ring_floats);
#pragma unroll
            for (int q = 0; q < NCV; ++q)
                __pipeline_memcpy_async(dst + (size_t)(k * NCV + q) * T, ring_r + a + q * G, sizeof(float));
        }
        __pipeline_commit();
    };
    auto consume = [&](int buf, float* c, const float* xi) {
        const float* src = stage + (size_t)buf * SD * T + threadIdx.x;
        const int2* ed = esm + e0;
        float a0[NCV], a1[NCV];
#pragma unroll
        for (int q = 0; q < NCV; ++q) a0[q] = a1[q] = 0.0f;
        int k = 0;
        for (; k + 1 < deg; k += 2) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const float wk = __int_as_float(ed[k + h].y);
                float val[NCV];
#pragma unroll
                for (int q = 0; q < NCV; ++q) val[q] = src[(size_t)((k + h) * NCV + q) * T];
                float* acc = h ? a1 : a0;
                if constexpr (CF == CF_SIGMOIDAL_JR) {
                    const float pre = cf[0] + (cf[1] - cf[0]) / (1.0f + expf(cf[3] * (cf[2] - (val[0] - val[1]))));
                    acc[0] = fmaf(wk, pre, acc[0]);
                } else {
#pragma unroll
                    for (int q = 0; q < NCV; ++q) {
                        const float pre = (CF == CF_DIFFERENCE) ? val[q] - xi[q] : val[q];
                        acc[q] = fmaf(wk, pre, acc[q]);
                    }
                }
            }
        }
        if (k < deg) {
            const float wk = __int_as_float(ed[k].y);
            float val[NCV];
#pragma unroll
            for (int q = 0; q < NCV; ++q) val[q] = src[(size_t)(k * NCV + q) * T];
            if constexpr (CF == CF_SIGMOIDAL_JR) {
                const float pre = cf[0] + (cf[1] - cf[0]) / (1.0f + expf(cf[3] * (cf[2] - (val[0] - val[1]))));
                a0[0] = fmaf(wk, pre, a0[0]);
            } else {
#pragma unroll
                for (int q = 0; q < NCV; ++q) {
                    const float pre = (CF == CF_DIFFERENCE) ? val[q] - xi[q] : val[q];
                    a0[q] = fmaf(wk, pre, a0[q]);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NCV; ++q) a0[q] += a1[q];
        post<CF, NCV>(a0, cf, c);
    };

    const int K = L.sync_every;
    int since_sync = 0;
    int wslot = (int)(s0 % RL);  // slot of the last written time
    int buf = 0;
    if (PIPE && act) issue(wslot, 0);
    for (int ks = 0; ks < nsteps; ++ks) {
        const int prev = wslot;                     // slot of time s - 1
        wslot = (wslot + 1 == RL) ? 0 : wslot + 1;  // time s
        if (act) {
            if (STOCH_BLOCK_START(ks)) node.noise_block(L, i, s0 + 1 + ks);
            if constexpr (PIPE) {
                issue(wslot, buf ^ 1);      // step s + 1 reads times <= s - d_min
                __pipeline_wait_prior(1);   // this step's copies have landed
            } else {
                issue(prev, buf);
                __pipeline_wait_prior(0);
            }
            float xi[NCV];
#pragma unroll
            for (int q = 0; q < NCV; ++q) xi[q] = node.x[M::cvar(q)];
            float c[NCV];
            consume(buf, c, xi);
            node.advance(L, Ip, i, n, s0, ks, c);
            float* dst = ring + wslot * slot_floats + i * W + v;
#pragma unroll
            for (int q = 0; q < NCV; ++q) dst[q * G] = node.x[M::cvar(q)];
            if (PIPE) buf ^= 1;
        }
        if (++since_sync == K) {
            since_sync = 0;
            __syncthreads();
        }
    }
    __pipeline_wait_prior(0);
    __syncthreads();
    if (act) node.finish(L, Ip, i, n, L.status + (size_t)blockIdx.x * G + v);
    if (threadIdx.x < G) I0[threadIdx.x].step = s_end;
}

template <class M, int CF, int SCHEME, int G, bool PIPE, int MAXT>
int launch_group_t(const tvbk_launch& L, cudaStream_t st, int threads) {
    auto kern = sim_kernel_group<M, CF, SCHEME, G, PIPE, MAXT>;
    const size_t smem = group_smem_bytes(L.max_n, L.max_degree, M::NCV, threads);
    if (smem > 48 * 1024) {
        if (smem > 227 * 1024) return -1;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    kern<<<L.n_inst / G, threads, smem, st>>>(L);
    return (int)cudaGetLastError();
}

// Launch bounds by CTA size, so that smaller CTAs get more registers per thread.
template <class M, int CF, int SCHEME, int G, bool PIPE>
int launch_group_one(const tvbk_launch& L, cudaStream_t st) {
    const int threads = ((L.max_n * G + 31) / 32) * 32;
    if (threads <= 384) return launch_group_t<M, CF, SCHEME, G, PIPE, 384>(L, st, threads);
    if (threads <= 768) return launch_group_t<M, CF, SCHEME, G, PIPE, 768>(L, st, threads);
    if (threads <= 1024) return launch_group_t<M, CF, SCHEME, G, PIPE, 1024>(L, st, threads);
    return -1;
}

template <class M, int CF, int SCHEME>
int launch_group(const tvbk_launch& L, cudaStream_t st, int max_deg) {
    constexpr int G = 8 / M::NCV;
    if (L.lanes != G) return -1;
    if (L.prefetch) return launch_group_one<M, CF, SCHEME, G, true>(L, st);
    return launch_group_one<M, CF, SCHEME, G, false>(L, st);
}

// Dispatch on the launch's variant for one scheme: instance groups, clusters
// of CTAs per instance, else the row / edge-parallel kernels.
template <class M, int CF, int SCHEME>
int launch_all_scheme(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes) {
    if constexpr (CF == CF_GENERIC) {
        // run-time chosen couplings: the row kernel, one step at a time
        if (L.lanes > 1 || L.cluster > 1 || L.prefetch != 0) return -2;
    } else {
        if (L.lanes > 1) return launch_group<M, CF, SCHEME>(L, st, L.max_degree);
        if (L.cluster > 1) return launch_cluster<M, CF, SCHEME>(L, st);
        if (L.prefetch == 2) return launch_ws<M, CF, SCHEME>(L, st, smem_bytes);
    }
    return launch_scheme<M, CF, SCHEME>(L, st, smem_bytes, L.max_degree);
}

}  // namespace tvbk
