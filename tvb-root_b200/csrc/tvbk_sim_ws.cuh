// Warp-specialised variant of the row kernel (rings in shared memory).
//
// The CTA has two roles of ceil(n / 32) warps each.  Gather thread i sums
// row i of the connectome for step s + 1 (register-resident edges, the same
// branch-free gather as the row kernel) while update thread i advances region
// i through step s (noise, scheme, monitors, ring write); the sums pass
// through a shared buffer double-buffered by step parity, with one CTA
// barrier per step.  The two dependency chains that the row kernel runs one
// after the other in every thread -- the delayed-state gather and the
// per-region update -- run side by side in different warps, and the SM holds
// twice the warps.
//
// The gather of step s + 1 reads times s - d for d >= d_min >= 1, never the
// time s being written in the same iteration; with a barrier every step,
// ring_len >= horizon + 1 keeps the write of time s off every slot still to be
// read.  Needs every delay >= 1 and a coupling whose pre() ignores x_i
// (Linear, SigmoidalJansenRit) -- the conditions of the row kernel's
// prefetch.  The summation order and the arithmetic are the row kernel's (up
// to the compiler's choice of fused multiply-adds in each instantiation).
#pragma once
#include "tvbk_sim_impl.cuh"

namespace tvbk {

template <class M, int CF, int SCHEME, int MAXD>
__global__ void __launch_bounds__(512) sim_kernel_ws(const tvbk_launch L) {
    constexpr int NCV = M::NCV;
    constexpr bool SIGMA = GatherTraits<CF, NCV>::SIGMA;
    constexpr int NG = GatherTraits<CF, NCV>::NG;
    extern __shared__ __align__(16) float smem[];

    tvbk_inst* __restrict__ Ip = L.insts + blockIdx.x;
    const int n = Ip->n;
    const int WR = blockDim.x >> 1;                 // threads per role
    const bool gath = threadIdx.x >= WR;
    const int i = gath ? threadIdx.x - WR : threadIdx.x;
    const bool act = i < n;
    const int RL = Ip->ring_len;
    const int slot_floats = n * NG;
    const int ring_floats = RL * slot_floats;
    const int64_t s0 = Ip->step;
    const int64_t s_end = min(Ip->step_end, s0 + L.max_steps);
    if (s0 >= s_end) return;  // uniform over the block
    const int nsteps = (int)(s_end - s0);

    float cf[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) cf[k] = Ip->cfun[k];
    float* ring = smem;
    float* csum = smem + ((L.max_ring_len * L.max_n * NG + 3) & ~3);  // [2][n][NCV]
    if constexpr (SIGMA)
        sigma_ring(ring, Ip->ring, RL * n, threadIdx.x, blockDim.x, cf);
    else
        stage_ring(smem, Ip->ring, ring_floats);

    RegRow<M, CF, MAXD> row;
    row.deg = 0;
    Node<M, SCHEME> node;
    if (act) {
        if (gath) {
            const int e0 = Ip->row_ptr[i], e1 = Ip->row_ptr[i + 1];
            if (e1 - e0 > MAXD) atomicOr(L.status + blockIdx.x, TVBK_STATUS_DEGREE);
            row.load(Ip->edges, e0, e1);
        } else {
            node.init(L, Ip, i, n, s0);
            if (Ip->aff != nullptr) atomicOr(L.status + blockIdx.x, TVBK_STATUS_UNSUPPORTED);
        }
    }
    __syncthreads();
    int wslot = (int)(s0 % RL);  // slot of the last written time
    float xi_unused[NCV] = {};
    if (gath && act) {
        float c[NCV];
        row.couple(ring, wslot * slot_floats, ring_floats, xi_unused, cf, c);  // step s0 + 1
#pragma unroll
        for (int k = 0; k < NCV; ++k) csum[i * NCV + k] = c[k];
    }
    __syncthreads();
    for (int ks = 0; ks < nsteps; ++ks) {
        wslot = (wslot + 1 == RL) ? 0 : wslot + 1;  // time s
        if (act) {
            if (gath) {
                if (ks + 1 < nsteps) {
                    // coupling of step s + 1: times s - d with d >= d_min >= 1
                    float c[NCV];
                    row.couple(ring, wslot * slot_floats, ring_floats, xi_unused, cf, c);
                    float* out = csum + (size_t)((ks + 1) & 1) * n * NCV + i * NCV;
#pragma unroll
                    for (int k = 0; k < NCV; ++k) out[k] = c[k];
                }
            } else {
                if (STOCH_BLOCK_START(ks)) node.noise_block(L, i, s0 + 1 + ks);
                float c[NCV];
                const float* in = csum + (size_t)(ks & 1) * n * NCV + i * NCV;
#pragma unroll
                for (int k = 0; k < NCV; ++k) c[k] = in[k];
                node.advance(L, Ip, i, n, s0, ks, c);
                if constexpr (SIGMA) {
                    node.write_ring(Ip->ring + (size_t)wslot * n * NCV + i * NCV);  // raw history
                    ring[wslot * slot_floats + i] = sjr_pre(node.x[M::cvar(0)], node.x[M::cvar(1)], cf);
                } else {
                    node.write_ring(ring + wslot * slot_floats + i * NCV);
                }
            }
        }
        __syncthreads();
    }
    if (act && !gath) node.finish(L, Ip, i, n, L.status + blockIdx.x);
    if constexpr (!SIGMA) stage_ring(Ip->ring, smem, ring_floats);
    if (threadIdx.x == 0) Ip->step = s_end;
}

template <class M, int CF, int SCHEME, int MAXD>
int launch_ws_t(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes) {
    auto kern = sim_kernel_ws<M, CF, SCHEME, MAXD>;
    if (smem_bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
        if (e != cudaSuccess) return (int)e;
    }
    const int threads = 2 * (((L.max_n + 31) / 32) * 32);
    kern<<<L.n_inst, threads, smem_bytes, st>>>(L);
    return (int)cudaGetLastError();
}

template <class M, int CF, int SCHEME>
int launch_ws(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes) {
    if constexpr (CF == CF_DIFFERENCE) {
        return -2;
    } else {
        if (!L.ring_in_smem || L.max_n > 256) return -1;
        if (L.max_degree <= 32) return launch_ws_t<M, CF, SCHEME, 32>(L, st, smem_bytes);
        if (L.max_degree <= 64) return launch_ws_t<M, CF, SCHEME, 64>(L, st, smem_bytes);
        return -1;
    }
}

}  // namespace tvbk
