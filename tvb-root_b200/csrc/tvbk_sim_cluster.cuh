// Cluster variant of the simulation kernel for large instances.
//
// One instance is advanced by a thread-block cluster of C CTAs (C = the
// launch's `cluster`, 2..16).  CTA r of the cluster owns the rows (target
// regions) [r*R, min(n, r*R + R)), R = ceil(n / C): it keeps those rows'
// edges in shared memory, computes their coupling sums, and advances their
// regions.  The history ring stays in global memory (L2 / HBM) and is read
// with L2-coherent loads (ld.global.cg).
//
// Per step, within a CTA:
//   * gather warps: one warp per row at a time -- the 32 lanes take the
//     row's edges strided by 32 (coalesced edge reads, independent ring
//     loads), accumulate w * pre(x_i, x_j(t - d)) and reduce with warp
//     shuffles; rows are taken four at a time so that up to 4 * MAXE loads
//     per lane are in flight.  The sums go to a shared buffer, double
//     buffered by step parity.
//   * update warps (the first ceil(R / 32); thread t advances row r*R + t):
//     post(), the scheme step with noise, the ring write and the monitors --
//     the same per-region code as the single-CTA kernel.
// For SigmoidalJansenRit the gather reads a ring of pre-applied sigmoid
// values (GatherTraits), recomputed from the raw ring at the start of a launch
// and written beside it every step.
// With PIPE (every delay >= 1 and barrier interval K <= d_min), the gather
// warps compute the sums of step s + 1 while the update warps advance step
// s: that gather reads times <= s - d_min only.  Without it every warp
// gathers, then the update warps advance, in the same step.
//
// Across the cluster, ring writes become visible to the other CTAs at a
// cluster barrier (arrive.release / wait.acquire) every K steps.  Within a
// window of K <= d_min (PIPE) or K <= d_min + 1 steps no CTA reads a time
// written in the window, and ring_len >= horizon + K keeps every write of
// the window off slots still to be read, as in the single-CTA kernel.
#pragma once
#include <cooperative_groups.h>

#include "tvbk_sim_impl.cuh"

namespace tvbk {

namespace cgx = cooperative_groups;

constexpr int kClusterThreads = 512;
constexpr int kClusterRowsPerPass = 4;
// edges whose four-step windows a blocked-run gather thread requests together (one for eight-step blocks)
constexpr int kClusterBlockBatch = 2;
// edges whose values an edge-run gather thread (one step per gather) requests together
constexpr int kClusterRunBatch = 4;

__host__ __device__ inline int cluster_rows(int n, int C) { return (n + C - 1) / C; }

// CTA barrier 1 over nthreads threads (a multiple of 32), for warp-uniform
// roles that reach it from different loops; it orders memory like
// __syncthreads.
__device__ __forceinline__ void cta_barrier_all(int nthreads) {
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

// Cluster barrier (release on arrival, acquire on wait), in its form that
// may be reached from different places of the code.
__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// 32-byte load through L2 (ld.global.cg.v8.f32, sm_100 and later); p is
// 32-byte aligned.  The second form loads only when `on` and otherwise leaves
// v as it was.
__device__ __forceinline__ void ldcg32(const float* p, float (&v)[8]) {
    asm volatile("ld.global.cg.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
                 : "l"(p)
                 : "memory");
}

__device__ __forceinline__ void ldcg32_if(bool on, const float* p, float (&v)[8]) {
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %9, 0;\n\t"
        "@q ld.global.cg.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n\t}"
        : "+f"(v[0]), "+f"(v[1]), "+f"(v[2]), "+f"(v[3]), "+f"(v[4]), "+f"(v[5]), "+f"(v[6]), "+f"(v[7])
        : "l"(p), "r"((int)on)
        : "memory");
}

// Longest wait of one group barrier (all CTAs of a cooperative launch are
// resident, so a wait this long means the launch cannot go on).
constexpr uint64_t kGroupWaitNs = 4000000000ull;

// Group barrier, one thread per CTA: arrive on the group's counter, then wait
// until it reaches `target` (the group's CTAs x the barriers passed so far).
// Returns 0 when the launch is abandoned: the abort flag is set, or this wait
// ran past kGroupWaitNs (then this thread sets the flag, and every other wait
// of the launch returns 0 at its next poll).
__device__ __forceinline__ int group_arrive_wait(uint32_t* count, uint32_t target, uint32_t* abort_flag) {
    __threadfence();  // this CTA's ring writes, ordered before the arrival by the CTA barrier before the call
    atomicAdd(count, 1u);
    const uint64_t t0 = globaltimer_ns();
    for (;;) {
        if ((int32_t)(ld_acquire_gpu(count) - target) >= 0) break;
        if (ld_acquire_gpu(abort_flag) != 0u) return 0;
        if (globaltimer_ns() - t0 > kGroupWaitNs) {
            atomicExch(abort_flag, 1u);
            return 0;
        }
        __nanosleep(32);
    }
    __threadfence();
    return 1;
}

// Shared memory of the edge-run variant: row pointers, then the double-buffered
// partials ([2][threads][2][ng] floats), then the CTA's edges.
__host__ __device__ inline size_t cluster_runs_head_rp(int R) { return ((size_t)(R + 1) * 4 + 15) / 16 * 16; }
__host__ __device__ inline size_t cluster_runs_head(int R, int ng, int threads) {
    return cluster_runs_head_rp(R) + ((size_t)2 * threads * 2 * ng * 4 + 15) / 16 * 16;
}
// the blocked variant keeps the partials of a block of B steps: [2][B][2][ng][threads] floats
__host__ __device__ inline size_t cluster_blocks_head(int R, int ng, int threads, int B) {
    return cluster_runs_head_rp(R) + ((size_t)2 * B * threads * 2 * ng * 4 + 15) / 16 * 16;
}

// Shared memory of one cluster CTA: row pointers, the double-buffered sums
// and (when they fit) the CTA's edges.
__host__ __device__ inline size_t cluster_smem_head(int R, int nacc) {
    return ((size_t)(R + 1) * 4 + 15) / 16 * 16 + ((size_t)2 * R * nacc * 4 + 15) / 16 * 16;
}

template <int NCV>
__device__ __forceinline__ void load_cg(const float* p, float* v) {
    if constexpr (NCV == 1) {
        v[0] = __ldcg(p);
    } else {
        const float2 t = __ldcg(reinterpret_cast<const float2*>(p));
        v[0] = t.x;
        v[1] = t.y;
    }
}

template <int CF, int NCV, int NACC>
__device__ __forceinline__ void accumulate_v(float* acc, float w, const float* v, const float* xi, const float* cf) {
    if constexpr (CF == CF_SIGMOIDAL_JR) {
        const float pre = cf[0] + (cf[1] - cf[0]) / (1.0f + expf(cf[3] * (cf[2] - (v[0] - v[1]))));
        acc[0] = fmaf(w, pre, acc[0]);
    } else {
#pragma unroll
        for (int q = 0; q < NCV; ++q) acc[q] = fmaf(w, (CF == CF_DIFFERENCE) ? v[q] - xi[q] : v[q], acc[q]);
    }
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// EXT = false: built without the region stimulus and the projection stream
// (launch.extras == 0), whose per-thread state would otherwise spill here.
template <class M, int CF, int SCHEME, int MAXE, bool PIPE, bool EXT = true>
__global__ void __launch_bounds__(kClusterThreads, 1) sim_kernel_cluster(const tvbk_launch L) {
    constexpr int NCV = M::NCV;
    constexpr int NACC = (CF == CF_SIGMOIDAL_JR) ? 1 : NCV;
    constexpr bool SIGMA = GatherTraits<CF, NCV>::SIGMA;
    constexpr int NG = GatherTraits<CF, NCV>::NG, GCF = GatherTraits<CF, NCV>::GCF;
    constexpr int RP = kClusterRowsPerPass;
    extern __shared__ __align__(16) unsigned char sm[];
    cgx::cluster_group cluster = cgx::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    // this cluster's instance: the launch may order the instances through inst_order (longest first)
    const int inst = L.inst_order != nullptr ? L.inst_order[blockIdx.x / C] : (int)(blockIdx.x / C);
    tvbk_inst* __restrict__ Ip = L.insts + inst;
    int32_t* status = L.status + inst;
    const int n = Ip->n;
    const int R = cluster_rows(n, C);
    const int r0 = min(n, rank * R), r1 = min(n, r0 + R), nr = r1 - r0;
    const int RL = Ip->ring_len;
    const int slot_floats = n * NG;  // the gather ring: NG floats per (slot, region)
    const int ring_floats = RL * slot_floats;
    const int64_t s0 = Ip->step;
    const int64_t s_end = min(Ip->step_end, s0 + L.max_steps);
    if (s0 >= s_end) return;  // uniform over the cluster
    const int nsteps = (int)(s_end - s0);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, W = blockDim.x >> 5;

    int* rp = reinterpret_cast<int*>(sm);
    float* csum = reinterpret_cast<float*>(sm + ((size_t)(R + 1) * 4 + 15) / 16 * 16);
    int2* esm = reinterpret_cast<int2*>(sm + cluster_smem_head(R, NACC));
    const int e_lo = Ip->row_ptr[r0], e_hi = Ip->row_ptr[r1];
    const int ne = e_hi - e_lo;
    const int2* eg = reinterpret_cast<const int2*>(Ip->edges) + e_lo;
    // the CTA's edges in shared memory when they fit the launch's allowance, else read from global
    const bool e_in_smem = ne <= L.cluster_edges;
    const int2* ed = e_in_smem ? esm : eg;
    for (int k = tid; k <= nr; k += blockDim.x) rp[k] = Ip->row_ptr[r0 + k] - e_lo;
    if (e_in_smem)
        for (int k = tid; k < ne; k += blockDim.x) esm[k] = __ldg(eg + k);

    float cf[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) cf[k] = Ip->cfun[k];
    const int U = (nr + 31) >> 5;                  // update warps
    const int G0 = PIPE ? U : 0;                   // first gather warp
    const int G = PIPE ? W - U : W;                // gather warps
    const bool upd = tid < nr;
    Node<M, SCHEME, EXT> node;
    if (upd) {
        node.init(L, Ip, r0 + tid, n, s0);
        if (Ip->row_ptr[r0 + tid + 1] - Ip->row_ptr[r0 + tid] > 32 * MAXE) atomicOr(status, TVBK_STATUS_DEGREE);
        if (Ip->aff != nullptr || (!EXT && (Ip->stim != nullptr || Ip->proj != nullptr)))
            atomicOr(status, TVBK_STATUS_UNSUPPORTED);
    }
    float* __restrict__ raw = Ip->ring;
    // gather ring: the raw ring, or for SigmoidalJansenRit the pre-applied sigmoid values, recomputed from
    // the raw ring at every launch (split over the cluster, visible to all of it after the cluster barrier)
    float* __restrict__ ring = SIGMA ? Ip->pre_ring : raw;
    if constexpr (SIGMA) {
        sigma_ring(ring, raw, RL * n, rank * blockDim.x + tid, C * blockDim.x, cf);
        cluster.sync();
    } else {
        __syncthreads();
    }

    // coupling sums of the step whose time s - 1 is in slot `prev`, into csum[buf]
    auto gather = [&](int prev, int buf) {
        const int base_off = prev * slot_floats;
        float* out = csum + (size_t)buf * R * NACC;
        for (int first = warp - G0; first < nr; first += G * RP) {
            float acc[RP][NACC];
#pragma unroll
            for (int h = 0; h < RP; ++h) {
#pragma unroll
                for (int q = 0; q < NACC; ++q) acc[h][q] = 0.0f;
                const int lr = first + h * G;
                if (lr < nr) {  // uniform over the warp
                    float xi[NCV];
                    if constexpr (CF == CF_DIFFERENCE) load_cg<NCV>(ring + base_off + (r0 + lr) * NCV, xi);
                    const int eb = rp[lr], ee = rp[lr + 1];
#pragma unroll
                    for (int k = 0; k < MAXE; ++k) {
                        const int e = eb + lane + 32 * k;
                        if (e < ee) {
                            const int2 p = ed[e];
                            float v[NG];
                            load_cg<NG>(ring + gather_addr(base_off, p.x, ring_floats), v);
                            accumulate_v<GCF, NG, NACC>(acc[h], __int_as_float(p.y), v, xi, cf);
                        }
                    }
                }
            }
#pragma unroll
            for (int h = 0; h < RP; ++h) {
                const int lr = first + h * G;
                if (lr < nr) {
#pragma unroll
                    for (int q = 0; q < NACC; ++q) {
                        const float t = warp_sum(acc[h][q]);
                        if (lane == 0) out[lr * NACC + q] = t;
                    }
                }
            }
        }
    };
    auto update = [&](int ks, int wslot, int buf) {
        const float* in = csum + (size_t)buf * R * NACC;
        float a[NACC], c[NCV];
#pragma unroll
        for (int q = 0; q < NACC; ++q) a[q] = in[tid * NACC + q];
        post<CF, NCV>(a, cf, c);
        if (STOCH_BLOCK_START(ks)) node.noise_block(L, r0 + tid, s0 + 1 + ks);
        node.advance(L, Ip, r0 + tid, n, s0, ks, c);
        node.write_ring(raw + (size_t)wslot * n * NCV + (r0 + tid) * NCV);
        if constexpr (SIGMA)
            ring[wslot * slot_floats + r0 + tid] = sjr_pre(node.x[M::cvar(0)], node.x[M::cvar(1)], cf);
    };

    const int K = L.sync_every;
    int since_sync = 0;
    int wslot = (int)(s0 % RL);  // slot of the last written time
    if constexpr (PIPE) {
        if (warp >= G0) gather(wslot, 0);
        __syncthreads();
    }
    for (int ks = 0; ks < nsteps; ++ks) {
        const int prev = wslot;
        wslot = (wslot + 1 == RL) ? 0 : wslot + 1;
        if constexpr (PIPE) {
            if (warp < U) {
                if (upd) update(ks, wslot, ks & 1);
            } else if (ks + 1 < nsteps) {
                gather(wslot, (ks + 1) & 1);  // step s + 1: times <= s - d_min
            }
            __syncthreads();
        } else {
            gather(prev, 0);
            __syncthreads();
            if (upd) update(ks, wslot, 0);
            __syncthreads();
        }
        if (++since_sync == K) {
            since_sync = 0;
            cluster.sync();
        }
    }
    cluster.sync();
    if (upd) node.finish(L, Ip, r0 + tid, n, status);
    if (rank == 0 && tid == 0) Ip->step = s_end;
}

// Edge-run variant of the cluster kernel (launch.edges_per_thread = E > 0).
// The CTA's edges, in CSR order and staged in shared memory, are cut into
// runs of E consecutive edges, one run per gather thread.  With E at most the
// smallest non-zero row degree of the CTA a run holds edges of at most two
// rows -- its first row (partial a) and the next row with edges (partial b) --
// so every thread issues E independent ring loads per step with no lane idle
// beyond the last run, instead of a warp per row whose lanes run out of
// edges unevenly.  The update thread of row r adds the partials of the runs
// covering r in run order (a fixed order: the result does not depend on
// timing).  Difference, w (x_j - x_i), is summed as sum_j w x_j - x_i sum_j w
// with the row's weight sum W taken once in CSR order, so the gather needs no
// x_i and, with PIPE, runs one step ahead like the other couplings.
template <class M, int CF, int SCHEME, int E, bool PIPE, bool EXT = true>
__global__ void __launch_bounds__(kClusterThreads, 1) sim_kernel_cluster_runs(const tvbk_launch L) {
    constexpr int NCV = M::NCV;
    constexpr bool SIGMA = GatherTraits<CF, NCV>::SIGMA;
    constexpr int NG = GatherTraits<CF, NCV>::NG;  // floats per gathered value and partial sums per run half
    extern __shared__ __align__(16) unsigned char sm[];
    cgx::cluster_group cluster = cgx::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    // this cluster's instance: the launch may order the instances through inst_order (longest first)
    const int inst = L.inst_order != nullptr ? L.inst_order[blockIdx.x / C] : (int)(blockIdx.x / C);
    tvbk_inst* __restrict__ Ip = L.insts + inst;
    int32_t* status = L.status + inst;
    const int n = Ip->n;
    const int R = cluster_rows(n, C);
    const int r0 = min(n, rank * R), r1 = min(n, r0 + R), nr = r1 - r0;
    const int RL = Ip->ring_len;
    const int slot_floats = n * NG;
    const int ring_floats = RL * slot_floats;
    const int64_t s0 = Ip->step;
    const int64_t s_end = min(Ip->step_end, s0 + L.max_steps);
    if (s0 >= s_end) return;  // uniform over the cluster
    const int nsteps = (int)(s_end - s0);
    const int tid = threadIdx.x;
    const int U = (nr + 31) >> 5;       // update warps
    const int T0 = PIPE ? 32 * U : 0;   // first gather thread
    const int Tg = blockDim.x - T0;     // gather threads

    int* rp = reinterpret_cast<int*>(sm);
    float* part = reinterpret_cast<float*>(sm + cluster_runs_head_rp(R));            // [2][2 NG][blockDim]
    int2* esm = reinterpret_cast<int2*>(sm + cluster_runs_head(R, NG, blockDim.x));  // the CTA's edges, interleaved
    const int e_lo = Ip->row_ptr[r0], e_hi = Ip->row_ptr[r1];
    const int ne = e_hi - e_lo;
    // the runs must cover the CTA's edges and fit the launch's shared-memory allowance (planned on the host);
    // a CTA whose edges do not fit flags the instance and takes part in every barrier without doing any work
    // (no early return: the other CTAs of the cluster wait for it at the cluster barriers)
    const bool fits = ne <= L.cluster_edges && ne <= Tg * E;
    if (!fits && tid == 0) atomicOr(status, TVBK_STATUS_DEGREE);
    const int2* eg = reinterpret_cast<const int2*>(Ip->edges) + e_lo;
    for (int k = tid; k <= nr; k += blockDim.x) rp[k] = Ip->row_ptr[r0 + k] - e_lo;
    // edge e (CSR order) is edge k = e % E of run g = e / E, kept at slot k * nrun + g: at every k the threads
    // of a warp read consecutive 8-byte words (one wavefront), where runs side by side would all read one bank
    const int nrun = (ne + E - 1) / E;
    auto eslot = [&](int e) { return (e % E) * nrun + e / E; };
    if (fits)
        for (int e = tid; e < ne; e += blockDim.x) esm[eslot(e)] = __ldg(eg + e);

    float cf[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) cf[k] = Ip->cfun[k];
    const bool upd = fits && tid < nr;
    Node<M, SCHEME, EXT> node;
    if (upd) {
        node.init(L, Ip, r0 + tid, n, s0);
        if (Ip->aff != nullptr || (!EXT && (Ip->stim != nullptr || Ip->proj != nullptr)))
            atomicOr(status, TVBK_STATUS_UNSUPPORTED);
    }
    float* __restrict__ raw = Ip->ring;
    float* __restrict__ ring = SIGMA ? Ip->pre_ring : raw;
    if constexpr (SIGMA) {
        sigma_ring(ring, raw, RL * n, rank * blockDim.x + tid, C * blockDim.x, cf);
        cluster.sync();
    } else {
        __syncthreads();
    }

    // this thread's run: edges [eb, eb + cnt), the first kb of them in its first row
    const int g = tid - T0;
    const int eb = g * E;
    const int cnt = (fits && g >= 0) ? max(0, min(E, ne - eb)) : 0;
    int kb = cnt;
    if (cnt > 0) {
        int lo = 0, hi = nr - 1;  // the row of edge eb: the largest lr with rp[lr] <= eb
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (rp[mid] <= eb) lo = mid; else hi = mid - 1;
        }
        kb = min(rp[lo + 1] - eb, cnt);
        if (kb < cnt) {  // the rest must lie in one row: the next one with edges
            int r2 = lo + 1;
            while (rp[r2 + 1] == rp[r2]) ++r2;
            if (rp[r2 + 1] < eb + cnt) atomicOr(status, TVBK_STATUS_DEGREE);
        }
    }
    // which partials make up row tid (update threads): half sf of run tf, then half a of runs tf+1 .. tl;
    // for Difference also the row's weight sum
    int tf = -1, sf = 0, tl = -1;
    float wsum = 0.0f;
    if (upd && rp[tid + 1] > rp[tid]) {
        tf = rp[tid] / E;
        sf = (rp[tid] == tf * E) ? 0 : 1;
        tl = (rp[tid + 1] - 1) / E;
        if constexpr (CF == CF_DIFFERENCE)
            for (int e = rp[tid]; e < rp[tid + 1]; ++e) wsum += __int_as_float(esm[eslot(e)].y);
    }
    __syncthreads();

    const size_t half = (size_t)blockDim.x * 2 * NG;  // floats of one buffer of partials: [2 NG][blockDim]
    const int TB = blockDim.x;
    // The edges go in batches of kClusterRunBatch whose loads are all issued before the first is used (one
    // L2 round trip per batch); slots past the run's count read region 0 at time prev and add nothing.  One
    // set of sums serves both rows of a run: at the second row's first edge (kb) the first row's sums go to
    // partial 0.
    auto gather = [&](int prev, int buf) {
        constexpr int BE = kClusterRunBatch;
        const int base_off = prev * slot_floats;
        float* out = part + buf * half + g;
        float pa[NG];
#pragma unroll
        for (int q = 0; q < NG; ++q) pa[q] = 0.0f;
#pragma unroll
        for (int k0 = 0; k0 < E; k0 += BE) {
            if (k0 < cnt) {
                float v[BE][NG];
                float wv[BE];
#pragma unroll
                for (int j = 0; j < BE; ++j) {
                    const int k = k0 + j;
                    const int2 ed = k < cnt ? esm[k * nrun + g] : make_int2(0, 0);
                    wv[j] = __int_as_float(ed.y);
                    load_cg<NG>(ring + gather_addr(base_off, ed.x, ring_floats), v[j]);
                }
#pragma unroll
                for (int j = 0; j < BE; ++j) {
                    const int k = k0 + j;
                    if (k < cnt) {
                        if (k == kb) {
#pragma unroll
                            for (int q = 0; q < NG; ++q) {
                                out[q * TB] = pa[q];
                                pa[q] = 0.0f;
                            }
                        }
#pragma unroll
                        for (int q = 0; q < NG; ++q) pa[q] = fmaf(wv[j], v[j][q], pa[q]);
                    }
                }
            }
        }
        // the last row's sums: partial 1 when the run holds a second row (partial 1 of a run without one is
        // never read), else partial 0
        const int h = kb < cnt ? 1 : 0;
#pragma unroll
        for (int q = 0; q < NG; ++q) out[(h * NG + q) * TB] = pa[q];
    };
    auto update = [&](int ks, int wslot, int buf) {
        const float* in = part + buf * half;
        float a[NG], c[NCV];
#pragma unroll
        for (int q = 0; q < NG; ++q) a[q] = 0.0f;
        if (tf >= 0) {
#pragma unroll
            for (int q = 0; q < NG; ++q) a[q] = in[(size_t)(sf * NG + q) * TB + tf];
            for (int u = tf + 1; u <= tl; ++u) {
#pragma unroll
                for (int q = 0; q < NG; ++q) a[q] += in[(size_t)q * TB + u];
            }
        }
        if constexpr (CF == CF_DIFFERENCE) {
            // sum_j w (x_j - x_i) = sum_j w x_j - x_i W, x_i the row's coupling variables at time s - 1
#pragma unroll
            for (int q = 0; q < NG; ++q) a[q] = fmaf(-node.x[M::cvar(q)], wsum, a[q]);
        }
        post<CF, NCV>(a, cf, c);
        if (STOCH_BLOCK_START(ks)) node.noise_block(L, r0 + tid, s0 + 1 + ks);
        node.advance(L, Ip, r0 + tid, n, s0, ks, c);
        node.write_ring(raw + (size_t)wslot * n * NCV + (r0 + tid) * NCV);
        if constexpr (SIGMA)
            ring[wslot * slot_floats + r0 + tid] = sjr_pre(node.x[M::cvar(0)], node.x[M::cvar(1)], cf);
    };

    const int K = L.sync_every;
    const int wslot0 = (int)(s0 % RL);  // slot of the last written time
    if constexpr (PIPE) {
        if (g >= 0) gather(wslot0, 0);
        __syncthreads();
        // The two roles run separate loops, so that the model state is not held in the gather threads'
        // registers.  Both end every step with CTA barrier 1 over all threads and every K steps with a
        // cluster barrier, in the same order.
        int wslot = wslot0, since_sync = 0;
        if (tid < T0) {
            for (int ks = 0; ks < nsteps; ++ks) {
                wslot = (wslot + 1 == RL) ? 0 : wslot + 1;
                if (upd) update(ks, wslot, ks & 1);
                cta_barrier_all(TB);
                if (++since_sync == K) {
                    since_sync = 0;
                    cluster_barrier();
                }
            }
        } else {
            for (int ks = 0; ks < nsteps; ++ks) {
                wslot = (wslot + 1 == RL) ? 0 : wslot + 1;
                if (ks + 1 < nsteps) gather(wslot, (ks + 1) & 1);  // step s + 1: times <= s - d_min
                cta_barrier_all(TB);
                if (++since_sync == K) {
                    since_sync = 0;
                    cluster_barrier();
                }
            }
        }
    } else {
        int wslot = wslot0, since_sync = 0;
        for (int ks = 0; ks < nsteps; ++ks) {
            const int prev = wslot;
            wslot = (wslot + 1 == RL) ? 0 : wslot + 1;
            gather(prev, 0);
            __syncthreads();
            if (upd) update(ks, wslot, 0);
            __syncthreads();
            if (++since_sync == K) {
                since_sync = 0;
                cluster.sync();
            }
        }
    }
    if (upd) node.finish(L, Ip, r0 + tid, n, status);
    cluster.sync();
    if (rank == 0 && tid == 0) Ip->step = s_end;
}

// Blocked edge runs on region-major rings (launch.ring_layout = 1).  The
// runs are those of sim_kernel_cluster_runs, but the gather threads take a
// block of B = 4 or 8 steps (launch.block_steps) at a time: for the next
// block an edge needs its source's values at B consecutive times, which sit
// side by side in the region-major ring -- one to three 32-byte L2 loads
// (ld.global.cg.v8), the later ones only when the times reach into the next
// 32-byte chunk, instead of B scattered 8-byte loads, each of which costs a
// 32-byte sector.  The window starts on the 32-byte boundary at or below
// the first time's slot and may run past ring_len into the region's guard
// slots, which mirror slots 0, 1, ....  The update warps advance the steps
// of the current block from the partials gathered during the previous
// block, so there is one CTA barrier per block.  The gather of block b + 1
// reads times up to 2B - 1 - d_min past the last time written before block
// b, so it needs d_min >= 2B - 1 and a barrier interval K <= d_min - B + 1
// between the instance's CTAs, a multiple of B (the windows start on block
// boundaries).
//
// blocked_instance runs one instance's launch window on the C CTAs of the
// instance (this CTA is `rank`); sync() is the barrier between those CTAs
// (every K steps and at the end), which returns false when the launch is
// being abandoned -- then so does blocked_instance.
template <class M, int CF, int SCHEME, int E, bool EXT, int B, class Sync>
__device__ __forceinline__ bool blocked_instance(const tvbk_launch& L, const int inst, const int C, const int rank,
                                                 Sync& sync) {
    static_assert(CF == CF_LINEAR || CF == CF_DIFFERENCE || CF == CF_SIGMOIDAL_JR,
                  "blocked runs: Linear, Difference or SigmoidalJansenRit coupling");
    constexpr int NCV = M::NCV;
    // SigmoidalJansenRit gathers a ring of pre-applied sigmoid values (one float per slot and region)
    constexpr bool SIGMA = GatherTraits<CF, NCV>::SIGMA;
    constexpr int NG = GatherTraits<CF, NCV>::NG;
    constexpr int SPW = 8 / NG;              // slots per 32-byte chunk
    extern __shared__ __align__(16) unsigned char sm[];
    tvbk_inst* __restrict__ Ip = L.insts + inst;
    int32_t* status = L.status + inst;
    const int n = Ip->n;
    const int R = cluster_rows(n, C);
    const int r0 = min(n, rank * R), r1 = min(n, r0 + R), nr = r1 - r0;
    const int RL = Ip->ring_len;
    const int RS = TVBK_RING_REGION_STRIDE(RL, NG);  // slots per region of the gathered ring
    constexpr int GUARD = TVBK_RING_REGION_GUARD(NG);
    const int RSR = TVBK_RING_REGION_STRIDE(RL, NCV);  // of the state ring (the same one unless SIGMA)
    constexpr int GUARDR = TVBK_RING_REGION_GUARD(NCV);
    const int64_t s0 = Ip->step;
    const int64_t s_end = min(Ip->step_end, s0 + L.max_steps);
    if (s0 >= s_end) return true;  // uniform over the instance's CTAs
    // the 32-byte window loads need a 32-byte aligned ring (uniform over the instance's CTAs)
    if (((reinterpret_cast<uintptr_t>(Ip->ring) | (SIGMA ? reinterpret_cast<uintptr_t>(Ip->pre_ring) : 0)) & 31) !=
        0) {
        if (rank == 0 && threadIdx.x == 0) atomicOr(L.status + inst, TVBK_STATUS_UNSUPPORTED);
        return true;
    }
    const int nsteps = (int)(s_end - s0);
    const int tid = threadIdx.x;
    const int TB = blockDim.x;
    const int U = (nr + 31) >> 5;       // update warps
    const int T0 = 32 * U;              // first gather thread
    const int Tg = TB - T0;             // gather threads

    int* rp = reinterpret_cast<int*>(sm);
    float* part = reinterpret_cast<float*>(sm + cluster_runs_head_rp(R));            // [2][4][2][NG][TB]
    int2* esm = reinterpret_cast<int2*>(sm + cluster_blocks_head(R, NG, TB, B));    // the CTA's edges, interleaved
    const int e_lo = Ip->row_ptr[r0], e_hi = Ip->row_ptr[r1];
    const int ne = e_hi - e_lo;
    // as in sim_kernel_cluster_runs: a CTA whose edges do not fit flags the instance and only takes part in
    // the barriers
    const bool fits = ne <= L.cluster_edges && ne <= Tg * E;
    if (!fits && tid == 0) atomicOr(status, TVBK_STATUS_DEGREE);
    const int2* eg = reinterpret_cast<const int2*>(Ip->edges) + e_lo;
    for (int k = tid; k <= nr; k += TB) rp[k] = Ip->row_ptr[r0 + k] - e_lo;
    const int nrun = (ne + E - 1) / E;
    auto eslot = [&](int e) { return (e % E) * nrun + e / E; };
    // edge records {d * 1024 + col, weight}: the packed gather edge holds (d n - col) ncvar
    if (fits)
        for (int e = tid; e < ne; e += TB) {
            int2 r = __ldg(eg + e);
            const int x = r.x / NG;
            const int d = (x + n - 1) / n;
            r.x = d * 1024 + (d * n - x);
            esm[eslot(e)] = r;
        }

    float cf[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) cf[k] = Ip->cfun[k];
    const bool upd = fits && tid < nr;
    Node<M, SCHEME, EXT> node;
    if (upd) {
        node.init(L, Ip, r0 + tid, n, s0);
        if (Ip->aff != nullptr || (!EXT && (Ip->stim != nullptr || Ip->proj != nullptr)))
            atomicOr(status, TVBK_STATUS_UNSUPPORTED);
    }
    float* __restrict__ raw = Ip->ring;
    float* __restrict__ ring = SIGMA ? Ip->pre_ring : raw;
    if constexpr (SIGMA) {
        // the sigmoid ring of this CTA's rows, guard slots included, from the state ring; every CTA's rows
        // are ready after the barrier
        for (int k = threadIdx.x; k < nr * (RL + GUARD); k += blockDim.x) {
            const int lr = k / (RL + GUARD), t = k - lr * (RL + GUARD);
            const float* v = raw + ((size_t)(r0 + lr) * RSR + (t < RL ? t : t - RL)) * NCV;
            ring[(size_t)(r0 + lr) * RS + t] = sjr_pre(v[0], v[1], cf);
        }
        __syncthreads();
        if (!sync()) return false;
    } else {
        __syncthreads();
    }

    // this thread's run and the partials of row tid, as in sim_kernel_cluster_runs
    const int g = tid - T0;
    const int eb = g * E;
    const int cnt = (fits && g >= 0) ? max(0, min(E, ne - eb)) : 0;
    int kb = cnt;
    if (cnt > 0) {
        int lo = 0, hi = nr - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (rp[mid] <= eb) lo = mid; else hi = mid - 1;
        }
        kb = min(rp[lo + 1] - eb, cnt);
        if (kb < cnt) {
            int r2 = lo + 1;
            while (rp[r2 + 1] == rp[r2]) ++r2;
            if (rp[r2 + 1] < eb + cnt) atomicOr(status, TVBK_STATUS_DEGREE);
        }
    }
    int tf = -1, sf = 0, tl = -1;
    float wsum = 0.0f;
    if (upd && rp[tid + 1] > rp[tid]) {
        tf = rp[tid] / E;
        sf = (rp[tid] == tf * E) ? 0 : 1;
        tl = (rp[tid + 1] - 1) / E;
        if constexpr (CF == CF_DIFFERENCE)
            for (int e = rp[tid]; e < rp[tid + 1]; ++e) wsum += __int_as_float(esm[eslot(e)].y);
    }

    // partial (buffer pb, step r of the block, half h, variable q) of run u
    auto pidx = [&](int pb, int r, int h, int q, int u) { return ((((pb * B + r) * 2 + h) * NG + q) * TB) + u; };
    // couplings of the B steps after the time in slot st0: step r reads times (that time) + r - d.  The
    // edges go in batches of BE: the windows of a batch are all requested before the first is used, so a
    // thread waits for one L2 round trip per batch rather than one per edge.  Slots past the run's count
    // load a harmless in-bounds window (region 0 at st0) and add nothing.  One set of sums serves both
    // rows of a run: at the second row's first edge (kb) the first row's sums go to partial 0.
    auto gatherB = [&](int st0, int pb) {
        constexpr int BE = B == 4 ? kClusterBlockBatch : 1;
        constexpr int NCH = (SPW - 1 + B + SPW - 1) / SPW;  // 32-byte chunks a window can touch
        float pa[B][NG];
#pragma unroll
        for (int r = 0; r < B; ++r)
#pragma unroll
            for (int q = 0; q < NG; ++q) pa[r][q] = 0.0f;
#pragma unroll
        for (int k0 = 0; k0 < E; k0 += BE) {
            if (k0 < cnt) {
                float wn[BE][NCH][8];
                int ov[BE];
                float wv[BE];
#pragma unroll
                for (int j = 0; j < BE; ++j) {
                    const int k = k0 + j;
                    const int2 ed = k < cnt ? esm[k * nrun + g] : make_int2(0, 0);
                    const int d = ed.x >> 10, col = ed.x & 1023;
                    int sl = st0 - d;
                    sl += sl < 0 ? RL : 0;
                    const int a = sl & ~(SPW - 1);
                    ov[j] = sl - a;
                    wv[j] = __int_as_float(ed.y);
                    const float* src = ring + ((size_t)col * RS + a) * NG;
                    ldcg32(src, wn[j][0]);
#pragma unroll
                    for (int c = 1; c < NCH; ++c) {
#pragma unroll
                        for (int e = 0; e < 8; ++e) wn[j][c][e] = 0.0f;
                        // chunk c holds times of the window only when the window reaches past c chunks
                        ldcg32_if(ov[j] + B > c * SPW, src + 8 * c, wn[j][c]);
                    }
                }
#pragma unroll
                for (int j = 0; j < BE; ++j) {
                    const int k = k0 + j;
                    if (k < cnt) {
                        if (k == kb) {
#pragma unroll
                            for (int r = 0; r < B; ++r)
#pragma unroll
                                for (int q = 0; q < NG; ++q) {
                                    part[pidx(pb, r, 0, q, g)] = pa[r][q];
                                    pa[r][q] = 0.0f;
                                }
                        }
                        float x[NCH * 8];
#pragma unroll
                        for (int c = 0; c < NCH; ++c)
#pragma unroll
                            for (int e = 0; e < 8; ++e) x[8 * c + e] = wn[j][c][e];
                        // the B times start o slots into the window: shift by o one bit at a time, keeping
                        // the floats still needed after each shift
                        const int o = ov[j];
#pragma unroll
                        for (int bit = SPW / 2; bit >= 1; bit /= 2) {
                            const bool on = (o & bit) != 0;
#pragma unroll
                            for (int c = 0; c < (bit - 1 + B) * NG; ++c) x[c] = on ? x[c + bit * NG] : x[c];
                        }
                        const float w = wv[j];
#pragma unroll
                        for (int r = 0; r < B; ++r)
#pragma unroll
                            for (int q = 0; q < NG; ++q) pa[r][q] = fmaf(w, x[r * NG + q], pa[r][q]);
                    }
                }
            }
        }
        // the last row's sums: partial 1 when the run holds a second row (partial 1 of a run without one is
        // never read), else partial 0
        const int h = kb < cnt ? 1 : 0;
#pragma unroll
        for (int r = 0; r < B; ++r)
#pragma unroll
            for (int q = 0; q < NG; ++q) part[pidx(pb, r, h, q, g)] = pa[r][q];
    };
    auto update = [&](int ks, int wslot, int pb, int r) {
        float a[NG], c[NCV];
#pragma unroll
        for (int q = 0; q < NG; ++q) a[q] = 0.0f;
        if (tf >= 0) {
#pragma unroll
            for (int q = 0; q < NG; ++q) a[q] = part[pidx(pb, r, sf, q, tf)];
            for (int u = tf + 1; u <= tl; ++u) {
#pragma unroll
                for (int q = 0; q < NG; ++q) a[q] += part[pidx(pb, r, 0, q, u)];
            }
        }
        if constexpr (CF == CF_DIFFERENCE) {
#pragma unroll
            for (int q = 0; q < NG; ++q) a[q] = fmaf(-node.x[M::cvar(q)], wsum, a[q]);
        }
        post<CF, NCV>(a, cf, c);
        if (STOCH_BLOCK_START(ks)) node.noise_block(L, r0 + tid, s0 + 1 + ks);
        node.advance(L, Ip, r0 + tid, n, s0, ks, c);
        float* dst = raw + ((size_t)(r0 + tid) * RSR + wslot) * NCV;
        node.write_ring(dst);
        if (wslot < GUARDR) node.write_ring(dst + (size_t)RL * NCV);  // the mirror past ring_len
        if constexpr (SIGMA) {
            const float pv = sjr_pre(node.x[M::cvar(0)], node.x[M::cvar(1)], cf);
            float* pd = ring + (size_t)(r0 + tid) * RS + wslot;
            pd[0] = pv;
            if (wslot < GUARD) pd[RL] = pv;
        }
    };

    const int K = L.sync_every;  // a multiple of 4
    const int bslot0 = (int)(s0 % RL);  // slot of the last time written before the first block
    if (g >= 0) gatherB(bslot0, 0);
    __syncthreads();
    const int nblk = (nsteps + B - 1) / B;
    // The two roles run separate loops, so that the model state is not held in the gather threads'
    // registers.  Both end every block with CTA barrier 1 over all threads and every K steps with sync(),
    // in the same order, and both see the same sync() results.
    bool ok = true;
    if (tid < T0) {
        int bslot = bslot0, since_sync = 0;
        for (int b = 0; b < nblk; ++b) {
            if (upd) {
                int ws = bslot;
#pragma unroll 1
                for (int r = 0; r < B; ++r) {
                    const int ks = B * b + r;
                    if (ks >= nsteps) break;
                    ws = (ws + 1 == RL) ? 0 : ws + 1;
                    update(ks, ws, b & 1, r);
                }
            }
            bslot += B;
            bslot -= bslot >= RL ? RL : 0;
            cta_barrier_all(TB);
            since_sync += B;
            if (since_sync >= K) {
                since_sync = 0;
                if (!sync()) {
                    ok = false;
                    break;
                }
            }
        }
        if (upd) node.finish(L, Ip, r0 + tid, n, status);
    } else {
        int bslot = bslot0, since_sync = 0;
        for (int b = 0; b < nblk; ++b) {
            if (b + 1 < nblk) {
                int nxt = bslot + B;  // the next block's base time
                nxt -= nxt >= RL ? RL : 0;
                gatherB(nxt, (b & 1) ^ 1);
            }
            bslot += B;
            bslot -= bslot >= RL ? RL : 0;
            cta_barrier_all(TB);
            since_sync += B;
            if (since_sync >= K) {
                since_sync = 0;
                if (!sync()) {
                    ok = false;
                    break;
                }
            }
        }
    }
    if (!ok || !sync()) return false;
    if (rank == 0 && tid == 0) Ip->step = s_end;
    return true;
}

// One thread-block cluster of C CTAs per instance (cluster b takes instance
// inst_order[b], or b); the cluster barrier keeps its CTAs in step.
template <class M, int CF, int SCHEME, int E, bool EXT, int B>
__global__ void __launch_bounds__(kClusterThreads, 1) sim_kernel_cluster_blocks(const tvbk_launch L) {
    cgx::cluster_group cluster = cgx::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int inst = L.inst_order != nullptr ? L.inst_order[blockIdx.x / C] : (int)(blockIdx.x / C);
    auto sync = []() {
        cluster_barrier();
        return true;
    };
    blocked_instance<M, CF, SCHEME, E, EXT, B>(L, inst, C, (int)cluster.block_rank(), sync);
}

// Cooperative form (launch.groups = G > 0): G x C CTAs, all resident at once.
// CTAs gC .. gC + C - 1 form group g, which claims queue positions j = 0, 1,
// ... from a device counter (rank 0 claims, the others read the claim after a
// group barrier) and runs instance inst_order[j] (or j) with blocked_instance,
// until the queue is empty.  Thread-block clusters hold at most 16 CTAs and
// only as many of them run at once as the GPCs fit (7 clusters of 16 on 148
// SMs); groups fill every SM and take any C.  The group barrier is a counter
// in global memory with a bounded wait; a barrier that gives up abandons the
// launch, and every instance in flight gets TVBK_STATUS_TIMEOUT.
template <class M, int CF, int SCHEME, int E, bool EXT, int B>
__global__ void __launch_bounds__(kClusterThreads, 1) sim_kernel_group_blocks(const tvbk_launch L) {
    __shared__ int s_ok, s_next;
    const int C = L.cluster;
    const int grp = (int)blockIdx.x / C, rank = (int)blockIdx.x % C;
    uint32_t* const queue = L.group_sync;
    uint32_t* const abort_flag = L.group_sync + 1;
    uint32_t* const count = L.group_sync + 2 + grp;
    uint32_t* const claim = L.group_sync + 2 + L.groups + grp;
    uint32_t target = 0;
    int inst = -1;
    auto sync = [&]() -> bool {
        target += (uint32_t)C;
        cta_barrier_all((int)blockDim.x);
        if (threadIdx.x == 0) {
            const int r = group_arrive_wait(count, target, abort_flag);
            if (!r && inst >= 0) atomicOr(L.status + inst, TVBK_STATUS_TIMEOUT);
            s_ok = r;
        }
        cta_barrier_all((int)blockDim.x);
        return s_ok != 0;
    };
    for (;;) {
        if (rank == 0 && threadIdx.x == 0) st_release_gpu(claim, atomicAdd(queue, 1u));
        if (!sync()) return;
        if (threadIdx.x == 0) s_next = (int)ld_acquire_gpu(claim);
        cta_barrier_all((int)blockDim.x);
        const int j = s_next;
        if (j >= L.n_inst) return;
        inst = L.inst_order != nullptr ? L.inst_order[j] : j;
        if (!blocked_instance<M, CF, SCHEME, E, EXT, B>(L, inst, C, rank, sync)) return;
        // every CTA of the group has read the claim and is done with its shared memory before the next claim
        if (!sync()) return;
    }
}

template <class M, int CF, int SCHEME, int E, bool EXT, int B>
int launch_cluster_blocks_t(const tvbk_launch& L, cudaStream_t st) {
    if constexpr (CF != CF_LINEAR && CF != CF_DIFFERENCE && CF != CF_SIGMOIDAL_JR) {
        return -2;
    } else {
        auto kern = sim_kernel_cluster_blocks<M, CF, SCHEME, E, EXT, B>;
        const int C = L.cluster;
        const int R = cluster_rows(L.max_n, C);
        constexpr int NG = GatherTraits<CF, M::NCV>::NG;
        const size_t smem = cluster_blocks_head(R, NG, kClusterThreads, B) + ((size_t)L.cluster_edges + E) * 8;
        if (smem > 227 * 1024) return -1;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        if (C > 8) {
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            if (e != cudaSuccess) return (int)e;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(L.n_inst * C), 1, 1);
        cfg.blockDim = dim3(kClusterThreads, 1, 1);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)C;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelEx(&cfg, kern, L);
        return (int)e;
    }
}

template <class M, int CF, int SCHEME, int E, bool EXT, int B>
int launch_group_blocks_t(const tvbk_launch& L, cudaStream_t st) {
    if constexpr (CF != CF_LINEAR && CF != CF_DIFFERENCE && CF != CF_SIGMOIDAL_JR) {
        return -2;
    } else {
        auto kern = sim_kernel_group_blocks<M, CF, SCHEME, E, EXT, B>;
        const int C = L.cluster;
        const int R = cluster_rows(L.max_n, C);
        constexpr int NG = GatherTraits<CF, M::NCV>::NG;
        const size_t smem = cluster_blocks_head(R, NG, kClusterThreads, B) + ((size_t)L.cluster_edges + E) * 8;
        if (smem + 64 > 227 * 1024) return -1;  // 64: the kernel's own shared words
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        // every CTA must be resident at once: at most (CTAs per SM) x SMs
        int dev = 0, sms = 0, per_sm = 0;
        e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kClusterThreads, smem);
        if (e != cudaSuccess) return (int)e;
        if ((int64_t)L.groups * C > (int64_t)per_sm * sms) return -4;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(L.groups * C), 1, 1);
        cfg.blockDim = dim3(kClusterThreads, 1, 1);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelEx(&cfg, kern, L);
        return (int)e;
    }
}

template <class M, int CF, int SCHEME, bool EXT, int B>
int launch_cluster_blocks_b(const tvbk_launch& L, cudaStream_t st) {
    if (L.groups > 0) {
        switch (L.edges_per_thread) {
            case 8: return launch_group_blocks_t<M, CF, SCHEME, 8, EXT, B>(L, st);
            case 16: return launch_group_blocks_t<M, CF, SCHEME, 16, EXT, B>(L, st);
            case 32: return launch_group_blocks_t<M, CF, SCHEME, 32, EXT, B>(L, st);
            default: return -2;
        }
    }
    switch (L.edges_per_thread) {
        case 8: return launch_cluster_blocks_t<M, CF, SCHEME, 8, EXT, B>(L, st);
        case 16: return launch_cluster_blocks_t<M, CF, SCHEME, 16, EXT, B>(L, st);
        case 32: return launch_cluster_blocks_t<M, CF, SCHEME, 32, EXT, B>(L, st);
        default: return -2;
    }
}

// Blocks of eight steps are built for the lean kernels (launch.extras = 0) only.
template <class M, int CF, int SCHEME, bool EXT>
int launch_cluster_blocks(const tvbk_launch& L, cudaStream_t st) {
    if (L.block_steps == 8) {
        if constexpr (EXT) {
            return -2;
        } else {
            return launch_cluster_blocks_b<M, CF, SCHEME, EXT, 8>(L, st);
        }
    }
    return launch_cluster_blocks_b<M, CF, SCHEME, EXT, 4>(L, st);
}

template <class M, int CF, int SCHEME, int E, bool PIPE, bool EXT>
int launch_cluster_runs_t(const tvbk_launch& L, cudaStream_t st) {
    auto kern = sim_kernel_cluster_runs<M, CF, SCHEME, E, PIPE, EXT>;
    constexpr int NG = GatherTraits<CF, M::NCV>::NG;
    const int C = L.cluster;
    const int R = cluster_rows(L.max_n, C);
    // interleaved runs take up to cluster_edges + E - 1 edge slots
    const size_t smem = cluster_runs_head(R, NG, kClusterThreads) + ((size_t)L.cluster_edges + E) * 8;
    if (smem > 227 * 1024) return -1;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    if (C > 8) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return (int)e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(L.n_inst * C), 1, 1);
    cfg.blockDim = dim3(kClusterThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, kern, L);
    return (int)e;
}

template <class M, int CF, int SCHEME, bool PIPE, bool EXT>
int launch_cluster_runs(const tvbk_launch& L, cudaStream_t st) {
    switch (L.edges_per_thread) {
        case 8: return launch_cluster_runs_t<M, CF, SCHEME, 8, PIPE, EXT>(L, st);
        case 16: return launch_cluster_runs_t<M, CF, SCHEME, 16, PIPE, EXT>(L, st);
        case 32: return launch_cluster_runs_t<M, CF, SCHEME, 32, PIPE, EXT>(L, st);
        default: return -2;
    }
}

template <class M, int CF, int SCHEME, int MAXE, bool PIPE, bool EXT>
int launch_cluster_t(const tvbk_launch& L, cudaStream_t st) {
    auto kern = sim_kernel_cluster<M, CF, SCHEME, MAXE, PIPE, EXT>;
    constexpr int NACC = (CF == CF_SIGMOIDAL_JR) ? 1 : M::NCV;
    const int C = L.cluster;
    const int R = cluster_rows(L.max_n, C);
    const size_t smem = cluster_smem_head(R, NACC) + (size_t)L.cluster_edges * 8;
    if (smem > 227 * 1024) return -1;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    if (C > 8) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return (int)e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(L.n_inst * C), 1, 1);
    cfg.blockDim = dim3(kClusterThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, kern, L);
    return (int)e;
}

template <class M, int CF, int SCHEME, bool PIPE, bool EXT>
int launch_cluster_p(const tvbk_launch& L, cudaStream_t st) {
    if (L.max_degree <= 64) return launch_cluster_t<M, CF, SCHEME, 2, PIPE, EXT>(L, st);
    if (L.max_degree <= 128) return launch_cluster_t<M, CF, SCHEME, 4, PIPE, EXT>(L, st);
    if (L.max_degree <= 256) return launch_cluster_t<M, CF, SCHEME, 8, PIPE, EXT>(L, st);
    if (L.max_degree <= 1024) return launch_cluster_t<M, CF, SCHEME, 32, PIPE, EXT>(L, st);
    return -1;
}

template <class M, int CF, int SCHEME>
int launch_cluster(const tvbk_launch& L, cudaStream_t st) {
    if (L.ring_layout == 1) {  // blocked edge runs on region-major rings
        if (L.edges_per_thread <= 0 || !L.prefetch) return -2;
        if (L.extras == 0) return launch_cluster_blocks<M, CF, SCHEME, false>(L, st);
        return launch_cluster_blocks<M, CF, SCHEME, true>(L, st);
    }
    if (L.edges_per_thread > 0) {  // edge runs
        if (L.extras == 0) {
            if (L.prefetch) return launch_cluster_runs<M, CF, SCHEME, true, false>(L, st);
            return launch_cluster_runs<M, CF, SCHEME, false, false>(L, st);
        }
        if (L.prefetch) return launch_cluster_runs<M, CF, SCHEME, true, true>(L, st);
        return launch_cluster_runs<M, CF, SCHEME, false, true>(L, st);
    }
    // the warp-per-row gather reads x_i of the step it sums: no prefetch with Difference
    if (CF == CF_DIFFERENCE && L.prefetch) return -2;
    if (L.extras == 0) {
        if (L.prefetch) return launch_cluster_p<M, CF, SCHEME, true, false>(L, st);
        return launch_cluster_p<M, CF, SCHEME, false, false>(L, st);
    }
    if (L.prefetch) return launch_cluster_p<M, CF, SCHEME, true, true>(L, st);
    return launch_cluster_p<M, CF, SCHEME, false, true>(L, st);
}

}  // namespace tvbk
