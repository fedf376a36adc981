// The fused region-simulation kernel: one CTA per simulation instance, one
// thread per region, all steps of a chunk in one launch.
//
// Per step s (the loop of tvb/simulator/simulator.py:356-364), thread i:
//   1. gathers its row of the connectome from the delayed-history ring,
//      value of region j at time s - 1 - d_ij (history.py:251-256), applies
//      pre(), weights and sums (coupling.py:149-167) and post();
//   2. advances its region's state with the scheme (integrators.py:296-426),
//      drawing additive noise from the fed array or the Philox stream;
//   3. writes its coupling variables for time s into the ring (history.py:203-204);
//   4. feeds the observed variables to Raw / TemporalAverage / Bold
//      (monitors.py:188-190,380-391,942-962).
//
// Ring and barriers: time t lives in slot t % ring_len.  The gather of step s
// reads times s-1-d for d_min <= d <= horizon-1.  With ring_len >= horizon + K
// and K <= d_min + 1, the CTA only needs a barrier every K steps: within a
// window of K steps no thread reads a time written inside the window, and no
// write of the window lands on a slot that is still to be read.  The ring is
// staged in shared memory when it fits (SMEM = true), else read in place.
//
// Edges: with MAXD > 0 a thread keeps its row's packed edges (ring offset and
// weight) in registers for the whole launch, MAXD >= the largest row degree;
// with MAXD = 0 it reads them from global memory (L1) every step.
#pragma once
#include <cstdint>

#include "tvbk.h"
#include "tvbk_models.cuh"
#include "tvbk_philox.cuh"

namespace tvbk {

template <int SCHEME>
struct SchemeTraits {
    static constexpr bool stoch = (SCHEME == TVBK_SCHEME_EULER_STOCH || SCHEME == TVBK_SCHEME_HEUN_STOCH);
};

// acc += w * pre(x_i, x_j) for one edge whose delayed value(s) start at src.
template <int CF, int NCV>
__device__ __forceinline__ void accumulate(float* acc, float w, const float* src, const float* xi, const float* cf) {
    if constexpr (NCV == 1) {
        const float v = src[0];
        if constexpr (CF == CF_DIFFERENCE)
            acc[0] = fmaf(w, v - xi[0], acc[0]);
        else
            acc[0] = fmaf(w, v, acc[0]);
    } else {
        const float2 v = *reinterpret_cast<const float2*>(src);
        if constexpr (CF == CF_DIFFERENCE) {
            acc[0] = fmaf(w, v.x - xi[0], acc[0]);
            acc[1] = fmaf(w, v.y - xi[1], acc[1]);
        } else if constexpr (CF == CF_SIGMOIDAL_JR) {
            const float pre = cf[0] + (cf[1] - cf[0]) / (1.0f + expf(cf[3] * (cf[2] - (v.x - v.y))));
            acc[0] = fmaf(w, pre, acc[0]);
        } else {
            acc[0] = fmaf(w, v.x, acc[0]);
            acc[1] = fmaf(w, v.y, acc[1]);
        }
    }
}

// post(): Linear a * gx + b; Difference a * gx; SigmoidalJansenRit a * gx (one output).
template <int CF, int NCV>
__device__ __forceinline__ void post(const float* acc, const float* cf, float* c) {
    if constexpr (CF == CF_LINEAR) {
#pragma unroll
        for (int k = 0; k < NCV; ++k) c[k] = cf[0] * acc[k] + cf[1];
    } else if constexpr (CF == CF_DIFFERENCE) {
#pragma unroll
        for (int k = 0; k < NCV; ++k) c[k] = cf[0] * acc[k];
    } else {
        c[0] = cf[4] * acc[0];
#pragma unroll
        for (int k = 1; k < NCV; ++k) c[k] = 0.0f;
    }
}

// Row gather with edges in registers: two partial sums (even / odd edges).
// The loop is branch-free so that every shared-memory load can be issued
// ahead of its use: padding slots (k >= deg) carry weight 0 and offset 0,
// which reads the region-0 value of time s - 1, always inside the ring.
// (With a non-finite value there, 0 * value would be NaN; the state is then
// non-finite already and the instance's status reports it.)
template <class M, int CF, int MAXD>
struct RegRow {
    int off[MAXD];
    float w[MAXD];
    int deg;

    __device__ __forceinline__ void load(const tvbk_edge* __restrict__ edges, int e0, int e1) {
        deg = e1 - e0;
        const int2* ed2 = reinterpret_cast<const int2*>(edges) + e0;
#pragma unroll
        for (int k = 0; k < MAXD; ++k) {
            const int2 ed = (k < deg) ? __ldg(ed2 + k) : make_int2(0, 0);
            off[k] = ed.x;
            w[k] = __int_as_float(ed.y);
        }
    }

    __device__ __forceinline__ void couple(const float* __restrict__ ring, int base_off, int ring_floats,
                                           const float* xi, const float* cf, float* c) const {
        constexpr int NCV = M::NCV;
        float a0[NCV], a1[NCV];
#pragma unroll
        for (int k = 0; k < NCV; ++k) a0[k] = a1[k] = 0.0f;
#pragma unroll
        for (int k = 0; k < MAXD; ++k) {
            const int a = gather_addr(base_off, off[k], ring_floats);
            accumulate<CF, NCV>((k & 1) ? a1 : a0, w[k], ring + a, xi, cf);
        }
#pragma unroll
        for (int k = 0; k < NCV; ++k) a0[k] += a1[k];
        post<CF, NCV>(a0, cf, c);
    }
};

// Row gather reading the packed edges from global memory every step.
template <class M, int CF>
struct RegRow<M, CF, 0> {
    const int2* ed2;
    int deg;

    __device__ __forceinline__ void load(const tvbk_edge* __restrict__ edges, int e0, int e1) {
        ed2 = reinterpret_cast<const int2*>(edges) + e0;
        deg = e1 - e0;
    }

    __device__ __forceinline__ void couple(const float* __restrict__ ring, int base_off, int ring_floats,
                                           const float* xi, const float* cf, float* c) const {
        constexpr int NCV = M::NCV;
        float a0[NCV], a1[NCV];
#pragma unroll
        for (int k = 0; k < NCV; ++k) a0[k] = a1[k] = 0.0f;
        int e = 0;
        for (; e + 1 < deg; e += 2) {
            const int2 p = __ldg(ed2 + e), q = __ldg(ed2 + e + 1);
            accumulate<CF, NCV>(a0, __int_as_float(p.y), ring + gather_addr(base_off, p.x, ring_floats), xi, cf);
            accumulate<CF, NCV>(a1, __int_as_float(q.y), ring + gather_addr(base_off, q.x, ring_floats), xi, cf);
        }
        if (e < deg) {
            const int2 p = __ldg(ed2 + e);
            accumulate<CF, NCV>(a0, __int_as_float(p.y), ring + gather_addr(base_off, p.x, ring_floats), xi, cf);
        }
#pragma unroll
        for (int k = 0; k < NCV; ++k) a0[k] += a1[k];
        post<CF, NCV>(a0, cf, c);
    }
};

template <class M, int CF, int SCHEME, bool SMEM, int MAXT, int MAXD>
__global__ void __launch_bounds__(MAXT) sim_kernel(const tvbk_launch L) {
    constexpr int NSV = M::NSV, NCV = M::NCV, NP = M::NP, NINT = M::NINT;
    constexpr bool STOCH = SchemeTraits<SCHEME>::stoch;
    constexpr int MV = M::NOBS < TVBK_MAX_VOI ? M::NOBS : TVBK_MAX_VOI;  // nvoi <= nobs is checked on the host
    extern __shared__ __align__(16) float smem[];

    tvbk_inst* __restrict__ Ip = L.insts + blockIdx.x;
    const int n = Ip->n;
    const int i = threadIdx.x;
    const bool act = i < n;
    const int RL = Ip->ring_len;
    const int slot_floats = n * NCV;
    const int ring_floats = RL * slot_floats;
    const int64_t s0 = Ip->step;
    const int64_t s_end = min(Ip->step_end, s0 + L.max_steps);
    if (s0 >= s_end) return;  // uniform over the block
    const int nsteps = (int)(s_end - s0);

    float* ring = SMEM ? smem : Ip->ring;
    if (SMEM) {
        const float4* src = reinterpret_cast<const float4*>(Ip->ring);
        float4* dst = reinterpret_cast<float4*>(smem);
        const int n4 = ring_floats >> 2;
        for (int k = i; k < n4; k += blockDim.x) dst[k] = src[k];
        for (int k = (n4 << 2) + i; k < ring_floats; k += blockDim.x) smem[k] = Ip->ring[k];
        __syncthreads();
    }

    const float dt = L.dt;
    const int nvoi = L.nvoi;
    float x[NSV], p[NP], cf[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) cf[k] = Ip->cfun[k];
    RegRow<M, CF, MAXD> row;
    row.deg = 0;
    float sig[NINT];
    float tacc[MV];
    double bacc[MV];
    float* raw = Ip->raw;
    float* tavg = Ip->tavg;
    double* bold = Ip->bold;
    const bool do_tavg = tavg != nullptr, do_bold = bold != nullptr;
#pragma unroll
    for (int v = 0; v < MV; ++v) {
        tacc[v] = 0.0f;
        bacc[v] = 0.0;
    }
    if (act) {
#pragma unroll
        for (int k = 0; k < NSV; ++k) x[k] = Ip->state[k * n + i];
#pragma unroll
        for (int k = 0; k < NP; ++k) p[k] = Ip->params[k * n + i];
        const int e0 = Ip->row_ptr[i], e1 = Ip->row_ptr[i + 1];
        if (MAXD > 0 && e1 - e0 > MAXD) atomicOr(L.status + blockIdx.x, TVBK_STATUS_DEGREE);
        row.load(Ip->edges, e0, e1);
#pragma unroll
        for (int k = 0; k < NINT; ++k) sig[k] = STOCH ? Ip->noise_sigma[k * n + i] : 0.0f;
#pragma unroll
        for (int v = 0; v < MV; ++v) {
            if (v < nvoi) {
                if (do_tavg) tacc[v] = Ip->tavg_acc[v * n + i];
                if (do_bold) bacc[v] = Ip->bold_acc[v * n + i];
            }
        }
    }
    // monitor phases (64-bit divisions once per launch)
    const int t_istep = Ip->tavg_istep, b_istep = Ip->bold_istep, b_ii = Ip->bold_ii, SL = Ip->stock_len;
    int ph_t = do_tavg ? (int)(s0 % t_istep) : 0;
    int ph_b = do_bold ? (int)(s0 % b_istep) : 0;
    int ph_i = do_bold ? (int)(s0 % b_ii) : 0;
    int q_prev = do_bold ? (int)((s0 / b_ii) % SL) : 0;
    float* raw_p = raw ? raw + (size_t)(s0 - Ip->raw_base) * nvoi * n + i : nullptr;
    const float* fed_p = Ip->noise_fed ? Ip->noise_fed + (size_t)(s0 - Ip->fed_base) * NINT * n + i : nullptr;
    float* tavg_p = do_tavg ? tavg + (size_t)(s0 / t_istep - Ip->tavg_base) * nvoi * n + i : nullptr;
    double* bold_p = do_bold ? bold + (size_t)(s0 / b_istep - Ip->bold_base) * nvoi * n + i : nullptr;
    const int noise_kind = L.noise;
    const uint32_t seed = Ip->seed, stream = Ip->stream;
    float zc[NINT][4];
#pragma unroll
    for (int k = 0; k < NINT; ++k)
#pragma unroll
        for (int r = 0; r < 4; ++r) zc[k][r] = 0.0f;
    int rphase = (int)((s0 + 1) & 3);  // s & 3 of the first step

    const int K = L.sync_every;
    int since_sync = 0;
    int wslot = (int)(s0 % RL);  // slot of the last written time
    for (int ks = 0; ks < nsteps; ++ks) {
        const int base_off = wslot * slot_floats;  // time s - 1
        wslot = (wslot + 1 == RL) ? 0 : wslot + 1;  // time s
        if (act) {
            float xi[NCV];
#pragma unroll
            for (int k = 0; k < NCV; ++k) xi[k] = x[M::cvar(k)];
            float c[NCV];
            row.couple(ring, base_off, ring_floats, xi, cf, c);

            float z[NINT];
            if constexpr (STOCH) {
                if (noise_kind == TVBK_NOISE_FED) {
#pragma unroll
                    for (int k = 0; k < NINT; ++k) z[k] = fed_p[k * n];
                    fed_p += (size_t)NINT * n;
                } else {
                    if (rphase == 0 || ks == 0) {
                        const int64_t s = s0 + 1 + ks;
#pragma unroll
                        for (int k = 0; k < NINT; ++k)
                            if (sig[k] != 0.0f) philox_normals4(seed, stream, s, i, k, zc[k]);
                    }
#pragma unroll
                    for (int k = 0; k < NINT; ++k)
                        z[k] = (rphase == 0) ? zc[k][0] : (rphase == 1) ? zc[k][1] : (rphase == 2) ? zc[k][2] : zc[k][3];
                }
            }

            float m0[NSV];
            M::dfun(x, c, p, m0);
            if constexpr (SCHEME == TVBK_SCHEME_EULER_DET) {
#pragma unroll
                for (int k = 0; k < NSV; ++k) x[k] = x[k] + dt * m0[k];
            } else if constexpr (SCHEME == TVBK_SCHEME_EULER_STOCH) {
#pragma unroll
                for (int k = 0; k < NSV; ++k) x[k] = x[k] + dt * m0[k] + sig[k] * z[k];
            } else if constexpr (SCHEME == TVBK_SCHEME_HEUN_DET || SCHEME == TVBK_SCHEME_HEUN_STOCH) {
                float inter[NSV], nz[NSV];
#pragma unroll
                for (int k = 0; k < NSV; ++k) {
                    nz[k] = STOCH ? sig[k] * z[k] : 0.0f;
                    inter[k] = x[k] + dt * m0[k] + nz[k];
                }
                M::bound(inter);
                float m1[NSV];
                M::dfun(inter, c, p, m1);
                const float hdt = dt * 0.5f;
#pragma unroll
                for (int k = 0; k < NSV; ++k) x[k] = x[k] + (m0[k] + m1[k]) * hdt + nz[k];
            } else {  // identity
#pragma unroll
                for (int k = 0; k < NSV; ++k) x[k] = m0[k];
            }
            M::bound(x);

            // history update: coupling variables of time s
            float* dst = ring + wslot * slot_floats + i * NCV;
            if constexpr (NCV == 1) {
                dst[0] = x[M::cvar(0)];
            } else {
                *reinterpret_cast<float2*>(dst) = make_float2(x[M::cvar(0)], x[M::cvar(1)]);
            }

            // monitors
            if (raw_p != nullptr) {
#pragma unroll
                for (int v = 0; v < MV; ++v)
                    if (v < nvoi) raw_p[v * n] = M::observe(L.voi[v], x);
                raw_p += (size_t)nvoi * n;
            }
            if (do_tavg) {
#pragma unroll
                for (int v = 0; v < MV; ++v)
                    if (v < nvoi) tacc[v] += M::observe(L.voi[v], x);
                if (++ph_t == t_istep) {
                    ph_t = 0;
#pragma unroll
                    for (int v = 0; v < MV; ++v)
                        if (v < nvoi) {
                            tavg_p[v * n] = tacc[v] / (float)t_istep;
                            tacc[v] = 0.0f;
                        }
                    tavg_p += (size_t)nvoi * n;
                }
            }
            if (do_bold) {
#pragma unroll
                for (int v = 0; v < MV; ++v)
                    if (v < nvoi) bacc[v] += (double)M::observe(L.voi[v], x);
                double* stock = Ip->bold_stock;
                if (++ph_i == b_ii) {
                    ph_i = 0;
                    double* st = stock + (size_t)q_prev * nvoi * n + i;
#pragma unroll
                    for (int v = 0; v < MV; ++v)
                        if (v < nvoi) {
                            st[v * n] = bacc[v] / (double)b_ii;
                            bacc[v] = 0.0;
                        }
                    q_prev = (q_prev + 1 == SL) ? 0 : q_prev + 1;
                }
                if (++ph_b == b_istep) {
                    ph_b = 0;
                    const int64_t s = s0 + 1 + ks;
                    const int m = (int)((s / b_ii) % SL);
                    // numpy.roll(hrf, m - 1)[k] == hrf[(k - m + 1) mod SL]
                    int idx0 = 1 - m;
                    idx0 = idx0 < 0 ? idx0 + SL : (idx0 >= SL ? idx0 - SL : idx0);
                    const double* __restrict__ hrf = Ip->hrf;
                    const double k1v0 = Ip->bold_k1v0;
                    for (int v = 0; v < nvoi; ++v) {
                        double dot = 0.0;
                        int idx = idx0;
                        const double* sv = stock + (size_t)v * n + i;
                        for (int k = 0; k < SL; ++k) {
                            dot = fma(__ldg(hrf + idx), sv[(size_t)k * nvoi * n], dot);
                            idx = (idx + 1 == SL) ? 0 : idx + 1;
                        }
                        bold_p[v * n] = (dot - 1.0) * k1v0;
                    }
                    bold_p += (size_t)nvoi * n;
                }
            }
        }
        rphase = (rphase + 1) & 3;
        if (++since_sync == K) {
            since_sync = 0;
            __syncthreads();
        }
    }

    // write back
    __syncthreads();
    if (act) {
        bool finite = true;
#pragma unroll
        for (int k = 0; k < NSV; ++k) {
            Ip->state[k * n + i] = x[k];
            finite = finite && isfinite(x[k]);
        }
#pragma unroll
        for (int v = 0; v < MV; ++v)
            if (v < nvoi) {
                if (do_tavg) Ip->tavg_acc[v * n + i] = tacc[v];
                if (do_bold) Ip->bold_acc[v * n + i] = bacc[v];
            }
        if (!finite) atomicOr(L.status + blockIdx.x, TVBK_STATUS_NONFINITE);
    }
    if (SMEM) {
        float4* dst = reinterpret_cast<float4*>(Ip->ring);
        const float4* src = reinterpret_cast<const float4*>(smem);
        const int n4 = ring_floats >> 2;
        for (int k = i; k < n4; k += blockDim.x) dst[k] = src[k];
        for (int k = (n4 << 2) + i; k < ring_floats; k += blockDim.x) Ip->ring[k] = smem[k];
    }
    if (i == 0) Ip->step = s_end;
}

// ------------------------------------------------------------------ launch

template <class M, int CF, int SCHEME, bool SMEM, int MAXT, int MAXD>
int launch_one(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes) {
    auto kern = sim_kernel<M, CF, SCHEME, SMEM, MAXT, MAXD>;
    if (smem_bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
        if (e != cudaSuccess) return (int)e;
    }
    const int threads = ((L.max_n + 31) / 32) * 32;
    kern<<<L.n_inst, threads, smem_bytes, st>>>(L);
    return (int)cudaGetLastError();
}

// max_deg: the largest row degree over all instances of the launch.
template <class M, int CF, int SCHEME, bool SMEM, int MAXT>
int launch_deg(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes, int max_deg) {
    if (max_deg <= 32) return launch_one<M, CF, SCHEME, SMEM, MAXT, 32>(L, st, smem_bytes);
    if (max_deg <= 64) return launch_one<M, CF, SCHEME, SMEM, MAXT, 64>(L, st, smem_bytes);
    return launch_one<M, CF, SCHEME, SMEM, MAXT, 0>(L, st, smem_bytes);
}

template <class M, int CF, int SCHEME>
int launch_scheme(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes, int max_deg) {
    if (L.ring_in_smem) {
        if (L.max_n > 256) return -1;
        return launch_deg<M, CF, SCHEME, true, 256>(L, st, smem_bytes, max_deg);
    }
    if (L.max_n <= 256) return launch_deg<M, CF, SCHEME, false, 256>(L, st, 0, max_deg);
    return launch_one<M, CF, SCHEME, false, 1024, 0>(L, st, 0);
}

template <class M, int CF>
int launch_cfun(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes, int max_deg) {
    switch (L.scheme) {
        case TVBK_SCHEME_EULER_DET: return launch_scheme<M, CF, TVBK_SCHEME_EULER_DET>(L, st, smem_bytes, max_deg);
        case TVBK_SCHEME_EULER_STOCH:
            return launch_scheme<M, CF, TVBK_SCHEME_EULER_STOCH>(L, st, smem_bytes, max_deg);
        case TVBK_SCHEME_HEUN_DET: return launch_scheme<M, CF, TVBK_SCHEME_HEUN_DET>(L, st, smem_bytes, max_deg);
        case TVBK_SCHEME_HEUN_STOCH:
            return launch_scheme<M, CF, TVBK_SCHEME_HEUN_STOCH>(L, st, smem_bytes, max_deg);
        default: return -2;
    }
}

}  // namespace tvbk
