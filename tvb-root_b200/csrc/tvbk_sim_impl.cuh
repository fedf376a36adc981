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
#include <type_traits>
#include <cstdint>

#include "tvbk.h"
#include "tvbk_models.cuh"
#include "tvbk_philox.cuh"

namespace tvbk {

template <int SCHEME>
struct SchemeTraits {
    static constexpr bool stoch = (SCHEME == TVBK_SCHEME_EULER_STOCH || SCHEME == TVBK_SCHEME_HEUN_STOCH);
};

// True at the first step of a launch and at every step s with (s - 1) & 3 == 0:
// where a new block of four Philox normals starts.
#define STOCH_BLOCK_START(ks) ((ks) == 0 || ((s0 + (ks)) & 3) == 0)

// Per-edge pre() forms of the couplings whose pre / post are chosen at run
// time (CF_GENERIC kernels): HyperbolicTangent a (1 + tanh((b x_j - midpoint)
// / sigma)) (coupling.py:263-264) and Kuramoto sin(x_j - x_i)
// (coupling.py:504-505); Sigmoidal gathers x_j like Linear.
enum { PRE_TANH = 100, PRE_SIN = 101 };

// acc += w * pre(x_i, x_j) for one edge whose delayed value(s) start at src.
template <int CF, int NCV>
__device__ __forceinline__ void accumulate(float* acc, float w, const float* src, const float* xi, const float* cf) {
    if constexpr (CF == PRE_TANH || CF == PRE_SIN) {
        float v[NCV];
        if constexpr (NCV == 1) {
            v[0] = src[0];
        } else {
            const float2 t = *reinterpret_cast<const float2*>(src);
            v[0] = t.x;
            v[1] = t.y;
        }
#pragma unroll
        for (int k = 0; k < NCV; ++k) {
            const float pre = (CF == PRE_TANH) ? cf[0] * (1.0f + tanhf((cf[1] * v[k] - cf[2]) / cf[3]))
                                               : sinf(v[k] - xi[k]);
            acc[k] = fmaf(w, pre, acc[k]);
        }
    } else if constexpr (NCV == 1) {
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

// post() of the run-time chosen couplings: Sigmoidal cmin + (cmax - cmin) /
// (1 + exp(-a ((gx - midpoint) / sigma))) with cf = {cmin, cmax, midpoint, a,
// sigma} (coupling.py:321-322); HyperbolicTangent gx; Kuramoto a / ncvar * gx
// (coupling.py:507-508, which divides by gx.shape[0], the coupling variables).
template <int NCV>
__device__ __forceinline__ void post_generic(const float* acc, const float* cf, int kind, float* c) {
#pragma unroll
    for (int k = 0; k < NCV; ++k) {
        if (kind == TVBK_CFUN_SIGMOIDAL)
            c[k] = cf[0] + (cf[1] - cf[0]) / (1.0f + expf(-cf[3] * ((acc[k] - cf[2]) / cf[4])));
        else if (kind == TVBK_CFUN_KURAMOTO)
            c[k] = cf[0] / (float)NCV * acc[k];
        else
            c[k] = acc[k];
    }
}

// SigmoidalJansenRit's pre() depends on the source region's delayed state
// only, so the row and cluster kernels apply it once per (time, region), when
// the state is written, and keep a gather ring of those values (one float per
// slot and region): the same float32 expression on the same operands as
// applying it per edge, with one exp per region-step instead of one per edge.
// The ring of raw coupling variables is still written every step (it is the
// history the caller reads back).  GatherTraits gives the gather's view: the
// number of floats per (slot, region) it reads and the coupling it applies.
template <int CF, int NCV>
struct GatherTraits {
    static constexpr bool SIGMA = (CF == CF_SIGMOIDAL_JR);
    static constexpr int NG = SIGMA ? 1 : NCV;
    static constexpr int GCF = SIGMA ? CF_LINEAR : CF;
};

__device__ __forceinline__ float sjr_pre(float v0, float v1, const float* cf) {
    return cf[0] + (cf[1] - cf[0]) / (1.0f + expf(cf[3] * (cf[2] - (v0 - v1))));
}

// Fill a gather ring of pre-applied sigmoid values from the raw ring
// [nslots*n][2]: elements [k0, nelem) strided by `stride`.
__device__ __forceinline__ void sigma_ring(float* dst, const float* __restrict__ raw, int nelem, int k0, int stride,
                                           const float* cf) {
    for (int k = k0; k < nelem; k += stride) {
        const float2 v = reinterpret_cast<const float2*>(raw)[k];
        dst[k] = sjr_pre(v.x, v.y, cf);
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
            off[k] = ed.x * (int)sizeof(float);  // byte offsets: no scaling per edge
            w[k] = __int_as_float(ed.y);
        }
    }

    // all MAXD slots of row r from a slot table (bank-scheduled edges and padding)
    __device__ __forceinline__ void load_slots(const tvbk_edge* __restrict__ slots, int r, int e0, int e1) {
        deg = e1 - e0;
        const int2* s2 = reinterpret_cast<const int2*>(slots) + (size_t)r * MAXD;
#pragma unroll
        for (int k = 0; k < MAXD; ++k) {
            const int2 ed = __ldg(s2 + k);
            off[k] = ed.x * (int)sizeof(float);
            w[k] = __int_as_float(ed.y);
        }
    }

    // a0 = sum over the row of w * pre (two partial sums: even / odd slots)
    template <int GCF, int NG>
    __device__ __forceinline__ void sum(const float* __restrict__ ring, int base_off, int ring_floats,
                                        const float* xi, const float* cf, float* a0) const {
        float a1[NG];
#pragma unroll
        for (int k = 0; k < NG; ++k) a0[k] = a1[k] = 0.0f;
        const char* rb = reinterpret_cast<const char*>(ring);
        const int base_b = base_off * (int)sizeof(float), ring_b = ring_floats * (int)sizeof(float);
#pragma unroll
        for (int k = 0; k < MAXD; ++k) {
            const int a = gather_addr(base_b, off[k], ring_b);
            accumulate<GCF, NG>((k & 1) ? a1 : a0, w[k], reinterpret_cast<const float*>(rb + a), xi, cf);
        }
#pragma unroll
        for (int k = 0; k < NG; ++k) a0[k] += a1[k];
    }

    // kind: the launch's coupling code, read by the run-time chosen couplings (CF_GENERIC)
    __device__ __forceinline__ void couple(const float* __restrict__ ring, int base_off, int ring_floats,
                                           const float* xi, const float* cf, float* c, int kind = 0) const {
        constexpr int NCV = M::NCV;
        if constexpr (CF == CF_GENERIC) {
            float a[NCV];
            if (kind == TVBK_CFUN_HYPERBOLIC_TANGENT)
                sum<PRE_TANH, NCV>(ring, base_off, ring_floats, xi, cf, a);
            else if (kind == TVBK_CFUN_KURAMOTO)
                sum<PRE_SIN, NCV>(ring, base_off, ring_floats, xi, cf, a);
            else
                sum<CF_LINEAR, NCV>(ring, base_off, ring_floats, xi, cf, a);
            post_generic<NCV>(a, cf, kind, c);
        } else {
            constexpr int NG = GatherTraits<CF, NCV>::NG, GCF = GatherTraits<CF, NCV>::GCF;
            float a[NG];
            sum<GCF, NG>(ring, base_off, ring_floats, xi, cf, a);
            post<CF, NCV>(a, cf, c);
        }
    }

    // The couplings of four consecutive gathers, c[r] read at ring times
    // (time of base_off) + r - d, r = 0..3: one wrapped ring address per edge,
    // then r slots past it.  Those may run up to three slots past the ring's
    // end, into the guard slots that mirror slots 0..2 (TVBK_RING_GUARD).
    // Each gather sums its slots in the same order into the same two partial
    // sums as sum(), so c[r] equals couple() at base_off + r slots bit for
    // bit.  Couplings whose pre() ignores x_i only (the prefetching kernel's).
    __device__ __forceinline__ void couple4(const float* __restrict__ ring, int base_off, int ring_floats,
                                            int slot_floats, const float* cf, float (*c)[M::NCV]) const {
        static_assert(CF != CF_GENERIC && CF != CF_DIFFERENCE, "couple4 is for couplings whose pre() ignores x_i");
        constexpr int NCV = M::NCV;
        constexpr int NG = GatherTraits<CF, NCV>::NG, GCF = GatherTraits<CF, NCV>::GCF;
        float a0[4][NG], a1[4][NG];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int k = 0; k < NG; ++k) a0[r][k] = a1[r][k] = 0.0f;
        const char* rb = reinterpret_cast<const char*>(ring);
        const int base_b = base_off * (int)sizeof(float), ring_b = ring_floats * (int)sizeof(float);
        const int sb = slot_floats * (int)sizeof(float);
#pragma unroll
        for (int k = 0; k < MAXD; ++k) {
            const int a = gather_addr(base_b, off[k], ring_b);
#pragma unroll
            for (int r = 0; r < 4; ++r)
                accumulate<GCF, NG>((k & 1) ? a1[r] : a0[r], w[k], reinterpret_cast<const float*>(rb + r * sb + a),
                                    nullptr, cf);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            float s[NG];
#pragma unroll
            for (int k = 0; k < NG; ++k) s[k] = a0[r][k] + a1[r][k];
            post<CF, NCV>(s, cf, c[r]);
        }
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

    template <int GCF, int NG>
    __device__ __forceinline__ void sum(const float* __restrict__ ring, int base_off, int ring_floats,
                                        const float* xi, const float* cf, float* a0) const {
        float a1[NG];
#pragma unroll
        for (int k = 0; k < NG; ++k) a0[k] = a1[k] = 0.0f;
        int e = 0;
        for (; e + 1 < deg; e += 2) {
            const int2 p = __ldg(ed2 + e), q = __ldg(ed2 + e + 1);
            accumulate<GCF, NG>(a0, __int_as_float(p.y), ring + gather_addr(base_off, p.x, ring_floats), xi, cf);
            accumulate<GCF, NG>(a1, __int_as_float(q.y), ring + gather_addr(base_off, q.x, ring_floats), xi, cf);
        }
        if (e < deg) {
            const int2 p = __ldg(ed2 + e);
            accumulate<GCF, NG>(a0, __int_as_float(p.y), ring + gather_addr(base_off, p.x, ring_floats), xi, cf);
        }
#pragma unroll
        for (int k = 0; k < NG; ++k) a0[k] += a1[k];
    }

    __device__ __forceinline__ void couple(const float* __restrict__ ring, int base_off, int ring_floats,
                                           const float* xi, const float* cf, float* c, int kind = 0) const {
        constexpr int NCV = M::NCV;
        if constexpr (CF == CF_GENERIC) {
            float a[NCV];
            if (kind == TVBK_CFUN_HYPERBOLIC_TANGENT)
                sum<PRE_TANH, NCV>(ring, base_off, ring_floats, xi, cf, a);
            else if (kind == TVBK_CFUN_KURAMOTO)
                sum<PRE_SIN, NCV>(ring, base_off, ring_floats, xi, cf, a);
            else
                sum<CF_LINEAR, NCV>(ring, base_off, ring_floats, xi, cf, a);
            post_generic<NCV>(a, cf, kind, c);
        } else {
            constexpr int NG = GatherTraits<CF, NCV>::NG, GCF = GatherTraits<CF, NCV>::GCF;
            float a[NG];
            sum<GCF, NG>(ring, base_off, ring_floats, xi, cf, a);
            post<CF, NCV>(a, cf, c);
        }
    }
};

// Per-region state and update: scheme step with noise, ring write and the
// monitors (shared by all kernel variants).  EXT = false builds it without
// the region stimulus and the AfferentCoupling monitor, for launches that
// use neither (their terms and registers are then absent, not zero).
template <class M, int SCHEME, bool EXT = true>
struct Node {
    static constexpr int NSV = M::NSV, NCV = M::NCV, NP = M::NP, NINT = M::NINT;
    static constexpr bool STOCH = SchemeTraits<SCHEME>::stoch;
    static constexpr int MV = M::NOBS < TVBK_MAX_VOI ? M::NOBS : TVBK_MAX_VOI;  // nvoi <= nobs checked on the host

    // p: the NP parameters of the region, then the NPX - NP values M::prepare() derives from them
    float x[NSV], p[M::NPX], sig[NINT], zc[NINT][4], tacc[MV];
    double bacc[MV];
    float* raw_p;
    const float* fed_p;
    const float* stim_p;  // temporal stimulus of the launch's first step (NULL: none)
    float stim_w;         // this region's spatial weight
    uint32_t stim_vars;
    float* tavg_p;
    float* aff_p;         // AfferentCoupling output row of the next sample (NULL: monitor off)
    float aacc[NCV];      // its running sum
    int cd_a, a_istep;    // steps to its next sample, its period
    float* proj_p;        // projection stream row of the next sample (NULL: off)
    float pacc[MV];       // its running sums
    int cd_p, p_istep;
    double* bold_p;
    float* sub_p;
    int ph_t, ph_b, ph_i, ph_s, q_prev;
    // descriptor fields used every step, held in registers: read through the
    // descriptor pointer they would be reloaded after every store
    int t_istep, b_istep, b_ii, SL, s_istep;
    double* stock;
    const double* hrf;
    double k1v0;
    uint32_t seed, stream;

    __device__ __forceinline__ void init(const tvbk_launch& L, const tvbk_inst* Ip, int i, int n, int64_t s0) {
        const int nvoi = L.nvoi;
#pragma unroll
        for (int k = 0; k < NSV; ++k) x[k] = Ip->state[k * n + i];
#pragma unroll
        for (int k = 0; k < NP; ++k) p[k] = Ip->params[k * n + i];
        M::prepare(p);
#pragma unroll
        for (int k = 0; k < NINT; ++k) sig[k] = STOCH ? Ip->noise_sigma[k * n + i] : 0.0f;
#pragma unroll
        for (int k = 0; k < NINT; ++k)
#pragma unroll
            for (int r = 0; r < 4; ++r) zc[k][r] = 0.0f;
        const bool do_tavg = Ip->tavg != nullptr, do_bold = Ip->bold != nullptr;
#pragma unroll
        for (int v = 0; v < MV; ++v) {
            tacc[v] = (do_tavg && v < nvoi) ? Ip->tavg_acc[v * n + i] : 0.0f;
            bacc[v] = (do_bold && v < nvoi) ? Ip->bold_acc[v * n + i] : 0.0;
        }
        t_istep = Ip->tavg_istep;
        b_istep = Ip->bold_istep;
        b_ii = Ip->bold_ii;
        s_istep = Ip->sub_istep;
        SL = Ip->stock_len;
        stock = Ip->bold_stock;
        hrf = Ip->hrf;
        k1v0 = Ip->bold_k1v0;
        seed = Ip->seed;
        stream = Ip->stream;
        // monitor phases (64-bit divisions once per launch)
        ph_t = do_tavg ? (int)(s0 % Ip->tavg_istep) : 0;
        ph_b = do_bold ? (int)(s0 % Ip->bold_istep) : 0;
        ph_i = do_bold ? (int)(s0 % Ip->bold_ii) : 0;
        q_prev = do_bold ? (int)((s0 / Ip->bold_ii) % Ip->stock_len) : 0;
        ph_s = Ip->sub ? (int)(s0 % Ip->sub_istep) : 0;
        sub_p = Ip->sub ? Ip->sub + (size_t)(s0 / Ip->sub_istep - Ip->sub_base) * nvoi * n + i : nullptr;
        raw_p = Ip->raw ? Ip->raw + (size_t)(s0 - Ip->raw_base) * nvoi * n + i : nullptr;
        fed_p = Ip->noise_fed ? Ip->noise_fed + (size_t)(s0 - Ip->fed_base) * NINT * n + i : nullptr;
        tavg_p = do_tavg ? Ip->tavg + (size_t)(s0 / Ip->tavg_istep - Ip->tavg_base) * nvoi * n + i : nullptr;
        if constexpr (EXT) {
            stim_p = Ip->stim ? Ip->stim + (s0 - Ip->stim_base) : nullptr;
            stim_w = Ip->stim ? Ip->stim_weight[i] : 0.0f;
            stim_vars = Ip->stim ? Ip->stim_vars : 0u;
            a_istep = Ip->aff ? Ip->aff_istep : 1;
            aff_p = Ip->aff ? Ip->aff + (size_t)(s0 / a_istep - Ip->aff_base) * NCV * n + i : nullptr;
            cd_a = a_istep - (int)(s0 % a_istep);
#pragma unroll
            for (int k = 0; k < NCV; ++k) aacc[k] = Ip->aff ? Ip->aff_acc[k * n + i] : 0.0f;
            p_istep = Ip->proj ? Ip->proj_istep : 1;
            proj_p = Ip->proj ? Ip->proj + (size_t)(s0 / p_istep - Ip->proj_base) * nvoi * n + i : nullptr;
            cd_p = p_istep - (int)(s0 % p_istep);
#pragma unroll
            for (int v = 0; v < MV; ++v) pacc[v] = (Ip->proj && v < nvoi) ? Ip->proj_acc[v * n + i] : 0.0f;
        } else {
            stim_p = nullptr;
            stim_w = 0.0f;
            stim_vars = 0u;
            aff_p = nullptr;
            a_istep = cd_a = 1;
#pragma unroll
            for (int k = 0; k < NCV; ++k) aacc[k] = 0.0f;
            proj_p = nullptr;
            p_istep = cd_p = 1;
#pragma unroll
            for (int v = 0; v < MV; ++v) pacc[v] = 0.0f;
        }
        bold_p = do_bold ? Ip->bold + (size_t)(s0 / Ip->bold_istep - Ip->bold_base) * nvoi * n + i : nullptr;
    }

    // AfferentCoupling after a step: cn is the coupling the next step receives
    // (simulator.py:358-361 samples node_coupling of step + 1); the mean over
    // the period is written when the step is a multiple of a_istep (the
    // TemporalAverage rule, monitors.py:380-391; a_istep = 1 for Raw).
    __device__ __forceinline__ void afferent(const float* cn, int n) {
        // __fadd_rn: the coupling value is rounded before it is summed (no
        // contraction with the coupling's post into an FMA), so an average
        // taken here equals one taken on the host from the every-step stream
#pragma unroll
        for (int k = 0; k < NCV; ++k) aacc[k] = __fadd_rn(aacc[k], cn[k]);
        if (--cd_a == 0) {
            cd_a = a_istep;
            const float inv_n = (float)a_istep;
#pragma unroll
            for (int k = 0; k < NCV; ++k) {
                aff_p[k * n] = aacc[k] / inv_n;
                aacc[k] = 0.0f;
            }
            aff_p += (size_t)NCV * n;
        }
    }

    // Projection stream after a step: the mean of the observed variables over
    // p_istep steps, written when the step is a multiple of p_istep.  The
    // sensor gain is linear, so gain . mean equals the reference's per-step
    // gain products summed over the period and divided by it
    // (monitors.py:602-614); the host applies it.
    __device__ __forceinline__ void project(const tvbk_launch& L, int n) {
        if constexpr (EXT) {
            if (proj_p == nullptr) return;
            const int nvoi = L.nvoi;
#pragma unroll
            for (int v = 0; v < MV; ++v)
                if (v < nvoi) pacc[v] += M::observe(L.voi[v], x);
            if (--cd_p == 0) {
                cd_p = p_istep;
                const float inv_n = (float)p_istep;
#pragma unroll
                for (int v = 0; v < MV; ++v)
                    if (v < nvoi) {
                        proj_p[v * n] = pacc[v] / inv_n;
                        pacc[v] = 0.0f;
                    }
                proj_p += (size_t)nvoi * n;
            }
        }
    }

    // Philox normals of the 4-step block of step s (steps 4q+1 .. 4q+4, q = (s - 1) >> 2).
    __device__ __forceinline__ void noise_block(const tvbk_launch& L, int i, int64_t s) {
        if constexpr (STOCH) {
            if (L.noise == TVBK_NOISE_PHILOX) {
#pragma unroll
                for (int k = 0; k < NINT; ++k)
                    if (sig[k] != 0.0f) philox_normals4(seed, stream, s, i, k, zc[k]);
            }
        }
    }

    // Stimulus of step s0 + 1 + ks: spatial weight x temporal pattern (patterns.py:116-134).
    __device__ __forceinline__ float stim_at(int ks) const {
        if constexpr (!EXT) return 0.0f;
        return stim_p != nullptr ? stim_w * __ldg(stim_p + ks) : 0.0f;
    }

    // The scheme step with coupling input c, standard normals z and stimulus
    // value st (integrators.py:296-530), then the state-variable bounds.  The
    // stimulus reaches the variables in stim_vars; with none the added terms
    // are exact zeros and the step is the unstimulated one bit for bit.
    __device__ __forceinline__ void integrate(const float* c, const float* z, float dt, float st) {
        float m0[NSV], sv[NSV];
        M::dfun(x, c, p, m0);
#pragma unroll
        for (int k = 0; k < NSV; ++k) sv[k] = ((stim_vars >> k) & 1u) ? st : 0.0f;
        // a + stimulus, a + dt * stimulus (the identity without EXT)
        auto with_st = [&](float a, int k) -> float {
            if constexpr (EXT) return a + sv[k];
            return a;
        };
        auto add_dt_st = [&](float a, int k) -> float {
            if constexpr (EXT) return a + dt * sv[k];
            return a;
        };
        if constexpr (SCHEME == TVBK_SCHEME_EULER_DET) {
#pragma unroll
            for (int k = 0; k < NSV; ++k) x[k] = x[k] + dt * with_st(m0[k], k);
        } else if constexpr (SCHEME == TVBK_SCHEME_EULER_STOCH) {
#pragma unroll
            for (int k = 0; k < NSV; ++k) x[k] = add_dt_st(x[k] + dt * m0[k] + sig[k] * z[k], k);
        } else if constexpr (SCHEME == TVBK_SCHEME_HEUN_DET || SCHEME == TVBK_SCHEME_HEUN_STOCH) {
            float inter[NSV], nz[NSV];
#pragma unroll
            for (int k = 0; k < NSV; ++k) {
                nz[k] = STOCH ? sig[k] * z[k] : 0.0f;
                if constexpr (STOCH)
                    inter[k] = add_dt_st(x[k] + dt * m0[k] + nz[k], k);
                else  // + nz (0 here): the form of the stochastic predictor; it also schedules better
                    inter[k] = x[k] + dt * with_st(m0[k], k) + nz[k];
            }
            M::bound(inter);
            float m1[NSV];
            M::dfun(inter, c, p, m1);
            const float hdt = dt * 0.5f;
#pragma unroll
            for (int k = 0; k < NSV; ++k) x[k] = add_dt_st(x[k] + (m0[k] + m1[k]) * hdt + nz[k], k);
        } else if constexpr (SCHEME == TVBK_SCHEME_RK4) {
            const float dt2 = dt * 0.5f, dt6 = dt / 6.0f;
            float st[NSV], k2[NSV], k3[NSV], k4[NSV];
#pragma unroll
            for (int k = 0; k < NSV; ++k) st[k] = x[k] + dt2 * m0[k];
            M::bound(st);
            M::dfun(st, c, p, k2);
#pragma unroll
            for (int k = 0; k < NSV; ++k) st[k] = x[k] + dt2 * k2[k];
            M::bound(st);
            M::dfun(st, c, p, k3);
#pragma unroll
            for (int k = 0; k < NSV; ++k) st[k] = x[k] + dt * k3[k];
            M::bound(st);
            M::dfun(st, c, p, k4);
#pragma unroll
            for (int k = 0; k < NSV; ++k)
                x[k] = add_dt_st(x[k] + dt6 * (m0[k] + 2.0f * k2[k] + 2.0f * k3[k] + k4[k]), k);
        } else {  // identity
#pragma unroll
            for (int k = 0; k < NSV; ++k) x[k] = with_st(m0[k], k);
        }
        M::bound(x);
    }

    // One step s = s0 + 1 + ks with coupling input c.  The caller writes the
    // new coupling variables x[cvar(k)] to the ring.
    __device__ __forceinline__ void advance(const tvbk_launch& L, const tvbk_inst* Ip, int i, int n, int64_t s0,
                                            int ks, const float* c) {
        const float dt = L.dt;
        const int nvoi = L.nvoi;
        float z[NINT];
        if constexpr (STOCH) {
            if (L.noise == TVBK_NOISE_FED) {
#pragma unroll
                for (int k = 0; k < NINT; ++k) z[k] = fed_p[k * n];
                fed_p += (size_t)NINT * n;
            } else {
                const int r = philox_lane_of(s0 + 1 + ks);
#pragma unroll
                for (int k = 0; k < NINT; ++k)
                    z[k] = (r == 0) ? zc[k][0] : (r == 1) ? zc[k][1] : (r == 2) ? zc[k][2] : zc[k][3];
            }
        }

        integrate(c, z, dt, stim_at(ks));

        // monitors
        if (raw_p != nullptr) {
#pragma unroll
            for (int v = 0; v < MV; ++v)
                if (v < nvoi) raw_p[v * n] = M::observe(L.voi[v], x);
            raw_p += (size_t)nvoi * n;
        }
        if (tavg_p != nullptr) {
#pragma unroll
            for (int v = 0; v < MV; ++v)
                if (v < nvoi) tacc[v] += M::observe(L.voi[v], x);
            if (++ph_t == t_istep) {
                ph_t = 0;
                const float inv_n = (float)t_istep;
#pragma unroll
                for (int v = 0; v < MV; ++v)
                    if (v < nvoi) {
                        tavg_p[v * n] = tacc[v] / inv_n;
                        tacc[v] = 0.0f;
                    }
                tavg_p += (size_t)nvoi * n;
            }
        }
        if (bold_p != nullptr) {
#pragma unroll
            for (int v = 0; v < MV; ++v)
                if (v < nvoi) bacc[v] += (double)M::observe(L.voi[v], x);
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
        if (sub_p != nullptr && ++ph_s == s_istep) {
            ph_s = 0;
#pragma unroll
            for (int v = 0; v < MV; ++v)
                if (v < nvoi) sub_p[v * n] = M::observe(L.voi[v], x);
            sub_p += (size_t)nvoi * n;
        }
        project(L, n);
    }

    // ---- pieces of a step for the row kernel's blocked loop ----------------
    // Monitor clock: steps until the next TemporalAverage sample (cd_t), Bold
    // 4 ms stock write (cd_i) and Bold TR sample (cd_b); kBigCount when the
    // monitor is off.  It depends on the descriptor only, so every thread of
    // the CTA (active or not) keeps the same clock and the kernel's control
    // flow can branch on it uniformly.
    static constexpr int kBigCount = 1 << 30;
    int cd_t, cd_i, cd_b, cd_s;
    bool on_t, on_b, on_s;

    __device__ __forceinline__ void init_clock(const tvbk_inst* Ip, int64_t s0) {
        t_istep = Ip->tavg_istep;
        b_istep = Ip->bold_istep;
        b_ii = Ip->bold_ii;
        s_istep = Ip->sub_istep;
        on_t = Ip->tavg != nullptr;
        on_b = Ip->bold != nullptr;
        on_s = Ip->sub != nullptr;
        cd_s = on_s ? Ip->sub_istep - (int)(s0 % Ip->sub_istep) : kBigCount;
        cd_t = on_t ? Ip->tavg_istep - (int)(s0 % Ip->tavg_istep) : kBigCount;
        cd_i = on_b ? Ip->bold_ii - (int)(s0 % Ip->bold_ii) : kBigCount;
        cd_b = on_b ? Ip->bold_istep - (int)(s0 % Ip->bold_istep) : kBigCount;
    }

    // Per-step monitor accumulation (Raw rows, TemporalAverage and Bold sums), no sampling.
    __device__ __forceinline__ void accumulate(const tvbk_launch& L, int n) {
        const int nvoi = L.nvoi;
        if (raw_p != nullptr) {
#pragma unroll
            for (int v = 0; v < MV; ++v)
                if (v < nvoi) raw_p[v * n] = M::observe(L.voi[v], x);
            raw_p += (size_t)nvoi * n;
        }
        if (tavg_p != nullptr) {
#pragma unroll
            for (int v = 0; v < MV; ++v)
                if (v < nvoi) tacc[v] += M::observe(L.voi[v], x);
        }
        if (bold_p != nullptr) {
#pragma unroll
            for (int v = 0; v < MV; ++v)
                if (v < nvoi) bacc[v] += (double)M::observe(L.voi[v], x);
        }
        project(L, n);
    }

    // Advance the clock by m steps, the last of which is step s, and take the
    // samples that fall on step s (every thread calls it; `act` threads write).
    // m > 1 only when no sample falls on the m - 1 steps before s.
    // TemporalAverage and SubSample clocks alone (the straight-line block takes
    // their samples at any of its steps, one step at a time)
    __device__ __forceinline__ void tick_t(int m, bool act, int n, int nvoi) {
        if (on_t) cd_t -= m;
        if (cd_t == 0) {
            cd_t = t_istep;
            if (act) {
                const float inv_n = (float)t_istep;
#pragma unroll
                for (int v = 0; v < MV; ++v)
                    if (v < nvoi) {
                        tavg_p[v * n] = tacc[v] / inv_n;
                        tacc[v] = 0.0f;
                    }
                tavg_p += (size_t)nvoi * n;
            }
        }
    }

    __device__ __forceinline__ void tick_s(const tvbk_launch& L, int m, bool act, int n, int nvoi) {
        if (on_s) cd_s -= m;
        if (cd_s == 0) {
            cd_s = s_istep;
            if (act) {
#pragma unroll
                for (int v = 0; v < MV; ++v)
                    if (v < nvoi) sub_p[v * n] = M::observe(L.voi[v], x);
                sub_p += (size_t)nvoi * n;
            }
        }
    }

    // ts = false: the TemporalAverage and SubSample clocks were already advanced step by step
    __device__ __forceinline__ void tick(const tvbk_launch& L, int m, bool act, int64_t s, int i, int n,
                                         bool ts = true) {
        const int nvoi = L.nvoi;
        if (ts) tick_t(m, act, n, nvoi);
        if (on_b) {
            cd_i -= m;
            cd_b -= m;
        }
        if (cd_i == 0) {
            cd_i = b_ii;
            if (act) {
                double* st = stock + (size_t)q_prev * nvoi * n + i;
#pragma unroll
                for (int v = 0; v < MV; ++v)
                    if (v < nvoi) {
                        st[v * n] = bacc[v] / (double)b_ii;
                        bacc[v] = 0.0;
                    }
                q_prev = (q_prev + 1 == SL) ? 0 : q_prev + 1;
            }
        }
        if (cd_b == 0) {
            cd_b = b_istep;
            if (act) bold_sample(s, i, n, nvoi);
        }
        if (ts) tick_s(L, m, act, n, nvoi);
    }

    // Bold output at step s: (hrf . stock - 1) k1 V0 with the kernel rolled to the current stock position.
    __device__ __forceinline__ void bold_sample(int64_t s, int i, int n, int nvoi) {
        const int m = (int)((s / b_ii) % SL);
        // numpy.roll(hrf, m - 1)[k] == hrf[(k - m + 1) mod SL]
        int idx0 = 1 - m;
        idx0 = idx0 < 0 ? idx0 + SL : (idx0 >= SL ? idx0 - SL : idx0);
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

    // Standard normals of step s from the fed array or the Philox block held in zc.
    __device__ __forceinline__ void fetch_z(const tvbk_launch& L, int n, int64_t s, float* z) {
        if constexpr (STOCH) {
            if (L.noise == TVBK_NOISE_FED) {
#pragma unroll
                for (int k = 0; k < NINT; ++k) z[k] = fed_p[k * n];
                fed_p += (size_t)NINT * n;
            } else {
                const int r = philox_lane_of(s);
#pragma unroll
                for (int k = 0; k < NINT; ++k)
                    z[k] = (r == 0) ? zc[k][0] : (r == 1) ? zc[k][1] : (r == 2) ? zc[k][2] : zc[k][3];
            }
        }
    }

    // Philox normals of the block of step s into dst (every state variable with a non-zero sigma).
    __device__ __forceinline__ void philox_block(int i, int64_t s, float (*dst)[4]) {
        if constexpr (STOCH) {
#pragma unroll
            for (int k = 0; k < NINT; ++k)
                if (NINT == 1 || sig[k] != 0.0f) philox_normals4(seed, stream, s, i, k, dst[k]);
        }
    }

    // history update: the coupling variables of the new state go to dst
    __device__ __forceinline__ void write_ring(float* dst) const {
        if constexpr (NCV == 1) {
            dst[0] = x[M::cvar(0)];
        } else {
            *reinterpret_cast<float2*>(dst) = make_float2(x[M::cvar(0)], x[M::cvar(1)]);
        }
    }

    __device__ __forceinline__ void finish(const tvbk_launch& L, tvbk_inst* Ip, int i, int n, int32_t* status) {
        const int nvoi = L.nvoi;
        bool finite = true;
#pragma unroll
        for (int k = 0; k < NSV; ++k) {
            Ip->state[k * n + i] = x[k];
            finite = finite && isfinite(x[k]);
        }
#pragma unroll
        for (int v = 0; v < MV; ++v)
            if (v < nvoi) {
                if (Ip->tavg != nullptr) Ip->tavg_acc[v * n + i] = tacc[v];
                if (Ip->bold != nullptr) Ip->bold_acc[v * n + i] = bacc[v];
            }
        if (EXT && aff_p != nullptr) {
#pragma unroll
            for (int k = 0; k < NCV; ++k) Ip->aff_acc[k * n + i] = aacc[k];
        }
        if (EXT && proj_p != nullptr) {
#pragma unroll
            for (int v = 0; v < MV; ++v)
                if (v < nvoi) Ip->proj_acc[v * n + i] = pacc[v];
        }
        if (!finite) atomicOr(status, TVBK_STATUS_NONFINITE);
    }
};

__device__ __forceinline__ void stage_ring(float* dst, const float* src, int nfloats) {
    const float4* s4 = reinterpret_cast<const float4*>(src);
    float4* d4 = reinterpret_cast<float4*>(dst);
    const int n4 = nfloats >> 2;
    for (int k = threadIdx.x; k < n4; k += blockDim.x) d4[k] = s4[k];
    for (int k = (n4 << 2) + threadIdx.x; k < nfloats; k += blockDim.x) dst[k] = src[k];
}

// Row kernel: thread i gathers row i and advances region i.  With PIPE the
// gather of step s + 1 is issued before the update of step s (it reads times
// <= s - d_min only, so it does not wait for this step), which gives each
// warp two independent instruction streams; it needs every delay >= 1, a
// barrier interval K <= d_min, and a coupling whose pre() ignores x_i.
// EXT = false: no region stimulus and no AfferentCoupling monitor (launch.extras
// == 0); an instance that asks for either gets TVBK_STATUS_UNSUPPORTED.
template <class M, int CF, int SCHEME, bool SMEM, int MAXT, int MAXD, bool PIPE, bool EXT = true>
__global__ void __launch_bounds__(MAXT) sim_kernel(const tvbk_launch L) {
    constexpr int NCV = M::NCV;
    constexpr bool SIGMA = GatherTraits<CF, NCV>::SIGMA;
    constexpr int NG = GatherTraits<CF, NCV>::NG;
    extern __shared__ __align__(16) float smem[];

    // this CTA's instance: the launch may take a subset of the batch through inst_order
    const int b = L.inst_order != nullptr ? L.inst_order[blockIdx.x] : (int)blockIdx.x;
    tvbk_inst* __restrict__ Ip = L.insts + b;
    int32_t* const status = L.status + b;
    const int n = Ip->n;
    const int i = threadIdx.x;
    const bool act = i < n;
    const int RL = Ip->ring_len;
    const int slot_floats = n * NG;             // the gather ring: NG floats per (slot, region)
    const int ring_floats = RL * slot_floats;
    const int64_t s0 = Ip->step;
    const int64_t s_end = min(Ip->step_end, s0 + L.max_steps);
    if (s0 >= s_end) return;  // uniform over the block
    const int nsteps = (int)(s_end - s0);

    float cf[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) cf[k] = Ip->cfun[k];
    // gather ring: the raw ring (staged in shared memory or in place), or for
    // SigmoidalJansenRit the pre-applied sigmoid values computed from it
    float* ring = SMEM ? smem : (SIGMA ? Ip->pre_ring : Ip->ring);
    // A ring staged in shared memory for the prefetching loop has TVBK_RING_GUARD
    // slots past its end that mirror slots 0..GUARD-1 (the four-step gathers of
    // couple4 read up to three slots past a wrapped address); every write of
    // one of those slots also goes to its mirror.
    constexpr bool GUARDED = SMEM && PIPE && MAXD > 0;
    constexpr int GUARD = GUARDED ? TVBK_RING_GUARD : 0;
    if constexpr (SIGMA) {
        sigma_ring(ring, Ip->ring, RL * n, threadIdx.x, blockDim.x, cf);
        if constexpr (GUARDED) sigma_ring(ring + ring_floats, Ip->ring, GUARD * n, threadIdx.x, blockDim.x, cf);
        __syncthreads();
    } else if (SMEM) {
        stage_ring(smem, Ip->ring, ring_floats);
        if constexpr (GUARDED)
            for (int k = threadIdx.x; k < GUARD * slot_floats; k += blockDim.x) smem[ring_floats + k] = Ip->ring[k];
        __syncthreads();
    }
    RegRow<M, CF, MAXD> row;
    row.deg = 0;
    Node<M, SCHEME, EXT> node;
    if (act) {
        const int e0 = Ip->row_ptr[i], e1 = Ip->row_ptr[i + 1];
        if (MAXD > 0 && e1 - e0 > MAXD) atomicOr(status, TVBK_STATUS_DEGREE);
        if (!EXT && (Ip->stim != nullptr || Ip->aff != nullptr || Ip->proj != nullptr))
            atomicOr(status, TVBK_STATUS_UNSUPPORTED);
        if constexpr (MAXD > 0) {
            if (Ip->slots != nullptr && Ip->slot_width == MAXD)
                row.load_slots(Ip->slots, i, e0, e1);
            else
                row.load(Ip->edges, e0, e1);
        } else {
            row.load(Ip->edges, e0, e1);
        }
        node.init(L, Ip, i, n, s0);
    }
    const int K = L.sync_every;
    int since_sync = 0;
    int wslot = (int)(s0 % RL);  // slot of the last written time
    // the new state's coupling variables go to the gather ring (and the raw history for SigmoidalJansenRit)
    auto write = [&](int slot) {
        if constexpr (SIGMA) {
            node.write_ring(Ip->ring + (size_t)slot * n * NCV + i * NCV);
            const float v = sjr_pre(node.x[M::cvar(0)], node.x[M::cvar(1)], cf);
            ring[slot * slot_floats + i] = v;
            if (GUARDED && slot < GUARD) ring[(slot + RL) * slot_floats + i] = v;
        } else {
            node.write_ring(ring + slot * slot_floats + i * NCV);
            if (GUARDED && slot < GUARD) node.write_ring(ring + (slot + RL) * slot_floats + i * NCV);
        }
    };
    if constexpr (!PIPE) {
        for (int ks = 0; ks < nsteps; ++ks) {
            const int prev = wslot;                     // slot of time s - 1
            wslot = (wslot + 1 == RL) ? 0 : wslot + 1;  // time s
            if (act) {
                if (STOCH_BLOCK_START(ks)) node.noise_block(L, i, s0 + 1 + ks);
                float c[NCV], xi[NCV];
#pragma unroll
                for (int k = 0; k < NCV; ++k) xi[k] = node.x[M::cvar(k)];
                row.couple(ring, prev * slot_floats, ring_floats, xi, cf, c, L.cfun);
                node.advance(L, Ip, i, n, s0, ks, c);
                write(wslot);
            }
            if (++since_sync == K) {
                since_sync = 0;
                __syncthreads();
            }
            // AfferentCoupling: the coupling of step s + 1, gathered where the
            // next iteration would gather it (after its barrier)
            if (EXT && act && node.aff_p != nullptr) {
                float cn[NCV], xi[NCV];
#pragma unroll
                for (int k = 0; k < NCV; ++k) xi[k] = node.x[M::cvar(k)];
                row.couple(ring, wslot * slot_floats, ring_floats, xi, cf, cn, L.cfun);
                node.afferent(cn, n);
            }
        }
    } else {
        // Blocked loop: steps go in blocks of four aligned to the Philox noise
        // blocks (s = 4q + 1 .. 4q + 4).  A block with no monitor sample before its
        // last step runs as straight-line code -- the four steps' normals come
        // from registers, the next block's normals are drawn in between, the
        // monitors only accumulate, and the samples that fall on its last step
        // are taken after it; every other step (the launch's first partial
        // block, blocks with a sample inside, fed noise, a barrier interval
        // below 4) runs one at a time.  Both paths do the same arithmetic.
        node.init_clock(Ip, s0);
        const bool fed = L.noise == TVBK_NOISE_FED;
        int64_t zq = -1;  // Philox block whose normals are in node.zc
        float cnext[NCV];
        if (act) row.couple(ring, wslot * slot_floats, ring_floats, node.x, cf, cnext);
        int64_t s = s0 + 1;  // the step to do next
        int ks = 0;
        while (ks < nsteps) {
            // TemporalAverage / SubSample samples may fall anywhere in a block, Bold ones only on its last step
            const bool fast = !fed && K >= 4 && philox_lane_of(s) == 0 && nsteps - ks >= 4 && node.cd_i >= 4 &&
                              node.cd_b >= 4;  // uniform over the CTA
            if (fast) {
                if (since_sync + 4 > K) {
                    since_sync = 0;
                    __syncthreads();
                }
                // a TemporalAverage or SubSample sample before the block's last step: the block takes the
                // samples step by step (a second copy of the block); else its clocks advance at its end
                const bool inside = node.cd_t < 4 || node.cd_s < 4;  // uniform over the CTA
                auto block = [&](auto inside_tag) {
                    constexpr bool IN = decltype(inside_tag)::value;
                    if (act) {
                        if (SchemeTraits<SCHEME>::stoch && zq != philox_block_of(s)) node.philox_block(i, s, node.zc);
                        // variables with a zero sigma draw nothing: their normals stay 0 (0 * z must not see garbage)
                        float zn[M::NINT][4] = {};
                        // the couplings of steps s + 1 .. s + 4, all gathered first: they read times
                        // s + r - d <= s - 1 (d >= d_min >= K >= 4), none written in this block, so the
                        // four gathers are independent of the block's updates and of each other
                        float cb[4][NCV];
                        (void)cb;
                        if constexpr (GUARDED) {
                            const int s0slot = (wslot + 1 == RL) ? 0 : wslot + 1;  // slot of time s
                            row.couple4(ring, s0slot * slot_floats, ring_floats, slot_floats, cf, cb);
                        }
#pragma unroll
                        for (int r = 0; r < 4; ++r) {
                            float c[NCV], z[M::NINT];
#pragma unroll
                            for (int k = 0; k < NCV; ++k) c[k] = cnext[k];
                            wslot = (wslot + 1 == RL) ? 0 : wslot + 1;  // time s + r
                            if constexpr (GUARDED) {
#pragma unroll
                                for (int k = 0; k < NCV; ++k) cnext[k] = cb[r][k];
                            } else {
                                row.couple(ring, wslot * slot_floats, ring_floats, node.x, cf, cnext);
                            }
                            if (r == 1) node.philox_block(i, s + 4, zn);  // the next block's normals
#pragma unroll
                            for (int k = 0; k < M::NINT; ++k) z[k] = node.zc[k][r];
                            node.integrate(c, z, L.dt, node.stim_at(ks + r));
                            node.accumulate(L, n);
                            if constexpr (IN) {
                                node.tick_t(1, true, n, L.nvoi);
                                node.tick_s(L, 1, true, n, L.nvoi);
                            }
                            if (EXT && node.aff_p != nullptr) node.afferent(cnext, n);
                            write(wslot);
                        }
                        if constexpr (SchemeTraits<SCHEME>::stoch) {
#pragma unroll
                            for (int k = 0; k < M::NINT; ++k)
#pragma unroll
                                for (int r = 0; r < 4; ++r) node.zc[k][r] = zn[k][r];
                        }
                    } else {
#pragma unroll
                        for (int r = 0; r < 4; ++r) {
                            wslot = (wslot + 1 == RL) ? 0 : wslot + 1;
                            if constexpr (IN) {
                                node.tick_t(1, false, n, L.nvoi);
                                node.tick_s(L, 1, false, n, L.nvoi);
                            }
                        }
                    }
                    node.tick(L, 4, act, s + 3, i, n, !IN);
                };
                if (inside)
                    block(std::true_type{});
                else
                    block(std::false_type{});
                zq = philox_block_of(s) + 1;
                since_sync += 4;
                s += 4;
                ks += 4;
            } else {
                wslot = (wslot + 1 == RL) ? 0 : wslot + 1;  // time s
                if (act) {
                    if (SchemeTraits<SCHEME>::stoch && !fed && zq != philox_block_of(s))
                        node.philox_block(i, s, node.zc);
                    float c[NCV], z[M::NINT];
#pragma unroll
                    for (int k = 0; k < NCV; ++k) c[k] = cnext[k];
                    // coupling of step s + 1: times s - d with d >= d_min >= 1
                    row.couple(ring, wslot * slot_floats, ring_floats, node.x, cf, cnext);
                    node.fetch_z(L, n, s, z);
                    node.integrate(c, z, L.dt, node.stim_at(ks));
                    node.accumulate(L, n);
                    if (EXT && node.aff_p != nullptr) node.afferent(cnext, n);
                    write(wslot);
                }
                zq = philox_block_of(s);
                node.tick(L, 1, act, s, i, n);
                if (++since_sync == K) {
                    since_sync = 0;
                    __syncthreads();
                }
                s += 1;
                ks += 1;
            }
        }
    }
    __syncthreads();
    if (act) node.finish(L, Ip, i, n, status);
    if (SMEM && !SIGMA) stage_ring(Ip->ring, smem, ring_floats);
    if (i == 0) Ip->step = s_end;
}

// Edge-parallel kernel (ring in shared memory; Linear or SigmoidalJansenRit,
// whose pre() depends on the source region only).  Each step, thread t
// gathers edges [t*E, t*E + E) of the row-major edge list (E <= MAXE and
// E <= the smallest non-zero row degree, so the range covers at most two
// rows) into two partial sums; after one barrier, thread i < n adds the
// partials that cover row i and advances region i.  Partials are double
// buffered by step parity, so the next step's gather can start while other
// threads still read this step's partials; the ring needs no extra barrier
// when every delay is >= 1 (reads stop at time s - 1 - d_min), else a second
// barrier per step is taken.
template <class M, int CF, int SCHEME, int MAXE>
__global__ void __launch_bounds__(512) sim_kernel_ep(const tvbk_launch L) {
    constexpr int NCV = M::NCV;
    constexpr int NACC = (CF == CF_SIGMOIDAL_JR) ? 1 : NCV;
    extern __shared__ __align__(16) float smem[];

    tvbk_inst* __restrict__ Ip = L.insts + blockIdx.x;
    const int n = Ip->n;
    const int t = threadIdx.x;
    const int T = blockDim.x;
    const bool act = t < n;
    const int RL = Ip->ring_len;
    const int slot_floats = n * NCV;
    const int ring_floats = RL * slot_floats;
    const int64_t s0 = Ip->step;
    const int64_t s_end = min(Ip->step_end, s0 + L.max_steps);
    if (s0 >= s_end) return;  // uniform over the block
    const int nsteps = (int)(s_end - s0);
    float* ring = smem;
    float* part = smem + ((ring_floats + 3) & ~3);  // [2][T][2][NACC]
    stage_ring(smem, Ip->ring, ring_floats);

    const int nnz = Ip->nnz;
    const int E = (nnz + T - 1) / T;
    if (E > MAXE) {
        if (t == 0) atomicOr(L.status + blockIdx.x, TVBK_STATUS_DEGREE);
        return;  // uniform over the block
    }
    // this thread's edges: two weight sets split at kb (start of the second row)
    const int eb = t * E;
    const int cnt = max(0, min(E, nnz - eb));
    int kb = MAXE;
    if (cnt > 0) {
        int lo = 0, hi = n - 1;  // largest r with row_ptr[r] <= eb
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(Ip->row_ptr + mid) <= eb) lo = mid; else hi = mid - 1;
        }
        kb = min(__ldg(Ip->row_ptr + lo + 1) - eb, cnt);
    }
    int off[MAXE];
    float wa[MAXE], wb[MAXE];
    const int2* ed2 = reinterpret_cast<const int2*>(Ip->edges) + eb;
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        const int2 ed = (k < cnt) ? __ldg(ed2 + k) : make_int2(0, 0);
        off[k] = ed.x;
        const float w = __int_as_float(ed.y);
        wa[k] = (k < kb) ? w : 0.0f;
        wb[k] = (k < kb) ? 0.0f : w;
    }
    // which partials make up row t
    int tf = -1, sf = 0, tl = -1;
    Node<M, SCHEME> node;
    float cf[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) cf[k] = Ip->cfun[k];
    if (act) {
        const int e0 = Ip->row_ptr[t], e1 = Ip->row_ptr[t + 1];
        if (e1 > e0) {
            tf = e0 / E;
            sf = (e0 == tf * E) ? 0 : 1;
            tl = (e1 - 1) / E;
        }
        node.init(L, Ip, t, n, s0);
        if (Ip->aff != nullptr) atomicOr(L.status + blockIdx.x, TVBK_STATUS_UNSUPPORTED);
    }
    __syncthreads();

    const bool zero_delay = L.sync_every <= 1;
    int wslot = (int)(s0 % RL);
    int par = 0;
    for (int ks = 0; ks < nsteps; ++ks) {
        if (act && STOCH_BLOCK_START(ks)) node.noise_block(L, t, s0 + 1 + ks);
        const int base_off = wslot * slot_floats;  // time s - 1
        wslot = (wslot + 1 == RL) ? 0 : wslot + 1;  // time s
        float pa[NACC], pb[NACC];
#pragma unroll
        for (int k = 0; k < NACC; ++k) pa[k] = pb[k] = 0.0f;
#pragma unroll
        for (int k = 0; k < MAXE; ++k) {
            const float* src = ring + gather_addr(base_off, off[k], ring_floats);
            if constexpr (CF == CF_SIGMOIDAL_JR) {
                const float2 v = *reinterpret_cast<const float2*>(src);
                const float pre = cf[0] + (cf[1] - cf[0]) / (1.0f + expf(cf[3] * (cf[2] - (v.x - v.y))));
                pa[0] = fmaf(wa[k], pre, pa[0]);
                pb[0] = fmaf(wb[k], pre, pb[0]);
            } else if constexpr (NCV == 1) {
                const float v = src[0];
                pa[0] = fmaf(wa[k], v, pa[0]);
                pb[0] = fmaf(wb[k], v, pb[0]);
            } else {
                const float2 v = *reinterpret_cast<const float2*>(src);
                pa[0] = fmaf(wa[k], v.x, pa[0]);
                pa[1] = fmaf(wa[k], v.y, pa[1]);
                pb[0] = fmaf(wb[k], v.x, pb[0]);
                pb[1] = fmaf(wb[k], v.y, pb[1]);
            }
        }
        float* pp = part + ((size_t)par * T + t) * 2 * NACC;
#pragma unroll
        for (int k = 0; k < NACC; ++k) {
            pp[k] = pa[k];
            pp[NACC + k] = pb[k];
        }
        __syncthreads();
        if (act) {
            float acc[NCV];
#pragma unroll
            for (int k = 0; k < NCV; ++k) acc[k] = 0.0f;
            if (tf >= 0) {
                const float* base = part + (size_t)par * T * 2 * NACC;
#pragma unroll
                for (int k = 0; k < NACC; ++k) acc[k] = base[(tf * 2 + sf) * NACC + k];
                for (int u = tf + 1; u <= tl; ++u) {
#pragma unroll
                    for (int k = 0; k < NACC; ++k) acc[k] += base[u * 2 * NACC + k];
                }
            }
            float c[NCV];
            post<CF, NCV>(acc, cf, c);
            node.advance(L, Ip, t, n, s0, ks, c);
            node.write_ring(ring + wslot * slot_floats + t * NCV);
        }
        if (zero_delay) __syncthreads();
        par ^= 1;
    }
    __syncthreads();
    if (act) node.finish(L, Ip, t, n, L.status + blockIdx.x);
    stage_ring(Ip->ring, smem, ring_floats);
    if (t == 0) Ip->step = s_end;
}

// ------------------------------------------------------------------ launch

template <class M, int CF, int SCHEME, bool SMEM, int MAXT, int MAXD, bool PIPE = false, bool EXT = true>
int launch_one(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes) {
    auto kern = sim_kernel<M, CF, SCHEME, SMEM, MAXT, MAXD, PIPE, EXT>;
    if (smem_bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
        if (e != cudaSuccess) return (int)e;
    }
    const int threads = ((L.max_n + 31) / 32) * 32;
    if (L.occupancy != nullptr) {  // a query: resident CTAs per SM of this variant, no launch
        int nb = 0;
        const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads, smem_bytes);
        *L.occupancy = nb;
        return (int)e;
    }
    kern<<<L.n_inst, threads, smem_bytes, st>>>(L);
    return (int)cudaGetLastError();
}

// max_deg: the largest row degree over all instances of the launch.
template <class M, int CF, int SCHEME, bool SMEM, int MAXT>
int launch_deg(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes, int max_deg) {
    if (max_deg <= 0) return launch_one<M, CF, SCHEME, SMEM, MAXT, 0>(L, st, smem_bytes);
    if constexpr (CF != CF_DIFFERENCE && CF != CF_GENERIC) {
        if (L.prefetch) {
            // rings in shared memory without stimulus or AfferentCoupling: the lean build
            if (SMEM && L.extras == 0) {
                if (max_deg <= 32) return launch_one<M, CF, SCHEME, SMEM, MAXT, 32, true, false>(L, st, smem_bytes);
                if (max_deg <= 64) return launch_one<M, CF, SCHEME, SMEM, MAXT, 64, true, false>(L, st, smem_bytes);
            }
            if (max_deg <= 32) return launch_one<M, CF, SCHEME, SMEM, MAXT, 32, true>(L, st, smem_bytes);
            if (max_deg <= 64) return launch_one<M, CF, SCHEME, SMEM, MAXT, 64, true>(L, st, smem_bytes);
        }
    }
    if (max_deg <= 32) return launch_one<M, CF, SCHEME, SMEM, MAXT, 32>(L, st, smem_bytes);
    if (max_deg <= 64) return launch_one<M, CF, SCHEME, SMEM, MAXT, 64>(L, st, smem_bytes);
    return launch_one<M, CF, SCHEME, SMEM, MAXT, 0>(L, st, smem_bytes);
}

template <class M, int CF, int SCHEME, int MAXE>
int launch_ep(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes) {
    auto kern = sim_kernel_ep<M, CF, SCHEME, MAXE>;
    if (smem_bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
        if (e != cudaSuccess) return (int)e;
    }
    kern<<<L.n_inst, L.block_threads, smem_bytes, st>>>(L);
    return (int)cudaGetLastError();
}

template <class M, int CF, int SCHEME>
int launch_scheme(const tvbk_launch& L, cudaStream_t st, size_t smem_bytes, int max_deg) {
    if (L.edges_per_thread > 0) {
        if constexpr (CF == CF_DIFFERENCE || CF == CF_GENERIC) {
            return -2;
        } else {
            if (!L.ring_in_smem) return -2;
            switch (L.edges_per_thread) {
                case 8: return launch_ep<M, CF, SCHEME, 8>(L, st, smem_bytes);
                case 12: return launch_ep<M, CF, SCHEME, 12>(L, st, smem_bytes);
                case 16: return launch_ep<M, CF, SCHEME, 16>(L, st, smem_bytes);
                case 24: return launch_ep<M, CF, SCHEME, 24>(L, st, smem_bytes);
                default: return -2;
            }
        }
    }
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
