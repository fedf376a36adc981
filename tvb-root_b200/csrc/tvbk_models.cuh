// Model derivatives, observables and coupling functions, float32.
//
// Each model is a struct with its dimensions, its parameter order (the order
// the host packs tvbk_inst.params in), dfun() in the operation order of the
// reference's numba gufunc, observe() for the variables-of-interest
// expressions and bound() for state-variable boundaries.
#pragma once
#include <cstdint>

namespace tvbk {

// Ring address (in floats) of an edge's delayed value: base_off is the ring
// offset of time s - 1, edge_off = (idelay * n - col) * ncvar.  The slot of
// time s - 1 - idelay wraps around when base_off - edge_off is negative.
__device__ __forceinline__ int gather_addr(int base_off, int edge_off, int ring_floats) {
    // as unsigned, a negative base_off - edge_off is above every wrapped address:
    // min(a, a + ring_floats) picks the in-ring one (one fused add-min)
    const unsigned a = (unsigned)(base_off - edge_off);
    return (int)__viaddmin_u32(a, (unsigned)ring_floats, a);
}

// Generic2dOscillator (tvb/simulator/models/oscillator.py:387-395).
// params: tau, I, a, b, c, d, e, f, g, alpha, beta, gamma
struct G2D {
    static constexpr int NSV = 2, NCV = 1, NINT = 2, NOBS = 4, NP = 12, NPX = NP;
    __device__ static constexpr int cvar(int k) { return 0; }
    __device__ __forceinline__ static void prepare(float* p) {}
    __device__ __forceinline__ static void dfun(const float* x, const float* c, const float* p, float* dx) {
        const float V = x[0], W = x[1];
        const float V2 = V * V;
        const float tau = p[0], I = p[1], a = p[2], b = p[3], cc = p[4], d = p[5], e = p[6], f = p[7],
                    g = p[8], alpha = p[9], beta = p[10], gamma = p[11];
        dx[0] = d * tau * (alpha * W - f * V2 * V + e * V2 + g * V + gamma * I + gamma * c[0]);
        dx[1] = d * (a + b * V + cc * V2 - beta * W) / tau;
    }
    // choices: V, W, V + W, V - W (oscillator.py:318-323)
    __device__ __forceinline__ static float observe(int k, const float* x) {
        switch (k) {
            case 0: return x[0];
            case 1: return x[1];
            case 2: return x[0] + x[1];
            default: return x[0] - x[1];
        }
    }
    __device__ __forceinline__ static void bound(float* x) {}
};

// JansenRit (tvb/simulator/models/jansen_rit.py:274-289); coupling enters dy4 via c[0].
// params: A, B, a, b, v0, nu_max, r, J, a_1, a_2, a_3, a_4, mu
struct JansenRit {
    static constexpr int NSV = 6, NCV = 2, NINT = 6, NOBS = 6, NP = 13, NPX = NP;
    __device__ static constexpr int cvar(int k) { return k == 0 ? 1 : 2; }
    __device__ __forceinline__ static void prepare(float* p) {}
    __device__ __forceinline__ static void dfun(const float* y, const float* c, const float* p, float* dx) {
        const float A = p[0], B = p[1], a = p[2], b = p[3], v0 = p[4], nu = p[5], r = p[6], J = p[7],
                    a1 = p[8], a2 = p[9], a3 = p[10], a4 = p[11], mu = p[12];
        const float s12 = 2.0f * nu / (1.0f + expf(r * (v0 - (y[1] - y[2]))));
        const float s01 = 2.0f * nu / (1.0f + expf(r * (v0 - (a1 * J * y[0]))));
        const float s03 = 2.0f * nu / (1.0f + expf(r * (v0 - (a3 * J * y[0]))));
        dx[0] = y[3];
        dx[1] = y[4];
        dx[2] = y[5];
        dx[3] = A * a * s12 - 2.0f * a * y[3] - a * a * y[0];
        dx[4] = A * a * (mu + a2 * J * s01 + c[0]) - 2.0f * a * y[4] - a * a * y[1];
        dx[5] = B * b * (a4 * J * s03) - 2.0f * b * y[5] - b * b * y[2];
    }
    __device__ __forceinline__ static float observe(int k, const float* x) {
        float v = x[0];
#pragma unroll
        for (int s = 1; s < NSV; ++s)
            if (k == s) v = x[s];
        return v;
    }
    __device__ __forceinline__ static void bound(float* x) {}
};

// z / (1 - exp(-z)) for |z| <= 1 from its Bernoulli-number series,
//   z / (1 - e^-z) = 1 + z/2 + sum_k B_2k z^2k / (2k)!
//                  = 1 + z/2 + z^2/12 - z^4/720 + z^6/30240 - z^8/1209600 + z^10/47900160 - ...
// (B_2 = 1/6, B_4 = -1/30, B_6 = 1/42, B_8 = -1/30, B_10 = 5/66).  Truncated
// after z^10: the rest is below 9e-10 relative on |z| <= 1, far under float32
// rounding.  Even powers only, so the polynomial runs in w = z^2: five
// dependent fmas instead of the thirteen of a Taylor series in z.
__device__ __forceinline__ float z_over_one_minus_exp(float z) {
    const float w = z * z;
    float q = 1.0f / 47900160.0f;
    q = fmaf(q, w, -1.0f / 1209600.0f);
    q = fmaf(q, w, 1.0f / 30240.0f);
    q = fmaf(q, w, -1.0f / 720.0f);
    q = fmaf(q, w, 1.0f / 12.0f);
    return fmaf(w, q, fmaf(z, 0.5f, 1.0f));
}

// ReducedWongWang (tvb/simulator/models/wong_wang.py:36-42); S bounded to [0, 1] (wong_wang.py:129-133).
// params: a, b, d, gamma, tau_s, w, J_N, I_o; prepare() replaces tau_s by 1 / tau_s and appends
// 1 / d and w J_N (NPX = 10 kernel-side values)
//
// H(x) = (a x - b) / (1 - exp(-d (a x - b))) = y / (1 - exp(-z)) with
// y = a x - b, z = d y.  For |z| <= 1 it is (1 / d) * z / (1 - exp(-z)),
// the series above: no cancellation near y = 0 and no 0/0 at y = 0 (the
// limit 1/d comes out of the same expression); for |z| > 1, where
// 1 - exp(-z) does not cancel, y / (1 - exp(-z)) with the hardware
// exponential and reciprocal (__fdividef: for z -> -inf the denominator
// overflows to -inf and H to the limit 0).  Both forms are evaluated and one
// is selected (no branch).
struct RWW {
    static constexpr int NSV = 1, NCV = 1, NINT = 1, NOBS = 1, NP = 8, NPX = 10;
    __device__ static constexpr int cvar(int k) { return 0; }
    __device__ __forceinline__ static void prepare(float* p) {
        p[4] = 1.0f / p[4];
        p[8] = 1.0f / p[2];
        p[9] = p[5] * p[6];
    }
    __device__ __forceinline__ static void dfun(const float* x, const float* c, const float* p, float* dx) {
        const float S = x[0];
        const float a = p[0], b = p[1], d = p[2], gamma = p[3], inv_tau_s = p[4], JN = p[6], Io = p[7];
        const float inv_d = p[8], wJN = p[9];
        const float xx = wJN * S + Io + JN * c[0];
        const float y = a * xx - b;
        const float z = d * y;
        const float h_small = z_over_one_minus_exp(z) * inv_d;
        const float h_large = __fdividef(y, 1.0f - __expf(-z));
        const float h = fabsf(z) <= 1.0f ? h_small : h_large;
        dx[0] = fmaf((1.0f - S) * h, gamma, -(S * inv_tau_s));
    }
    __device__ __forceinline__ static float observe(int k, const float* x) { return x[0]; }
    __device__ __forceinline__ static void bound(float* x) { x[0] = fminf(fmaxf(x[0], 0.0f), 1.0f); }
};

// Epileptor (tvb/simulator/models/epileptor.py:36-71).
// params: a, b, c, d, r, x0, Iext, slope, Iext2, tau, aa, bb, Kvf, Kf, Ks, tt, modification
struct Epileptor {
    static constexpr int NSV = 6, NCV = 2, NINT = 6, NOBS = 7, NP = 17, NPX = NP;
    __device__ static constexpr int cvar(int k) { return k == 0 ? 0 : 3; }
    __device__ __forceinline__ static void prepare(float* p) {}
    __device__ __forceinline__ static void dfun(const float* y, const float* c, const float* p, float* dx) {
        const float a = p[0], b = p[1], cc = p[2], d = p[3], r = p[4], x0 = p[5], Iext = p[6], slope = p[7],
                    Iext2 = p[8], tau = p[9], aa = p[10], bb = p[11], Kvf = p[12], Kf = p[13], Ks = p[14],
                    tt = p[15], modification = p[16];
        const float cp1 = c[0], cp2 = c[1];
        float f1;
        if (y[0] < 0.0f)
            f1 = -a * y[0] * y[0] + b * y[0];
        else
            f1 = slope - y[3] + 0.6f * (y[2] - 4.0f) * (y[2] - 4.0f);
        dx[0] = tt * (y[1] - y[2] + Iext + Kvf * cp1 + f1 * y[0]);
        dx[1] = tt * (cc - d * y[0] * y[0] - y[1]);
        float z7 = 0.0f;
        if (y[2] < 0.0f) {
            const float z2 = y[2] * y[2];
            z7 = -0.1f * (z2 * z2 * z2 * y[2]);
        }
        float h;
        if (modification != 0.0f)
            h = x0 + 3.0f / (1.0f + expf(-(y[0] + 0.5f) / 0.1f));
        else
            h = 4.0f * (y[0] - x0) + z7;
        dx[2] = tt * (r * (h - y[2] + Ks * cp1));
        dx[3] = tt * (-y[4] + y[3] - y[3] * y[3] * y[3] + Iext2 + bb * y[5] - 0.3f * (y[2] - 3.5f) + Kf * cp2);
        const float f2 = (y[3] < -0.25f) ? 0.0f : aa * (y[3] + 0.25f);
        dx[4] = tt * ((-y[4] + f2) / tau);
        dx[5] = tt * (-0.01f * (y[5] - 0.1f * y[0]));
    }
    // choices: x1, y1, z, x2, y2, g, x2 - x1 (epileptor.py:262-268)
    __device__ __forceinline__ static float observe(int k, const float* x) {
        if (k == 6) return x[3] - x[0];
        float v = x[0];
#pragma unroll
        for (int s = 1; s < NSV; ++s)
            if (k == s) v = x[s];
        return v;
    }
    __device__ __forceinline__ static void bound(float* x) {}
};

// dx = x + c: the model of the reference's exact-propagation test
// (tvb/tests/library/simulator/history_test.py), used with the Identity scheme.
struct SumModel {
    static constexpr int NSV = 1, NCV = 1, NINT = 1, NOBS = 1, NP = 1, NPX = NP;
    __device__ static constexpr int cvar(int k) { return 0; }
    __device__ __forceinline__ static void prepare(float* p) {}
    __device__ __forceinline__ static void dfun(const float* x, const float* c, const float* p, float* dx) {
        dx[0] = x[0] + c[0];
    }
    __device__ __forceinline__ static float observe(int k, const float* x) { return x[0]; }
    __device__ __forceinline__ static void bound(float* x) {}
};

// ---------------------------------------------------------------- coupling
// Coupling kinds: the gather accumulates sum_j w_ij * pre(x_i, x_j(t - d_ij)),
// post() maps the sums to the model's coupling input.

enum { CF_LINEAR = 0, CF_DIFFERENCE = 1, CF_SIGMOIDAL_JR = 2, CF_GENERIC = 3 };
// CF_GENERIC kernels serve TVBK_CFUN_SIGMOIDAL, _HYPERBOLIC_TANGENT and _KURAMOTO, choosing
// the pre / post forms at run time from the launch's coupling code.

template <int CF>
struct CouplingTraits;

// Linear: pre = x_j, post = a * gx + b (coupling.py:170-200)
template <>
struct CouplingTraits<CF_LINEAR> {
    static constexpr int NOUT_FROM_NCV = 1;  // one output per coupling variable
};
// Difference: pre = x_j - x_i, post = a * gx (coupling.py:462-486)
template <>
struct CouplingTraits<CF_DIFFERENCE> {
    static constexpr int NOUT_FROM_NCV = 1;
};
// SigmoidalJansenRit: pre = cmin + (cmax - cmin) / (1 + exp(r (midpoint - (x_j0 - x_j1)))),
// post = a * gx, one output (coupling.py:370-376)
template <>
struct CouplingTraits<CF_SIGMOIDAL_JR> {
    static constexpr int NOUT_FROM_NCV = 0;
};

}  // namespace tvbk
