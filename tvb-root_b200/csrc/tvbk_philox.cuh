// Counter-based normal variates for the stochastic integrators.
//
// Philox4x32 with 10 rounds (J. K. Salmon, M. A. Moraes, R. O. Dror,
// D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11), written
// from the paper's round function and published multiplier / Weyl constants.
// Uniforms are ((x >> 9) + 0.5) * 2^-23, exact in float32 and never 0 or 1;
// a Box-Muller transform turns each pair into two normals.
//
// Stream layout (mirrored by the CPU oracle): the normal of (step s, region i,
// state variable k) is element (s - 1) & 3 of the 4 normals from
// Philox(key = (seed, stream), counter = ((s - 1) >> 2, i, k, 0)), the pairs
// (x0, x1) and (x2, x3) giving steps 4q+1..4q+2 and 4q+3..4q+4.  Blocks end on
// steps that are multiples of 4, where monitor samples with periods in
// multiples of 4 steps fall (the 4 ms Bold stock, a TR).  The stream is keyed
// by instance, not by batch slot, so a simulation draws the same noise alone
// or batched with others.
#pragma once
#include <cstdint>

namespace tvbk {

struct Philox4 {
    uint32_t x[4];
};

__device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                 uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        // each 32 x 32 -> 64-bit product in one wide multiply (high and low halves together)
        const uint64_t p0 = (uint64_t)M0 * c0, p1 = (uint64_t)M1 * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += W0;
        k1 += W1;
    }
    Philox4 out;
    out.x[0] = c0;
    out.x[1] = c1;
    out.x[2] = c2;
    out.x[3] = c3;
    return out;
}

// (m + 1/2) 2^-23 with m = x >> 9 < 2^23, built from the bits: 1 + m 2^-23 is
// the float with exponent 0 and mantissa m, and subtracting 1 - 2^-24 from
// it is exact (Sterbenz), giving (2m + 1) 2^-24 -- the same value as
// (float(m) + 0.5) * 2^-23, without the integer-to-float conversion.
__device__ __forceinline__ float uniform_open(uint32_t x) {
    return __uint_as_float((x >> 9) | 0x3f800000u) - 0.99999994039535522461f;  // 1 - 2^-24
}

// Box-Muller: r = sqrt(-2 ln u1); (r cos 2 pi u2, r sin 2 pi u2), with the
// hardware approximations of log, sin and cos: the angle is taken as
// pi (2 u2 - 1) in (-pi, pi), where __sinf / __cosf are accurate to about
// 2^-21 absolute, and cos(2 pi u2) = -cos(pi (2 u2 - 1)),
// sin(2 pi u2) = -sin(pi (2 u2 - 1)).  -2 ln u1 > 0 since u1 < 1, so
// r = r2 * rsqrt(r2).  The deviates differ from exactly rounded ones by
// ~1e-6 relative (more only for the rare u1 within ~1e-5 of 1, where r is
// tiny), which the noise does not notice.
__device__ __forceinline__ void box_muller(uint32_t a, uint32_t b, float& z0, float& z1) {
    const float u1 = uniform_open(a);
    const float u2 = uniform_open(b);
    const float r2 = __log2f(u1) * -1.38629436111989061883f;  // -2 ln u1 = log2(u1) * (-2 ln 2)
    const float r = r2 * rsqrtf(r2);
    float s, c;
    __sincosf(fmaf(6.28318530717958647693f, u2, -3.14159265358979323846f), &s, &c);  // pi (2 u2 - 1)
    z0 = -r * c;
    z1 = -r * s;
}

// Block of step s (>= 1): steps 4q+1 .. 4q+4 share block q = (s - 1) >> 2.
__device__ __forceinline__ int64_t philox_block_of(int64_t step) { return (step - 1) >> 2; }
__device__ __forceinline__ int philox_lane_of(int64_t step) { return (int)((step - 1) & 3); }

// The 4 normals of the block of step s for region i, state variable k.
__device__ __forceinline__ void philox_normals4(uint32_t seed, uint32_t stream, int64_t step, int i, int k,
                                                float z[4]) {
    const Philox4 r = philox4x32_10((uint32_t)philox_block_of(step), (uint32_t)i, (uint32_t)k, 0u, seed, stream);
    box_muller(r.x[0], r.x[1], z[0], z[1]);
    box_muller(r.x[2], r.x[3], z[2], z[3]);
}

}  // namespace tvbk
