// Counter-based random streams and the engine's own trigonometry.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).  Keying: key = (seed lo,
// seed hi); counter = (pixel index, view id, phase, block), phase 0 for the
// initial hypotheses and 1 + iteration for that iteration's refinement draws.
// A pixel's draws therefore depend only on (seed, view, pixel, iteration):
// a view solved alone or inside any batch sees the same numbers.
#pragma once
#include <stdint.h>

namespace hp {

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// Uniform in (0,1): (2*(x>>9)+1) * 2^-24, exact in FP32.
__device__ __forceinline__ float u01(uint32_t x) {
    return __uint2float_rn(2u * (x >> 9) + 1u) * 5.9604644775390625e-8f;
}

// sin/cos of 2*pi*u: quadrant reduction, Taylor series (degree 11 / 12) on
// |a| <= pi/4 in Horner form.  Every step is an explicitly rounded intrinsic so
// the host restatement reproduces it bit for bit.
__device__ __forceinline__ void sincos_2pi(float u, float* s_out, float* c_out) {
    float q = rintf(__fmul_rn(u, 4.0f));
    float f = __fsub_rn(u, __fmul_rn(q, 0.25f));
    float a = __fmul_rn(f, 6.28318530717958647692f);
    float a2 = __fmul_rn(a, a);
    float s = __fmaf_rn(a2, -2.50521083854417187751e-8f, 2.75573192239858906526e-6f);
    s = __fmaf_rn(a2, s, -1.98412698412698412698e-4f);
    s = __fmaf_rn(a2, s, 8.33333333333333333333e-3f);
    s = __fmaf_rn(a2, s, -1.66666666666666666667e-1f);
    s = __fmaf_rn(__fmul_rn(a2, a), s, a);
    float c = __fmaf_rn(a2, 2.08767569878680989792e-9f, -2.75573192239858906526e-7f);
    c = __fmaf_rn(a2, c, 2.48015873015873015873e-5f);
    c = __fmaf_rn(a2, c, -1.38888888888888888889e-3f);
    c = __fmaf_rn(a2, c, 4.16666666666666666667e-2f);
    c = __fmaf_rn(a2, c, -0.5f);
    c = __fmaf_rn(a2, c, 1.0f);
    int qi = static_cast<int>(q) & 3;
    float so = qi == 0 ? s : (qi == 1 ? c : (qi == 2 ? -s : -c));
    float co = qi == 0 ? c : (qi == 1 ? -s : (qi == 2 ? -c : s));
    *s_out = so;
    *c_out = co;
}

// Unit viewing ray K^-1 [x, y, 1] / |.|, IEEE-rounded throughout.
__device__ __forceinline__ float3 view_ray(const float* k, int x, int y) {
    const float fx = static_cast<float>(x), fy = static_cast<float>(y);
    float a = __fmaf_rn(k[0], fx, __fmaf_rn(k[1], fy, k[2]));
    float b = __fmaf_rn(k[3], fx, __fmaf_rn(k[4], fy, k[5]));
    float c = __fmaf_rn(k[6], fx, __fmaf_rn(k[7], fy, k[8]));
    float len = __fsqrt_rn(__fmaf_rn(a, a, __fmaf_rn(b, b, __fmul_rn(c, c))));
    if (len > 1e-12f) {
        a = __fdiv_rn(a, len);
        b = __fdiv_rn(b, len);
        c = __fdiv_rn(c, len);
    }
    return make_float3(a, b, c);
}

__device__ __forceinline__ float3 normalize3_rn(float x, float y, float z) {
    float len = __fsqrt_rn(__fmaf_rn(x, x, __fmaf_rn(y, y, __fmul_rn(z, z))));
    if (len > 1e-12f) {
        x = __fdiv_rn(x, len);
        y = __fdiv_rn(y, len);
        z = __fdiv_rn(z, len);
    }
    return make_float3(x, y, z);
}

__device__ __forceinline__ float dot3_rn(float3 a, float3 b) {
    return __fmaf_rn(a.x, b.x, __fmaf_rn(a.y, b.y, __fmul_rn(a.z, b.z)));
}

}  // namespace hp
