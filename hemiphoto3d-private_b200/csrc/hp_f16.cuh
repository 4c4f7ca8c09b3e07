// FP16-storage / FP32-accumulate PatchMatch device code for sm_100a, templated
// on the window (radius R, stride ST), the tile height TH (64 x TH pixels per
// CTA, TH warps) and the staging depth D (quad loads in flight per window
// row).  Every (TH, D) gives the same bits: they change how work is grouped
// and when loads are issued, not what is computed.  Instantiated by
// hp_kernels_f16.cu (TH = 8) and hp_kernels_f16t4.cu (TH = 4).
//
// Same algorithm as the FP32 path (initialisation is shared; cost,
// propagation and refinement follow src/dense_recon/patchmatch_mvs.cu:222-343
// and :519-655), re-derived for throughput:
//  - Sources are FP16 textures (half the texel bytes of FP32); the hardware
//    linear filter returns FP32.
//  - Per (candidate, source) the plane-induced homography is folded into one
//    3x3 H = A + b (K^-T n)^T / (n.P), with the +0.5 texel-centre offset folded
//    into its first two rows; along a window row a tap is w += s*H[:,0]: three
//    adds, one reciprocal and two multiplies instead of ~25 operations.  Each
//    row issues all its texture fetches before consuming them.
//  - If the warped window's four corners lie inside the valid source region
//    (the warp of a rectangle with one-signed depth is the convex quad of its
//    corners) every tap is valid and the per-tap bounds tests are skipped.
//  - The reference window is mean-subtracted per pixel once per visit and kept
//    in shared memory as half2 pairs ([row][thread][pairs], one vector load a
//    row) for windows of up to 64 taps.  Window sums use mean-shifted values
//    (compensated variance): FP16 products and per-row FP16 partial sums,
//    flushed into FP32 accumulators every row.
//  - Windows touching the source border mask invalid taps per the
//    reference's validity rules (|w_z| >= 1e-8, u in [0, W-1), v in [0, H-1),
//    count >= taps/2), vectorised like the fast path.
#pragma once

#include <cuda_fp16.h>

#include "hp_check.cuh"
#include "hp_internal.h"
#include "hp_rng.cuh"
#include "hp_filter.cuh"
#include "hp_tile.cuh"

#ifndef HP_F16_MIN_BLOCKS
#define HP_F16_MIN_BLOCKS 3
#endif

namespace hp {
namespace f16 {
namespace {

#ifdef HP_COUNT_TAPS
// Instrumented builds only (make count): taps sampled, window taps per
// (candidate, source) whose window is not wholly outside the source.
__device__ unsigned long long g_taps;
#endif

// Tile shapes: TILE_W x TH pixels per CTA, TH warps (one per tile row).
template <int TH>
struct Tile {
    static constexpr int NT = 32 * TH;  // threads per CTA
    static constexpr int MIN_BLOCKS = TH == 8 ? HP_F16_MIN_BLOCKS : 2 * HP_F16_MIN_BLOCKS;
};

__device__ __forceinline__ const ViewDesc* locate_tile16(const BatchList& bl, int t, int* tx, int* ty) {
    int lo = 0, hi = bl.n_active - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (bl.tile_prefix[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const ViewDesc* v = &bl.views[bl.active[lo]];
    int local = t - bl.tile_prefix[lo];
    *tx = local % v->tiles_x;
    *ty = local / v->tiles_x;
    return v;
}

template <int NT>
__device__ __forceinline__ void load_ref_tile16(float* s_ref, int tw, int th, const ViewDesc* v, int x0, int y0,
                                                int r) {
    const int W = v->W, H = v->H;
    for (int i = threadIdx.x; i < tw * th; i += NT) {
        int ty = i / tw, tx = i - ty * tw;
        int gx = min(max(x0 - r + tx, 0), W - 1);
        int gy = min(max(y0 - r + ty, 0), H - 1);
        s_ref[i] = __half2float(v->ref16[static_cast<size_t>(gy) * v->ref16_pitch + gx]);
    }
}

template <int R, int ST>
struct Win {
    static constexpr int SIDE = (2 * R) / ST + 1;
    static constexpr int N = SIDE * SIDE;
    static constexpr int PAIRS = (SIDE + 1) / 2;  // half2 per row (the last may be half empty)
    static constexpr int VEC = PAIRS <= 1 ? 1 : (PAIRS <= 2 ? 2 : 4);  // a row's pairs, padded, in one load
    static constexpr bool IN_SMEM = PAIRS <= 4 && SIDE * VEC <= 32;
};
template <int V> struct WinRow;
template <> struct WinRow<1> { using T = unsigned; };
template <> struct WinRow<2> { using T = uint2; };
template <> struct WinRow<4> { using T = uint4; };
constexpr int WIN_PAIRS_MAX = 32;

// Per-pixel window statistics; the mean-subtracted window itself goes to s_win,
// laid out [row][thread][VEC half2]: one row of a pixel's residual pairs is one
// vector load (16 bytes for 7 or 8 taps a row), and the lanes of a warp read
// consecutive vectors.
struct RefStats {
    float mean;  // window mean (the shift of every sum)
    float ssd;   // sum (r - mean)^2
};

template <int R, int ST, int NT>
__device__ __forceinline__ RefStats load_window(__half2* s_win, const float* s_ref, int tw, int lx, int ly) {
    constexpr int SIDE = Win<R, ST>::SIDE;
    float sum = 0.f;
#pragma unroll 1
    for (int i = 0; i < SIDE; ++i)
#pragma unroll
        for (int j = 0; j < SIDE; ++j) sum = __fadd_rn(sum, s_ref[(ly + i * ST) * tw + lx + j * ST]);
    const float mean = __fmul_rn(sum, 1.0f / Win<R, ST>::N);
    float ssd = 0.f;
#pragma unroll 1
    for (int i = 0; i < SIDE; ++i)
#pragma unroll
        for (int j = 0; j < SIDE; ++j) {
            const float d = __fsub_rn(s_ref[(ly + i * ST) * tw + lx + j * ST], mean);
            ssd = __fmaf_rn(d, d, ssd);
        }
    if constexpr (Win<R, ST>::IN_SMEM) {
        constexpr int PAIRS = Win<R, ST>::PAIRS;
#pragma unroll 1
        for (int i = 0; i < SIDE; ++i) {
            constexpr int VEC = Win<R, ST>::VEC;
            unsigned rw[VEC] = {};
#pragma unroll
            for (int p = 0; p < PAIRS; ++p) {
                const float a = __fsub_rn(s_ref[(ly + i * ST) * tw + lx + (2 * p) * ST], mean);
                const float b =
                    (2 * p + 1 < SIDE) ? __fsub_rn(s_ref[(ly + i * ST) * tw + lx + (2 * p + 1) * ST], mean) : 0.f;
                const __half2 h = __floats2half2_rn(a, b);
                memcpy(&rw[p], &h, sizeof h);
            }
            typename WinRow<VEC>::T row;
            memcpy(&row, rw, sizeof row);
            *reinterpret_cast<typename WinRow<VEC>::T*>(s_win + (i * NT + threadIdx.x) * VEC) = row;
        }
    }
    return RefStats{mean, ssd};
}

// Approximate reciprocal (PTX rcp.approx.ftz.f32, ~1 ulp): the warped-coordinate
// divide of the fast path.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Row flush: s + x + y for the FP16 pair (x, y), each add rounded to FP32.
// sm_100's mixed-precision add takes the FP16 operand directly, so the flush
// needs no conversions (two instructions instead of four).
__device__ __forceinline__ float add_pair(float s, __half2 a) {
    asm("add.rn.f32.f16 %0, %1, %0;" : "+f"(s) : "h"(__half_as_ushort(__low2half(a))));
    asm("add.rn.f32.f16 %0, %1, %0;" : "+f"(s) : "h"(__half_as_ushort(__high2half(a))));
    return s;
}

struct Plane {
    float h[9];  // homography with the +0.5 texel offset folded into rows 0, 1
};

// Software bilinear sampler (sources whose bit is set in soft_mask).  The
// texture unit filters about four taps per SM clock; these taps go through the
// load/store pipe and the FP16 units instead, which run alongside it.
//
// A warped coordinate c (texel centres at integers) becomes fixed point with
// 8 fractional bits by one FMA: the bits of RN(c + 49152) are
// 0x47400000 + RN(256 c) for 0 <= c < 16384.  Two byte permutes then give
//  - the quad's element offset: bytes 1 and 2 are the low and high bytes of
//    0x4000 + floor(c); the quad plane is tiled in 256 x 256 blocks so that
//    (x_lo, y_lo, x_hi, y_hi) of the two coordinates, in that byte order, is
//    the offset itself (hpx::QuadPlane), with the 0x40 bias of both high
//    bytes folded into the base pointer, and
//  - the weights as FP16 numbers: 0x47 above the fraction byte is the FP16
//    encoding of 7 + frac/256, exact, so one FP16 subtraction of 7 leaves the
//    8-bit fraction (the texture unit's weight resolution).
// The quad plane stores each 2x2 texel block in difference form, shifted by
// -0.5 (see quads_kernel), so a sample is two FP16 FMAs on values of
// magnitude <= 0.5 (half-ulp <= 2^-13).
constexpr float SOFT_MAGIC = 49152.0f;
constexpr unsigned SOFT_ORIGIN = 0x47400000u;  // bits of SOFT_MAGIC: coordinate 0

__device__ __forceinline__ const uint2* soft_base(const uint2* quad) {
    // quad - (0x40 << 16 | 0x40 << 24) elements, formed on the integer address.
    return reinterpret_cast<const uint2*>(reinterpret_cast<uintptr_t>(quad) -
                                          static_cast<uintptr_t>(0x40400000u) * sizeof(uint2));
}

__device__ __forceinline__ unsigned soft_offset(unsigned bu, unsigned bv) {
    return __byte_perm(bu, bv, 0x6251);  // bu.b1, bv.b1, bu.b2, bv.b2
}

__device__ __forceinline__ __half soft_lerp(uint2 q, unsigned wbits) {
    __half2 w;
    memcpy(&w, &wbits, sizeof w);
    w = __hsub2(w, __float2half2_rn(7.0f));  // (fx, fy), exact
    __half2 a, b;
    memcpy(&a, &q.x, sizeof a);  // (t00 - 0.5, t01 - t00)
    memcpy(&b, &q.y, sizeof b);  // (t10 - t00, dxy)
    const __half2 c = __hfma2(__low2half2(w), b, a);  // (row y0 at fx, column difference at fx)
    return __hfma(__high2half(w), __high2half(c), __low2half(c));
}

// Cost (1 - NCC, or 2 when invalid) of one source.  Sums of e = s - mean and
// products (r - mean) e are formed in FP16 per window row and flushed to FP32.
// CHECK = false assumes every tap is valid (the caller's corner test proved
// it); CHECK = true applies the reference's validity rules per tap
// (|w_z| >= 1e-8, u in [0, W-1), v in [0, H-1), count >= taps/2) by masking
// the tap's terms.  With every tap valid both forms execute the same
// arithmetic on the same values, so the choice (made per warp) never changes
// a result.  SOFT selects the software sampler; P then holds the homography
// without the texture's +0.5 texel-centre offset.
template <int R, int ST, bool CHECK, bool SOFT, int NT, int D>
__device__ __forceinline__ float source_cost(const Plane& P, cudaTextureObject_t tex, const uint2* qbase, RefStats st,
                                             const __half2* s_win, const float* s_ref, int tw, int lx, int ly, int x,
                                             int y, float fW, float fH) {
    constexpr int SIDE = Win<R, ST>::SIDE;
    constexpr int PAIRS = Win<R, ST>::PAIRS;
    constexpr int N = Win<R, ST>::N;
    const float c0 = st.mean;
    // Software taps are interpolated on texels shifted by -0.5, so their
    // residual is s' - (mean - 0.5).  The FP16 rounding of that shift is a
    // constant offset over the window, which the compensated sums cancel.
    const __half2 c0s = __float2half2_rn(__fsub_rn(c0, 0.5f));
    float s1 = 0.f, s2 = 0.f, s3 = 0.f, r1 = 0.f, r2 = 0.f;
    int count = 0;
    const float sx0 = static_cast<float>(x - R), sy0 = static_cast<float>(y - R);
    const float hx0 = __fmul_rn(P.h[0], ST), hx1 = __fmul_rn(P.h[3], ST), hx2 = __fmul_rn(P.h[6], ST);
    const float rx0 = __fmaf_rn(P.h[0], sx0, P.h[2]), rx1 = __fmaf_rn(P.h[3], sx0, P.h[5]);
    const float rx2 = __fmaf_rn(P.h[6], sx0, P.h[8]);
    // Validity bounds of the (offset) coordinate: [lo, W - 1 + lo) with lo = 0.5 for texture taps.
    constexpr float LO = SOFT ? 0.0f : 0.5f;
#pragma unroll 1
    for (int i = 0; i < SIDE; ++i) {
        const float py = __fadd_rn(sy0, static_cast<float>(i * ST));
        // (w_x, w_y) advance as a pair: sm_100's paired FP32 instructions round
        // each element as the scalar ones do, so the bits are the same.
        const float2 wxy0 = __ffma2_rn(make_float2(P.h[1], P.h[4]), make_float2(py, py), make_float2(rx0, rx1));
        float wx = wxy0.x, wy = wxy0.y;
        float wz = __fmaf_rn(P.h[7], py, rx2);
        unsigned ok = (1u << SIDE) - 1u;
        constexpr int VEC = Win<R, ST>::VEC;
        unsigned rw[VEC];
        if constexpr (Win<R, ST>::IN_SMEM) {  // the row's reference residuals, one load
            const auto row = *reinterpret_cast<const typename WinRow<VEC>::T*>(s_win + i * NT * VEC);
            memcpy(rw, &row, sizeof row);
        }
        __half2 a1, a2, a3, a4, a5;  // set by the row's first pair
        // Folds the residual pair of taps (2p, 2p + 1) into the row sums.
        auto accumulate = [&](int p, __half2 e) {
            __half2 rq;
            if constexpr (Win<R, ST>::IN_SMEM) {
                memcpy(&rq, &rw[p], sizeof rq);
            } else {
                const float* row = s_ref + (ly + i * ST) * tw + lx;
                const float ra = __fsub_rn(row[(2 * p) * ST], c0);
                const float rb = (2 * p + 1 < SIDE) ? __fsub_rn(row[(2 * p + 1) * ST], c0) : 0.f;
                rq = __floats2half2_rn(ra, rb);
            }
            if constexpr (CHECK) {
                const bool va = (ok >> (2 * p)) & 1u;
                const bool vb = (2 * p + 1 < SIDE) && ((ok >> (2 * p + 1)) & 1u);
                // Bitwise masks (exact; a multiply by 1 would not preserve FP16 subnormals).
                const unsigned m = (va ? 0x0000ffffu : 0u) | (vb ? 0xffff0000u : 0u);
                unsigned bits;
                memcpy(&bits, &rq, sizeof bits);
                bits &= m;
                memcpy(&rq, &bits, sizeof bits);
                memcpy(&bits, &e, sizeof bits);
                bits &= m;
                memcpy(&e, &bits, sizeof bits);
            }
            if (p == 0) {
                a1 = e;
                a2 = __hmul2(e, e);
                a3 = __hmul2(rq, e);
                if constexpr (CHECK) {
                    a4 = rq;
                    a5 = __hmul2(rq, rq);
                }
            } else {
                a1 = __hadd2(a1, e);
                a2 = __hfma2(e, e, a2);
                a3 = __hfma2(rq, e, a3);
                if constexpr (CHECK) {
                    a4 = __hadd2(a4, rq);
                    a5 = __hfma2(rq, rq, a5);
                }
            }
        };
        if constexpr (SOFT) {
            // Chunks of D taps (the staging depth): D quad loads in flight, then D / 2 pairs folded.
            constexpr int CHUNKS = (SIDE + D - 1) / D;
#pragma unroll
            for (int ch = 0; ch < CHUNKS; ++ch) {
                uint2 q[D];
                unsigned wb[D];
#pragma unroll
                for (int jj = 0; jj < D; ++jj) {
                    const int j = D * ch + jj;
                    if (j >= SIDE) break;
                    const float iz = rcp_approx(wz);
                    const float2 wxy = make_float2(wx, wy), izz = make_float2(iz, iz);
                    const float2 fxy = __ffma2_rn(wxy, izz, make_float2(SOFT_MAGIC, SOFT_MAGIC));
                    unsigned bu = __float_as_uint(fxy.x);
                    unsigned bv = __float_as_uint(fxy.y);
                    if constexpr (CHECK) {
                        const float2 uv = __fmul2_rn(wxy, izz);
                        const float u = uv.x, v = uv.y;
                        const bool skip = fabsf(wz) < 1e-8f || !(u >= LO) || !(u < fW - 1.0f + LO) || !(v >= LO) ||
                                          !(v < fH - 1.0f + LO);
                        ok &= ~(static_cast<unsigned>(skip) << j);
                        bu = skip ? SOFT_ORIGIN : bu;  // an in-bounds quad; the tap is masked
                        bv = skip ? SOFT_ORIGIN : bv;
                    }
#ifdef HP_SELF_CHECK
                    {
                        const int xi = static_cast<int>(bu - SOFT_ORIGIN) >> 8;
                        const int yi = static_cast<int>(bv - SOFT_ORIGIN) >> 8;
                        if (!HP_CHECK(xi >= 0 && xi < static_cast<int>(fW) && yi >= 0 && yi < static_cast<int>(fH),
                                      HP_CHECK_QUAD, x, y, xi, yi, CHECK ? 1 : 0, i * SIDE + j, wx, wy, wz, 0.f)) {
                            bu = SOFT_ORIGIN;
                            bv = SOFT_ORIGIN;
                        }
                    }
#endif
                    wb[jj] = __byte_perm(bu, bv, 0x7430);
                    q[jj] = __ldg(qbase + soft_offset(bu, bv));
                    const float2 next = __fadd2_rn(wxy, make_float2(hx0, hx1));
                    wx = next.x;
                    wy = next.y;
                    wz = __fadd_rn(wz, hx2);
                }
#pragma unroll
                for (int pp = 0; pp < D / 2; ++pp) {
                    const int p = (D / 2) * ch + pp;
                    if (p >= PAIRS) break;
                    const __half sa = soft_lerp(q[2 * pp], wb[2 * pp]);
                    const __half sb = (2 * p + 1 < SIDE) ? soft_lerp(q[2 * pp + 1], wb[2 * pp + 1]) : __low2half(c0s);
                    accumulate(p, __hsub2(__halves2half2(sa, sb), c0s));
                }
            }
        } else {
            float smp[2 * PAIRS];
#pragma unroll
            for (int j = 0; j < SIDE; ++j) {
                const float iz = rcp_approx(wz);
                const float u = __fmul_rn(wx, iz), v = __fmul_rn(wy, iz);  // texel-centre offset already folded in
                if constexpr (CHECK) {
                    const bool skip = fabsf(wz) < 1e-8f || !(u >= LO) || !(u < fW - 1.0f + LO) || !(v >= LO) ||
                                      !(v < fH - 1.0f + LO);
                    ok &= ~(static_cast<unsigned>(skip) << j);
                }
                smp[j] = tex2D<float>(tex, u, v);
                wx = __fadd_rn(wx, hx0);
                wy = __fadd_rn(wy, hx1);
                wz = __fadd_rn(wz, hx2);
            }
            if constexpr (SIDE & 1) smp[SIDE] = c0;  // pads the last pair: e = 0
#pragma unroll
            for (int p = 0; p < PAIRS; ++p) {
                // The shift is subtracted in FP32 and only the small residual is
                // rounded to FP16 (rounding the sample first would cost ~2.4e-4).
                accumulate(p, __floats2half2_rn(__fsub_rn(smp[2 * p], c0), __fsub_rn(smp[2 * p + 1], c0)));
            }
        }
        s1 = add_pair(s1, a1);
        s2 = add_pair(s2, a2);
        s3 = add_pair(s3, a3);
        if constexpr (CHECK) {
            r1 = add_pair(r1, a4);
            r2 = add_pair(r2, a5);
            count += __popc(ok);
        }
    }
    float n = static_cast<float>(N), dr, num;
    if (!CHECK || count == N) {
        // n*sum(r^2)-sum(r)^2 = n*ssd and the covariance numerator is n*s3 (sum(r - mean) = 0).
        dr = __fmul_rn(n, st.ssd);
        num = __fmul_rn(n, s3);
    } else {
        if (count < N / 2) return 2.0f;
        n = static_cast<float>(count);
        dr = __fmaf_rn(n, r2, -__fmul_rn(r1, r1));
        num = __fmaf_rn(n, s3, -__fmul_rn(r1, s1));
    }
    const float ds = __fmaf_rn(n, s2, -__fmul_rn(s1, s1));
    if (dr < 1e-6f || ds < 1e-6f) return 2.0f;
    const float ncc = fmaxf(-1.0f, fminf(1.0f, __fmul_rn(__fmul_rn(num, rsqrtf(dr)), rsqrtf(ds))));
    return __fsub_rn(1.0f, ncc);
}

template <int R, int ST, int NT, int D>
__device__ __forceinline__ float cost_f16(RefStats st, const __half2* s_win, const float* s_ref, int tw, int lx,
                                          int ly, int x, int y, float d, float cnx, float cny, float cnz,
                                          const ViewDesc* __restrict__ v, int topk, unsigned soft_mask) {
    const float* k = v->kinv;
    const float fx = static_cast<float>(x), fy = static_cast<float>(y);
    const float Px = __fmul_rn(d, __fmaf_rn(k[0], fx, __fmaf_rn(k[1], fy, k[2])));
    const float Py = __fmul_rn(d, __fmaf_rn(k[3], fx, __fmaf_rn(k[4], fy, k[5])));
    const float Pz = __fmul_rn(d, __fmaf_rn(k[6], fx, __fmaf_rn(k[7], fy, k[8])));
    const float ndp = __fmaf_rn(cnx, Px, __fmaf_rn(cny, Py, __fmul_rn(cnz, Pz)));
    if (fabsf(ndp) < 1e-8f) return 2.0f;
    const float ind = __frcp_rn(ndp);
    const float m0 = __fmul_rn(__fmaf_rn(k[0], cnx, __fmaf_rn(k[3], cny, __fmul_rn(k[6], cnz))), ind);
    const float m1 = __fmul_rn(__fmaf_rn(k[1], cnx, __fmaf_rn(k[4], cny, __fmul_rn(k[7], cnz))), ind);
    const float m2 = __fmul_rn(__fmaf_rn(k[2], cnx, __fmaf_rn(k[5], cny, __fmul_rn(k[8], cnz))), ind);
    const float fW = static_cast<float>(v->W), fH = static_cast<float>(v->H);
    const float xa = static_cast<float>(x - R);
    const float ya = static_cast<float>(y - R);
    float top0 = 2.0f, top1 = 2.0f, top2 = 2.0f;
    const int S = v->S;
    for (int s = 0; s < S; ++s) {
        // A (9) and b (3) of the source: three 16-byte loads (ViewDesc::ab is 16-byte aligned).
        const float4* A4 = reinterpret_cast<const float4*>(v->ab[s]);
        const float4 q0 = __ldg(A4), q1 = __ldg(A4 + 1), q2 = __ldg(A4 + 2);
        const float A[12] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w};
        // Uniform over the launch: every lane of a warp takes the same sampler.
        const bool soft = (soft_mask >> s) & 1u;
        const float lo = soft ? 0.0f : 0.5f;  // texel-centre offset of the sampler's coordinate
        Plane P;
        P.h[6] = __fmaf_rn(A[11], m0, A[6]);
        P.h[7] = __fmaf_rn(A[11], m1, A[7]);
        P.h[8] = __fmaf_rn(A[11], m2, A[8]);
        P.h[0] = __fmaf_rn(A[9], m0, A[0]);
        P.h[1] = __fmaf_rn(A[9], m1, A[1]);
        P.h[2] = __fmaf_rn(A[9], m2, A[2]);
        P.h[3] = __fmaf_rn(A[10], m0, A[3]);
        P.h[4] = __fmaf_rn(A[10], m1, A[4]);
        P.h[5] = __fmaf_rn(A[10], m2, A[5]);
        if (!soft) {  // texture taps: fold the +0.5 texel-centre offset into rows 0 and 1
            P.h[0] = __fmaf_rn(0.5f, P.h[6], P.h[0]);
            P.h[1] = __fmaf_rn(0.5f, P.h[7], P.h[1]);
            P.h[2] = __fmaf_rn(0.5f, P.h[8], P.h[2]);
            P.h[3] = __fmaf_rn(0.5f, P.h[6], P.h[3]);
            P.h[4] = __fmaf_rn(0.5f, P.h[7], P.h[4]);
            P.h[5] = __fmaf_rn(0.5f, P.h[8], P.h[5]);
        }
        // Corner test: in front of the source (w_z > 1e-6) with all four
        // corners inside [lo, W - 1 + lo) x [lo, H - 1 + lo) by a 0.05 px
        // margin, which covers the rounding of the row-stepped taps and of the
        // corners themselves (stepped here from the first along the window's
        // edges) where the homography is well conditioned (below).  The warp
        // of the window rectangle is then the convex quad of its corners, so
        // every tap is valid by the per-tap rules too.
        const float ulo = __fadd_rn(lo, 0.05f), uhi = __fsub_rn(__fadd_rn(fW, lo), 1.05f);
        const float vhi = __fsub_rn(__fadd_rn(fH, lo), 1.05f);
        constexpr float SPAN = static_cast<float>((Win<R, ST>::SIDE - 1) * ST);
        float cz[4], cx[4], cy[4];
        cz[0] = __fmaf_rn(P.h[6], xa, __fmaf_rn(P.h[7], ya, P.h[8]));
        cx[0] = __fmaf_rn(P.h[0], xa, __fmaf_rn(P.h[1], ya, P.h[2]));
        cy[0] = __fmaf_rn(P.h[3], xa, __fmaf_rn(P.h[4], ya, P.h[5]));
        cz[1] = __fmaf_rn(P.h[6], SPAN, cz[0]);
        cx[1] = __fmaf_rn(P.h[0], SPAN, cx[0]);
        cy[1] = __fmaf_rn(P.h[3], SPAN, cy[0]);
        cz[2] = __fmaf_rn(P.h[7], SPAN, cz[0]);
        cx[2] = __fmaf_rn(P.h[1], SPAN, cx[0]);
        cy[2] = __fmaf_rn(P.h[4], SPAN, cy[0]);
        cz[3] = __fmaf_rn(P.h[7], SPAN, cz[1]);
        cx[3] = __fmaf_rn(P.h[1], SPAN, cx[1]);
        cy[3] = __fmaf_rn(P.h[4], SPAN, cy[1]);
        // Fully outside: in front at every corner and every corner beyond the
        // same edge of the valid region by the margin.  The window's warp is
        // the convex quad of its corners, so every tap is invalid, the count
        // is 0 and the reference's rule makes the source cost 2 - no tap needs
        // sampling.
        const float olo = __fsub_rn(lo, 0.05f), ohi = __fadd_rn(__fadd_rn(fW, lo), -0.95f);
        const float ovhi = __fadd_rn(__fadd_rn(fH, lo), -0.95f);
        // Each corner is projected (approximate reciprocal, error far below the
        // margin) and the tests run on the corners' bounding box: ~45
        // instructions for the four corners instead of ~90 for per-corner
        // products and compares.  A corner behind the camera fails `front`,
        // and its garbage coordinates then decide nothing.
        float umin = 0.f, umax = 0.f, vmin = 0.f, vmax = 0.f, zmin = 0.f;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float iz = rcp_approx(cz[c]);
            const float2 uv = __fmul2_rn(make_float2(cx[c], cy[c]), make_float2(iz, iz));
            if (c == 0) {
                umin = umax = uv.x;
                vmin = vmax = uv.y;
                zmin = cz[c];
            } else {
                umin = fminf(umin, uv.x);
                umax = fmaxf(umax, uv.x);
                vmin = fminf(vmin, uv.y);
                vmax = fmaxf(vmax, uv.y);
                zmin = fminf(zmin, cz[c]);
            }
        }
        // Conditioning.  The corners above and the row-stepped taps of
        // source_cost evaluate the homography in different orders, so their
        // rounding differs: by at most (SIDE + 5) roundings of the largest
        // partial sum, Mx = |h0| X1 + |h1| Y1 + |h2| for w_x (X1, Y1 bound the
        // window's absolute pixel coordinates), likewise My and Mz.  In the
        // projected coordinate that is (Mx + |u| Mz) (SIDE + 5) 2^-24 / z_min.
        // A plane seen nearly edge-on makes the terms large and cancelling,
        // and the corners can then pass the test while a tap falls outside
        // the source.  The decision stands only while the bound (with |u|
        // taken as at least 1, which also bounds the error of z) stays within
        // 0.04 px of the 0.05 px margin; other windows take the per-tap
        // checked form, which gives the same bits whenever every tap is valid.
        // NaN or infinite corners fail the comparison too.  COND counts one
        // rounding more than the bound above, for slack.
        constexpr float COND = 0.04f / ((Win<R, ST>::SIDE + 6) * 5.9604645e-8f);
        const float X1 = fabsf(xa) + SPAN, Y1 = fabsf(ya) + SPAN;
        const float Mx = __fmaf_rn(fabsf(P.h[0]), X1, __fmaf_rn(fabsf(P.h[1]), Y1, fabsf(P.h[2])));
        const float My = __fmaf_rn(fabsf(P.h[3]), X1, __fmaf_rn(fabsf(P.h[4]), Y1, fabsf(P.h[5])));
        const float Mz = __fmaf_rn(fabsf(P.h[6]), X1, __fmaf_rn(fabsf(P.h[7]), Y1, fabsf(P.h[8])));
        const float Ua = fmaxf(1.0f, fmaxf(fabsf(umin), fabsf(umax)));
        const float Va = fmaxf(1.0f, fmaxf(fabsf(vmin), fabsf(vmax)));
        const float zc = __fmul_rn(zmin, COND);
        const bool front = zmin > 1e-6f && __fmaf_rn(Ua, Mz, Mx) <= zc && __fmaf_rn(Va, Mz, My) <= zc;
        // SOFT_MASK_CHECKED (self-checking builds only, uniform over the
        // launch) turns both shortcuts off, to test that they change no result.
#ifdef HP_SELF_CHECK
        const bool shortcuts = (soft_mask & SOFT_MASK_CHECKED) == 0u;
#else
        constexpr bool shortcuts = true;
#endif
        const bool inside = front && umin >= ulo && umax < uhi && vmin >= ulo && vmax < vhi;
        const bool left = umax < olo, right = umin >= ohi, top = vmax < olo, bottom = vmin >= ovhi;
        const bool outside = shortcuts && front && (left || right || top || bottom);
        // One form per warp for the lanes that sample: the checked form gives
        // the unchecked form's bits whenever every tap is valid, so lanes that
        // are inside lose nothing.
        const bool all_inside = shortcuts && __all_sync(__activemask(), inside || outside);
        float c = 2.0f;
        if (outside) {
        } else if (soft) {
#ifdef HP_COUNT_TAPS
            atomicAdd(&g_taps, static_cast<unsigned long long>(Win<R, ST>::N));
#endif
            const uint2* qb = soft_base(v->src_quad[s]);
            c = all_inside ? source_cost<R, ST, false, true, NT, D>(P, 0, qb, st, s_win, s_ref, tw, lx, ly, x,
                                                             y, fW, fH)
                           : source_cost<R, ST, true, true, NT, D>(P, 0, qb, st, s_win, s_ref, tw, lx, ly, x,
                                                            y, fW, fH);
        } else {
#ifdef HP_COUNT_TAPS
            atomicAdd(&g_taps, static_cast<unsigned long long>(Win<R, ST>::N));
#endif
            const cudaTextureObject_t tex = v->src_tex16[s];
            c = all_inside ? source_cost<R, ST, false, false, NT, D>(P, tex, nullptr, st, s_win, s_ref, tw, lx, ly, x, y,
                                                              fW, fH)
                           : source_cost<R, ST, true, false, NT, D>(P, tex, nullptr, st, s_win, s_ref, tw, lx, ly, x, y,
                                                             fW, fH);
        }
        if (c < top2) {
            top2 = c;
            if (top2 < top1) {
                float t = top1; top1 = top2; top2 = t;
                if (top1 < top0) { t = top0; top0 = top1; top1 = t; }
            }
        }
    }
    const int kk = min(topk, S);
    float sum = top0;
    if (kk > 1) sum = __fadd_rn(sum, top1);
    if (kk > 2) sum = __fadd_rn(sum, top2);
    return __fdiv_rn(sum, static_cast<float>(kk));
}

__device__ __forceinline__ bool same_plane16(float4 a, float4 b) {
    return __float_as_uint(a.x) == __float_as_uint(b.x) && __float_as_uint(a.y) == __float_as_uint(b.y) &&
           __float_as_uint(a.z) == __float_as_uint(b.z) && __float_as_uint(a.w) == __float_as_uint(b.w);
}

template <int R, int ST, int TH, int D>
__device__ __forceinline__ void tile_cost16(const ViewDesc* v, int tile_x, int tile_y, const SolveConsts& sc,
                                            float* s_ref, __half2* s_win) {
    constexpr int NT = Tile<TH>::NT;
    constexpr int tw = TILE_W + 2 * R, th = TH + 2 * R;
    const int x0 = tile_x * TILE_W, y0 = tile_y * TH;
    load_ref_tile16<NT>(s_ref, tw, th, v, x0, y0, R);
    __syncthreads();
    const int ly = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = y0 + ly;
    if (y >= v->H) return;
    for (int j = 0; j < 2; ++j) {
        const int lx = 2 * lane + j, x = x0 + lx;
        if (x >= v->W) continue;
        const RefStats st = load_window<R, ST, NT>(s_win, s_ref, tw, lx, ly);
        const size_t idx = static_cast<size_t>(y) * v->W + x;
        const float4 h = v->hyp[idx];
        v->cost[idx] = cost_f16<R, ST, NT, D>(st, s_win + threadIdx.x * Win<R, ST>::VEC, s_ref, tw, lx, ly, x, y, h.x, h.y, h.z, h.w, v,
                                       sc.top_k, sc.soft_mask);
    }
}

template <int R, int ST, int TH, int D>
__global__ void __launch_bounds__(Tile<TH>::NT, Tile<TH>::MIN_BLOCKS) cost16_kernel(BatchList bl, SolveConsts sc) {
    __shared__ float s_ref[(TILE_W + 2 * R) * (TH + 2 * R)];
    __shared__ __align__(16) __half2 s_win[Win<R, ST>::IN_SMEM ? WIN_PAIRS_MAX * Tile<TH>::NT : 1];
    int tile_x, tile_y;
    const ViewDesc* v = locate_tile16(bl, blockIdx.x, &tile_x, &tile_y);
    tile_cost16<R, ST, TH, D>(v, tile_x, tile_y, sc, s_ref, s_win);
}

// One red-black half-pass.  The neighbour phase is compacted across the CTA:
// every lane lists the neighbour planes its pixel must score (duplicates of
// the current plane or of an earlier neighbour skipped), the lists of all
// eight warps are concatenated in shared memory, and the warps score the
// union 32 items at a time (warp w takes items [32 (w + 8 k), 32 (w + 8 k) +
// 32)).  An item reads its owner pixel's window statistics and s_win column
// from shared memory and leaves its cost in the owner's slot, so owners then
// fold the costs in L, R, U, D order exactly as if they had scored them
// themselves: results do not depend on which lane scored what.
// Shared memory of the half-pass beyond the reference tile and window (TH warps).
template <int TH>
struct PassSmem {
    float cost[TH][32 * 4];           // neighbour cost, slot (lane << 2 | cand) of the owner's warp
    unsigned short items[TH * 128];   // CTA item list: warp << 7 | lane << 2 | cand
    float2 stat[32 * TH];             // (mean, ssd) of each thread's pixel window
    int warp_total[TH];
};

template <int R, int ST, int TH, int D>
__device__ __forceinline__ void tile_propagate16(const ViewDesc* v, int tile_x, int tile_y, const SolveConsts& sc,
                                                 int iteration, int color, float* s_ref, __half2* s_win,
                                                 PassSmem<TH>& sm) {
    constexpr int NT = Tile<TH>::NT, WARPS = TH;
    constexpr int tw = TILE_W + 2 * R, th = TH + 2 * R;
    const int x0 = tile_x * TILE_W, y0 = tile_y * TH;
    load_ref_tile16<NT>(s_ref, tw, th, v, x0, y0, R);
    __syncthreads();
    const int W = v->W, H = v->H;
    const int ly = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = y0 + ly;
    const int parity = (y + color) & 1;
    const int lx = 2 * lane + parity;
    const int x = x0 + lx;
    const bool active = y < H && x < W;  // every thread takes part in the CTA barriers below
    const size_t idx = static_cast<size_t>(y) * W + x;
    const float dmin = v->dmin, dmax = v->dmax;
    RefStats st{0.f, 0.f};
    float4 best = make_float4(0.f, 0.f, 0.f, 0.f);
    float best_cost = 0.f;
    unsigned need = 0;
    if (active) {
        st = load_window<R, ST, NT>(s_win, s_ref, tw, lx, ly);
        best = v->hyp[idx];
        best_cost = v->cost[idx];
#pragma unroll
        for (int cand = 0; cand < 4; ++cand) {
            const int nxp = x + (cand == 0 ? -1 : (cand == 1 ? 1 : 0));
            const int nyp = y + (cand == 2 ? -1 : (cand == 3 ? 1 : 0));
            if (nxp < 0 || nxp >= W || nyp < 0 || nyp >= H) continue;
            const float4 h = v->hyp[static_cast<size_t>(nyp) * W + nxp];
            if (h.x < dmin || h.x > dmax) continue;
            bool dup = same_plane16(h, best);
            for (int j = 0; j < cand && !dup; ++j) {
                if (need & (1u << j)) {
                    const int jx = x + (j == 0 ? -1 : (j == 1 ? 1 : 0));
                    const int jy = y + (j == 2 ? -1 : (j == 3 ? 1 : 0));
                    dup = same_plane16(h, v->hyp[static_cast<size_t>(jy) * W + jx]);
                }
            }
            if (!dup) need |= 1u << cand;
        }
    }
    sm.stat[threadIdx.x] = make_float2(st.mean, st.ssd);
    const int cnt = __popc(need);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) sm.warp_total[ly] = incl;
    __syncthreads();  // warp totals, window statistics and s_win columns are complete
    int offset = 0, total = 0;
#pragma unroll
    for (int w = 0; w < WARPS; ++w) {
        const int t = sm.warp_total[w];
        offset += w < ly ? t : 0;
        total += t;
    }
    {
        int k = offset + incl - cnt;
        for (int cand = 0; cand < 4; ++cand)
            if (need & (1u << cand)) sm.items[k++] = static_cast<unsigned short>((ly << 7) | (lane << 2) | cand);
    }
    __syncthreads();  // the CTA's item list is complete
    for (int base = ly * 32; base < total; base += NT) {
        const int w = base + lane;
        if (w < total) {
            const int item = sm.items[w];
            const int oly = item >> 7, owner = (item >> 2) & 31, cand = item & 3;
            const int oy = y0 + oly, olx = 2 * owner + ((oy + color) & 1), ox = x0 + olx;
            const float2 os = sm.stat[oly * 32 + owner];
            const int nxp = ox + (cand == 0 ? -1 : (cand == 1 ? 1 : 0));
            const int nyp = oy + (cand == 2 ? -1 : (cand == 3 ? 1 : 0));
            if (!HP_CHECK(nxp >= 0 && nxp < W && nyp >= 0 && nyp < H, HP_CHECK_NEIGHBOUR, ox, oy, nxp, nyp, W, H,
                          0.f, 0.f, 0.f, 0.f))
                continue;
            const float4 h = v->hyp[static_cast<size_t>(nyp) * W + nxp];
            sm.cost[oly][item & 127] = cost_f16<R, ST, NT, D>(RefStats{os.x, os.y}, s_win + (oly * 32 + owner) * Win<R, ST>::VEC, s_ref, tw,
                                                       olx, oly, ox, oy, h.x, h.y, h.z, h.w, v, sc.top_k,
                                                       sc.soft_mask);
        }
    }
    __syncthreads();  // every neighbour cost is in its owner's slot
    if (!active) return;
#pragma unroll
    for (int cand = 0; cand < 4; ++cand) {
        if (need & (1u << cand)) {
            const float c = sm.cost[ly][(lane << 2) | cand];
            if (c < best_cost) {
                const int nxp = x + (cand == 0 ? -1 : (cand == 1 ? 1 : 0));
                const int nyp = y + (cand == 2 ? -1 : (cand == 3 ? 1 : 0));
                best_cost = c;
                best = v->hyp[static_cast<size_t>(nyp) * W + nxp];
            }
        }
    }
    const float3 ray = view_ray(v->kinv, x, y);
    float drange = __fmul_rn(__fsub_rn(dmax, dmin), 0.5f);
    float nrange = 1.0f;
    for (int i = 0; i < iteration; ++i) {
        drange = __fmul_rn(drange, sc.iter_decay);
        nrange = __fmul_rn(nrange, sc.iter_decay);
    }
    for (int step = 0; step < sc.refine_steps; ++step) {
        const uint4 rr = philox4x32_10(make_uint4(static_cast<uint32_t>(idx), v->view_id,
                                                  1u + static_cast<uint32_t>(iteration), static_cast<uint32_t>(step)),
                                       v->seed_lo, v->seed_hi);
        float cd = __fmaf_rn(__fmaf_rn(u01(rr.x), 2.0f, -1.0f), drange, best.x);
        cd = fmaxf(dmin, fminf(dmax, cd));
        const float cx = __fmaf_rn(__fmaf_rn(u01(rr.y), 2.0f, -1.0f), nrange, best.y);
        const float cy = __fmaf_rn(__fmaf_rn(u01(rr.z), 2.0f, -1.0f), nrange, best.z);
        const float cz = __fmaf_rn(__fmaf_rn(u01(rr.w), 2.0f, -1.0f), nrange, best.w);
        float3 cn = normalize3_rn(cx, cy, cz);
        if (dot3_rn(cn, ray) > 0.0f) cn = make_float3(-cn.x, -cn.y, -cn.z);
        const float c = cost_f16<R, ST, NT, D>(st, s_win + threadIdx.x * Win<R, ST>::VEC, s_ref, tw, lx, ly, x, y, cd, cn.x, cn.y, cn.z, v,
                                        sc.top_k, sc.soft_mask);
        if (c < best_cost) {
            best_cost = c;
            best = make_float4(cd, cn.x, cn.y, cn.z);
        }
        drange = __fmul_rn(drange, sc.step_decay);
        nrange = __fmul_rn(nrange, sc.step_decay);
    }
    v->hyp[idx] = best;
    v->cost[idx] = best_cost;
}

template <int R, int ST, int TH, int D>
__global__ void __launch_bounds__(Tile<TH>::NT, Tile<TH>::MIN_BLOCKS) propagate16_kernel(BatchList bl, SolveConsts sc,
                                                                                       int iteration, int color) {
    __shared__ float s_ref[(TILE_W + 2 * R) * (TH + 2 * R)];
    __shared__ __align__(16) __half2 s_win[Win<R, ST>::IN_SMEM ? WIN_PAIRS_MAX * Tile<TH>::NT : 1];
    __shared__ PassSmem<TH> sm;
    int tile_x, tile_y;
    const ViewDesc* v = locate_tile16(bl, blockIdx.x, &tile_x, &tile_y);
    tile_propagate16<R, ST, TH, D>(v, tile_x, tile_y, sc, iteration, color, s_ref, s_win, sm);
}

// Persistent form (see Schedule and the FP32 persistent kernel): the stage
// bodies are those of the per-stage kernels, so the results are bit-identical.
template <int R, int ST, int TH, int D>
__global__ void __launch_bounds__(Tile<TH>::NT, Tile<TH>::MIN_BLOCKS) persistent16_kernel(Schedule s) {
    __shared__ float s_ref[(TILE_W + 2 * R) * (TH + 2 * R)];
    __shared__ __align__(16) __half2 s_win[Win<R, ST>::IN_SMEM ? WIN_PAIRS_MAX * Tile<TH>::NT : 1];
    __shared__ PassSmem<TH> sm;
    // The claimed tile lives in shared memory: thread 0 decodes it once and
    // publishes it after the stage, so no thread carries it through the body.
    __shared__ SchedTile s_tile;
    __shared__ int s_ok;
    for (;;) {
        if (threadIdx.x == 0) s_ok = sched_claim(s, &s_tile);
        __syncthreads();
        if (!s_ok) break;
        // Rebuilt from the kernel parameter rather than read back from shared
        // memory, so the compiler knows it addresses global memory (a pointer
        // loaded from shared memory is generic: the FP32 kernel ran 22% slower).
        const ViewDesc* v = &s.views[s_tile.view];
        const int stage = s_tile.stage, tx = s_tile.tx, ty = s_tile.ty;
#ifdef HP_SELF_CHECK
        const bool state_ok = HP_CHECK(v->hyp && v->cost && v->done && v->W > 0 && v->H > 0, HP_CHECK_STATE, v->W,
                                       v->H, stage, s_tile.tile, s_tile.view, 0, 0.f, 0.f, 0.f, 0.f);
        const bool ticket_ok =
            HP_CHECK(s_tile.tile >= 0 && s_tile.tile < v->tiles_x * v->tiles_y && stage >= 0 &&
                         stage <= 2 * v->iterations + 1 + (v->filter ? 1 : 0),
                     HP_CHECK_TICKET, s_tile.view, stage, s_tile.tile, v->tiles_x * v->tiles_y, v->iterations, 0, 0.f,
                     0.f, 0.f, 0.f);
        if (!state_ok || !ticket_ok) {
            __syncthreads();
            if (threadIdx.x == 0) sched_publish(s, s_tile);
            continue;
        }
#endif
        if (stage == 0) {
            tile_init(v, tx, ty);
            __syncthreads();
            tile_cost16<R, ST, TH, D>(v, tx, ty, s.sc, s_ref, s_win);
        } else if (stage <= 2 * v->iterations) {
            const int k = stage - 1;
            tile_propagate16<R, ST, TH, D>(v, tx, ty, s.sc, k >> 1, k & 1, s_ref, s_win, sm);
        } else if (is_filter_stage(v, stage)) {
            tile_filter(s.views, v, tx, ty, true);  // geometric check, then the maps
        } else {
            tile_unpack(v, tx, ty);
        }
        __syncthreads();
        if (threadIdx.x == 0) sched_publish(s, s_tile);
    }
}


// Launch (or occupancy query) of one tile height, dispatched on (radius,
// stride, staging depth).  mode 0: full-map cost, 1: red-black half-pass,
// 2: persistent (occ non-null: occupancy query only).
template <int TH>
struct Dispatch {
    template <int R, int ST, int D>
    static cudaError_t run(int mode, const BatchList* bl, const SolveConsts& sc, int iteration, int color,
                           const Schedule* s, int grid, cudaStream_t st, int* occ) {
        constexpr int NT = Tile<TH>::NT;
        if (mode == 2) {
            if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, persistent16_kernel<R, ST, TH, D>, NT, 0);
            persistent16_kernel<R, ST, TH, D><<<grid, NT, 0, st>>>(*s);
        } else if (mode == 0) {
            cost16_kernel<R, ST, TH, D><<<bl->total_tiles, NT, 0, st>>>(*bl, sc);
        } else {
            propagate16_kernel<R, ST, TH, D><<<bl->total_tiles, NT, 0, st>>>(*bl, sc, iteration, color);
        }
        return cudaGetLastError();
    }
    template <int R, int ST>
    static cudaError_t depth(int mode, int staging, const BatchList* bl, const SolveConsts& sc, int iteration,
                             int color, const Schedule* s, int grid, cudaStream_t st, int* occ) {
        if (staging == 8) return run<R, ST, 8>(mode, bl, sc, iteration, color, s, grid, st, occ);
        if (staging == 4) return run<R, ST, 4>(mode, bl, sc, iteration, color, s, grid, st, occ);
        return cudaErrorInvalidValue;
    }
    static cudaError_t go(int mode, int radius, int stride, int staging, const BatchList* bl, const SolveConsts& sc,
                          int iteration, int color, const Schedule* s, int grid, cudaStream_t st, int* occ) {
        if (stride != 1 && stride != 2) return cudaErrorInvalidValue;
#define HP_CASE(RR)                                                                                     \
    case RR:                                                                                            \
        return stride == 1 ? depth<RR, 1>(mode, staging, bl, sc, iteration, color, s, grid, st, occ)   \
                           : depth<RR, 2>(mode, staging, bl, sc, iteration, color, s, grid, st, occ);
        switch (radius) {
            HP_CASE(1)
            HP_CASE(2)
            HP_CASE(3)
            HP_CASE(4)
            HP_CASE(5)
            HP_CASE(6)
            HP_CASE(7)
            default: return cudaErrorInvalidValue;
        }
#undef HP_CASE
    }
};

#ifdef HP_COUNT_TAPS
unsigned long long taps_read_reset() {
    unsigned long long v = 0, z = 0;
    cudaDeviceSynchronize();
    cudaMemcpyFromSymbol(&v, g_taps, sizeof v);
    cudaMemcpyToSymbol(g_taps, &z, sizeof z);
    return v;
}
#endif

}  // namespace
}  // namespace f16

// The FP16 launches of each tile height (hp_kernels_f16.cu: 64 x 8,
// hp_kernels_f16t4.cu: 64 x 4); arguments as f16::Dispatch<TH>::go.
cudaError_t f16_dispatch_th8(int mode, int radius, int stride, int staging, const BatchList* bl,
                             const SolveConsts& sc, int iteration, int color, const Schedule* s, int grid,
                             cudaStream_t st, int* occ);
cudaError_t f16_dispatch_th4(int mode, int radius, int stride, int staging, const BatchList* bl,
                             const SolveConsts& sc, int iteration, int color, const Schedule* s, int grid,
                             cudaStream_t st, int* occ);
#ifdef HP_COUNT_TAPS
unsigned long long f16_taps_th8();
unsigned long long f16_taps_th4();
unsigned long long f32_taps();
#endif

}  // namespace hp
