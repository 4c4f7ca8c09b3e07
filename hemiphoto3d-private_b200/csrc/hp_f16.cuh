// FP16-storage / FP32-accumulate PatchMatch device code for sm_100a, shared
// by the kernels of both lane layouts (hp_kernels_f16.cu: one lane per pixel
// visit; hp_kernels_f16x2.cu: two).
//
// Same algorithm as the FP32 path (initialisation is shared; cost,
// propagation and refinement follow src/dense_recon/patchmatch_mvs.cu:222-343
// and :519-655), re-derived for throughput:
//  - Sources are FP16: quad-packed texels read by a software bilinear sampler
//    (default), or FP16 textures through the hardware filter.
//  - Per (candidate, source) the plane-induced homography is folded into one
//    3x3 H = A + b (K^-T n)^T / (n.P).  A window row's taps are formed
//    directly from the row start: even taps j = 2m at w = fma(2m, H[:,0] s,
//    w_row), odd taps at fma(2m, H[:,0] s, w_row + H[:,0] s) - one paired
//    FMA per tap, the same bits whichever lane forms them.
//  - If the warped window's four corners lie inside the valid source region
//    (the warp of a rectangle with one-signed depth is the convex quad of its
//    corners) every tap is valid and the per-tap bounds tests are skipped.
//  - The reference window is mean-subtracted per pixel once per visit and kept
//    in shared memory as half2 pairs for windows of up to 64 taps.  Window
//    sums use mean-shifted values (compensated variance): FP16 products and
//    FP16 partial sums per window row (even and odd taps apart), flushed into
//    FP32 accumulators every row: the even taps' sum, then the odd taps'.
//  - Windows touching the source border mask invalid taps per the
//    reference's validity rules (|w_z| >= 1e-8, u in [0, W-1), v in [0, H-1),
//    count >= taps/2), vectorised like the fast path.
//
// Lane layouts (template parameter L).  L = 1: one lane scores a (pixel,
// candidate) item alone; a warp's 32 lanes are pixels 2 px apart, so one tap
// across the warp spans 64 px of a source row and touches every other 8-byte
// quad.  L = 2: a lane pair scores an item, the even lane its even taps and
// the odd lane its odd taps, two window rows per step; the pair's two lanes
// read taps 2 px apart and the next pixel's pair reads the same positions
// shifted by 2 px, so a warp's loads span 32 px and about half the L1
// wavefronts.  Each FP16 value is formed by the same operations in the same
// order in both layouts (a half2 holds two taps of one row for L = 1 and one
// tap of two rows for L = 2; every operation is elementwise), and the pair's
// even lane flushes the FP16 row sums of both lanes into FP32 in the one-lane
// order, so both layouts give the same bits.
#pragma once

#include <cuda_fp16.h>

#include <type_traits>

#include "hp_filter.cuh"
#include "hp_internal.h"
#include "hp_rng.cuh"
#include "hp_tile.cuh"

#ifndef HP_F16_MIN_BLOCKS
#define HP_F16_MIN_BLOCKS 3
#endif

namespace hp {
namespace f16 {

constexpr int MAX_TW = TILE_W + 2 * HP_MAX_RADIUS;
constexpr int MAX_TH = TILE_H + 2 * HP_MAX_RADIUS;
constexpr int WARPS = CTA_THREADS / 32;

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

__device__ __forceinline__ void load_ref_tile16(float* s_ref, int tw, int th, const ViewDesc* v, int x0, int y0,
                                                int r) {
    const int W = v->W, H = v->H;
    for (int i = threadIdx.x; i < tw * th; i += CTA_THREADS) {
        int ty = i / tw, tx = i - ty * tw;
        int gx = min(max(x0 - r + tx, 0), W - 1);
        int gy = min(max(y0 - r + ty, 0), H - 1);
        s_ref[i] = __half2float(v->ref16[static_cast<size_t>(gy) * v->ref16_pitch + gx]);
    }
}

// Window geometry and the shared-memory layout of the mean-subtracted
// reference window.  PAIRS half2 cover a row (L = 1: taps 2p and 2p + 1;
// L = 2: tap 2m + h of rows 2k and 2k + 1 for the lane of parity h).  The
// window sits in s_win as SLOTS slots (rows for L = 1, row pairs for L = 2)
// of [thread][L][VEC] half2, so a lane's part of a slot is one vector load.
template <int R, int ST, int L>
struct Win {
    static constexpr int SIDE = (2 * R) / ST + 1;
    static constexpr int N = SIDE * SIDE;
    static constexpr int PAIRS = (SIDE + 1) / 2;
    static constexpr int VEC = PAIRS <= 1 ? 1 : (PAIRS <= 2 ? 2 : 4);
    static constexpr int SLOTS = L == 1 ? SIDE : (SIDE + 1) / 2;
    static constexpr int COL = L * VEC;
    static constexpr bool IN_SMEM = PAIRS <= 4 && SLOTS * COL <= 32;
};
template <int V> struct WinRow;
template <> struct WinRow<1> { using T = unsigned; };
template <> struct WinRow<2> { using T = uint2; };
template <> struct WinRow<4> { using T = uint4; };
constexpr int WIN_PAIRS_MAX = 32;

struct RefStats {
    float mean;  // window mean (the shift of every sum)
    float ssd;   // sum (r - mean)^2
};

__device__ __forceinline__ __half2 pack_half2(float a, float b) { return __floats2half2_rn(a, b); }

// Window statistics of the pixel at (lx, ly) of the tile; with IN_SMEM its
// mean-subtracted window goes to this thread's s_win column.
template <int R, int ST, int L>
__device__ __forceinline__ RefStats load_window(__half2* s_win, const float* s_ref, int tw, int lx, int ly) {
    using Wn = Win<R, ST, L>;
    constexpr int SIDE = Wn::SIDE;
    float sum = 0.f;
#pragma unroll 1
    for (int i = 0; i < SIDE; ++i)
#pragma unroll
        for (int j = 0; j < SIDE; ++j) sum = __fadd_rn(sum, s_ref[(ly + i * ST) * tw + lx + j * ST]);
    const float mean = __fmul_rn(sum, 1.0f / Wn::N);
    float ssd = 0.f;
#pragma unroll 1
    for (int i = 0; i < SIDE; ++i)
#pragma unroll
        for (int j = 0; j < SIDE; ++j) {
            const float d = __fsub_rn(s_ref[(ly + i * ST) * tw + lx + j * ST], mean);
            ssd = __fmaf_rn(d, d, ssd);
        }
    if constexpr (Wn::IN_SMEM) {
        constexpr int PAIRS = Wn::PAIRS, VEC = Wn::VEC;
        auto res = [&](int i, int j) { return __fsub_rn(s_ref[(ly + i * ST) * tw + lx + j * ST], mean); };
#pragma unroll 1
        for (int k = 0; k < Wn::SLOTS; ++k) {
#pragma unroll
            for (int h = 0; h < L; ++h) {
                unsigned rw[VEC] = {};
#pragma unroll
                for (int p = 0; p < PAIRS; ++p) {
                    __half2 v;
                    if constexpr (L == 1) {
                        v = pack_half2(res(k, 2 * p), (2 * p + 1 < SIDE) ? res(k, 2 * p + 1) : 0.f);
                    } else {
                        const int j = 2 * p + h;
                        const bool tap = j < SIDE, two = 2 * k + 1 < SIDE;
                        v = pack_half2(tap ? res(2 * k, j) : 0.f, (tap && two) ? res(2 * k + 1, j) : 0.f);
                    }
                    memcpy(&rw[p], &v, sizeof v);
                }
                typename WinRow<VEC>::T row;
                memcpy(&row, rw, sizeof row);
                *reinterpret_cast<typename WinRow<VEC>::T*>(s_win + (k * CTA_THREADS + threadIdx.x) * Wn::COL +
                                                            h * VEC) = row;
            }
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

// s + x: sm_100's mixed-precision add takes the FP16 operand directly, with
// one rounding to FP32 (no conversion instruction).
__device__ __forceinline__ float add_h(float s, __half x) {
    asm("add.rn.f32.f16 %0, %1, %0;" : "+f"(s) : "h"(__half_as_ushort(x)));
    return s;
}

struct Plane {
    float h[9];  // homography (with the +0.5 texel offset folded into rows 0, 1 for texture taps)
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

// One tap's coordinates (w_x, w_y, w_z) from its parity's base: tap 2m of the
// base at fma(2m, step, base).
struct Coord {
    float2 xy;
    float z;
};
__device__ __forceinline__ Coord tap_coord(Coord base, int m2, float2 step_xy, float step_z) {
    if (m2 == 0) return base;
    const float f = static_cast<float>(m2);
    return Coord{__ffma2_rn(make_float2(f, f), step_xy, base.xy), __fmaf_rn(f, step_z, base.z)};
}

// A tap fetch in flight: the quad (software sampler) or the filtered sample
// (texture), its weight bits, and whether it is valid (CHECK).
template <bool CHECK, bool SOFT>
__device__ __forceinline__ void fetch_tap(Coord c, cudaTextureObject_t tex, const uint2* qbase, float lo, float fW,
                                          float fH, uint2* q, unsigned* wb, float* smp, bool* valid) {
    const float iz = rcp_approx(c.z);
    if constexpr (SOFT) {
        const float2 izz = make_float2(iz, iz);
        const float2 fxy = __ffma2_rn(c.xy, izz, make_float2(SOFT_MAGIC, SOFT_MAGIC));
        unsigned bu = __float_as_uint(fxy.x), bv = __float_as_uint(fxy.y);
        if constexpr (CHECK) {
            const float2 uv = __fmul2_rn(c.xy, izz);
            const bool skip = fabsf(c.z) < 1e-8f || !(uv.x >= lo) || !(uv.x < fW - 1.0f + lo) || !(uv.y >= lo) ||
                              !(uv.y < fH - 1.0f + lo);
            *valid = !skip;
            bu = skip ? SOFT_ORIGIN : bu;  // an in-bounds quad; the tap is masked
            bv = skip ? SOFT_ORIGIN : bv;
        }
        *wb = __byte_perm(bu, bv, 0x7430);
        *q = __ldg(qbase + soft_offset(bu, bv));
    } else {
        const float u = __fmul_rn(c.xy.x, iz), v = __fmul_rn(c.xy.y, iz);  // texel-centre offset folded in
        if constexpr (CHECK) {
            const bool skip =
                fabsf(c.z) < 1e-8f || !(u >= lo) || !(u < fW - 1.0f + lo) || !(v >= lo) || !(v < fH - 1.0f + lo);
            *valid = !skip;
        }
        *smp = tex2D<float>(tex, u, v);
    }
}

// Accumulators of one FP16 chain set: a1 = sum e, a2 = sum e^2, a3 = sum r e,
// and with CHECK a4 = sum r, a5 = sum r^2 (over the valid taps).
template <bool CHECK>
struct Acc16 {
    __half2 a1, a2, a3, a4, a5;
    __device__ __forceinline__ void add(int p, __half2 e, __half2 rq) {
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
    }
};

__device__ __forceinline__ unsigned mask_half2(unsigned bits, bool lo, bool hi) {
    return bits & ((lo ? 0x0000ffffu : 0u) | (hi ? 0xffff0000u : 0u));
}
__device__ __forceinline__ __half2 masked(__half2 v, bool lo, bool hi) {
    unsigned b;
    memcpy(&b, &v, sizeof b);
    b = mask_half2(b, lo, hi);
    memcpy(&v, &b, sizeof b);
    return v;
}

// FP32 accumulators of the window sums, flushed row by row from the FP16
// chains (the low or the high half of each).
template <bool CHECK>
struct Sum32 {
    float s1 = 0.f, s2 = 0.f, s3 = 0.f, r1 = 0.f, r2 = 0.f;
    __device__ __forceinline__ void flush(const Acc16<CHECK>& a, bool hi) {
        s1 = add_h(s1, hi ? __high2half(a.a1) : __low2half(a.a1));
        s2 = add_h(s2, hi ? __high2half(a.a2) : __low2half(a.a2));
        s3 = add_h(s3, hi ? __high2half(a.a3) : __low2half(a.a3));
        if constexpr (CHECK) {
            r1 = add_h(r1, hi ? __high2half(a.a4) : __low2half(a.a4));
            r2 = add_h(r2, hi ? __high2half(a.a5) : __low2half(a.a5));
        }
    }
};

// Cost (1 - NCC, or 2 when invalid) of one source for the pixel (x, y) whose
// window statistics are st and whose s_win column (with this lane's half, L =
// 2) starts at s_win.  CHECK = false assumes every tap is valid (the caller's
// corner test proved it); CHECK = true applies the reference's validity rules
// per tap by masking the tap's terms.  With every tap valid both forms give
// the same bits.  SOFT selects the software sampler; P then holds the
// homography without the texture's +0.5 texel-centre offset.  h is the lane's
// parity within its pair (L = 2); both lanes of a pair return the same value.
template <int R, int ST, bool CHECK, bool SOFT, int L>
__device__ __forceinline__ float source_cost(const Plane& P, cudaTextureObject_t tex, const uint2* qbase, RefStats st,
                                             const __half2* s_win, const float* s_ref, int tw, int lx, int ly, int x,
                                             int y, float fW, float fH, int h) {
    using Wn = Win<R, ST, L>;
    constexpr int SIDE = Wn::SIDE, PAIRS = Wn::PAIRS, N = Wn::N, VEC = Wn::VEC;
    const float c0 = st.mean;
    const __half2 c0s = __float2half2_rn(__fsub_rn(c0, 0.5f));
    constexpr float LO = SOFT ? 0.0f : 0.5f;  // validity bounds of the coordinate: [LO, W - 1 + LO)
    const float sx0 = static_cast<float>(x - R), sy0 = static_cast<float>(y - R);
    const float2 step = make_float2(__fmul_rn(P.h[0], ST), __fmul_rn(P.h[3], ST));
    const float stepz = __fmul_rn(P.h[6], ST);
    const float2 r01 = make_float2(__fmaf_rn(P.h[0], sx0, P.h[2]), __fmaf_rn(P.h[3], sx0, P.h[5]));
    const float r2 = __fmaf_rn(P.h[6], sx0, P.h[8]);
    const float2 h14 = make_float2(P.h[1], P.h[4]);
    // Row start of window row i.
    auto row_start = [&](int i) {
        const float py = __fadd_rn(sy0, static_cast<float>(i * ST));
        return Coord{__ffma2_rn(h14, make_float2(py, py), r01), __fmaf_rn(P.h[7], py, r2)};
    };
    // Base of the taps of parity q (0 or 1) of a row: the row start, or the
    // row start plus one step (fma(q, step, start): the start itself for q = 0,
    // up to the sign of a zero, which no later operation distinguishes).
    auto parity_base = [&](Coord c, float q) {
        return Coord{__ffma2_rn(make_float2(q, q), step, c.xy), __fmaf_rn(q, stepz, c.z)};
    };
    // Residual pair from the reference tile (windows too large for s_win).
    auto ref_res = [&](int i, int j) { return __fsub_rn(s_ref[(ly + i * ST) * tw + lx + j * ST], c0); };
    Sum32<CHECK> sum;  // FP32 row flushes, in row order, each row's even taps then its odd taps
    int count = 0;
    if constexpr (L == 1) {
#pragma unroll 1
        for (int i = 0; i < SIDE; ++i) {
            const Coord b0 = row_start(i), b1 = parity_base(b0, 1.0f);
            [[maybe_unused]] unsigned ok = 0;
            [[maybe_unused]] unsigned rw[VEC];
            if constexpr (Wn::IN_SMEM) {
                const auto row = *reinterpret_cast<const typename WinRow<VEC>::T*>(s_win + i * CTA_THREADS * VEC);
                memcpy(rw, &row, sizeof row);
            }
            Acc16<CHECK> acc;
            constexpr int CHUNKS = (SIDE + 3) / 4;
#pragma unroll
            for (int ch = 0; ch < CHUNKS; ++ch) {
                uint2 q[4];
                unsigned wb[4];
                float smp[4];
                bool val[4];
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) {
                    const int j = 4 * ch + jj;
                    val[jj] = false;
                    if (j >= SIDE) break;
                    const Coord c = tap_coord((j & 1) ? b1 : b0, j & ~1, step, stepz);
                    fetch_tap<CHECK, SOFT>(c, tex, qbase, LO, fW, fH, &q[jj], &wb[jj], &smp[jj], &val[jj]);
                    if constexpr (CHECK) ok |= static_cast<unsigned>(val[jj]) << j;
                }
#pragma unroll
                for (int pp = 0; pp < 2; ++pp) {
                    const int p = 2 * ch + pp;
                    if (p >= PAIRS) break;
                    const bool has_b = 2 * p + 1 < SIDE;
                    __half2 e;
                    if constexpr (SOFT) {
                        const __half sa = soft_lerp(q[2 * pp], wb[2 * pp]);
                        const __half sb = has_b ? soft_lerp(q[2 * pp + 1], wb[2 * pp + 1]) : __low2half(c0s);
                        e = __hsub2(__halves2half2(sa, sb), c0s);
                    } else {
                        e = pack_half2(__fsub_rn(smp[2 * pp], c0), has_b ? __fsub_rn(smp[2 * pp + 1], c0) : 0.f);
                    }
                    __half2 rq;
                    if constexpr (Wn::IN_SMEM) {
                        memcpy(&rq, &rw[p], sizeof rq);
                    } else {
                        rq = pack_half2(ref_res(i, 2 * p), has_b ? ref_res(i, 2 * p + 1) : 0.f);
                    }
                    if constexpr (CHECK) {
                        const bool va = val[2 * pp], vb = has_b && val[2 * pp + 1];
                        rq = masked(rq, va, vb);
                        e = masked(e, va, vb);
                    }
                    acc.add(p, e, rq);
                }
            }
            sum.flush(acc, false);
            sum.flush(acc, true);
            if constexpr (CHECK) count += __popc(ok);
        }
    } else {
        const float hf = static_cast<float>(h);
        const unsigned pm = 3u << (threadIdx.x & 30);  // this lane's pair
        // Row pair (i0, i0 + 1); TWO = false for the last, single row of an odd window.
        auto row_pair = [&](int i0, auto two_tag) {
            constexpr bool TWO = decltype(two_tag)::value;
            const Coord b0 = parity_base(row_start(i0), hf);
            const Coord b1 = TWO ? parity_base(row_start(i0 + 1), hf) : b0;
            [[maybe_unused]] unsigned ok = 0;
            [[maybe_unused]] unsigned rw[VEC];
            if constexpr (Wn::IN_SMEM) {
                const auto row = *reinterpret_cast<const typename WinRow<VEC>::T*>(
                    s_win + (i0 >> 1) * CTA_THREADS * Wn::COL);
                memcpy(rw, &row, sizeof row);
            }
            Acc16<CHECK> acc;
            constexpr int CH = 2;  // taps per chunk: 4 fetches in flight
            constexpr int CHUNKS = (PAIRS + CH - 1) / CH;
#pragma unroll
            for (int ch = 0; ch < CHUNKS; ++ch) {
                uint2 q[2 * CH];
                unsigned wb[2 * CH];
                float smp[2 * CH];
                bool val[2 * CH];
#pragma unroll
                for (int mm = 0; mm < CH; ++mm) {
                    const int m = CH * ch + mm;
                    val[2 * mm] = val[2 * mm + 1] = false;
                    if (m >= PAIRS) break;
                    fetch_tap<CHECK, SOFT>(tap_coord(b0, 2 * m, step, stepz), tex, qbase, LO, fW, fH, &q[2 * mm],
                                           &wb[2 * mm], &smp[2 * mm], &val[2 * mm]);
                    if (TWO)
                        fetch_tap<CHECK, SOFT>(tap_coord(b1, 2 * m, step, stepz), tex, qbase, LO, fW, fH,
                                               &q[2 * mm + 1], &wb[2 * mm + 1], &smp[2 * mm + 1], &val[2 * mm + 1]);
                }
#pragma unroll
                for (int mm = 0; mm < CH; ++mm) {
                    const int m = CH * ch + mm;
                    if (m >= PAIRS) break;
                    // The odd lane's last tap of an odd-width row is padding (e = 0, r = 0).
                    const bool tap = !((SIDE & 1) && m == PAIRS - 1 && h);
                    __half2 e;
                    if constexpr (SOFT) {
                        const __half sa = soft_lerp(q[2 * mm], wb[2 * mm]);
                        const __half sb = TWO ? soft_lerp(q[2 * mm + 1], wb[2 * mm + 1]) : __low2half(c0s);
                        e = __hsub2(__halves2half2(sa, sb), c0s);
                    } else {
                        e = pack_half2(__fsub_rn(smp[2 * mm], c0), TWO ? __fsub_rn(smp[2 * mm + 1], c0) : 0.f);
                    }
                    e = masked(e, tap, tap && TWO);
                    __half2 rq;
                    if constexpr (Wn::IN_SMEM) {
                        memcpy(&rq, &rw[m], sizeof rq);
                    } else {
                        const int j = 2 * m + h;
                        rq = pack_half2(tap ? ref_res(i0, j) : 0.f, (tap && TWO) ? ref_res(i0 + 1, j) : 0.f);
                    }
                    if constexpr (CHECK) {
                        const bool va = tap && val[2 * mm], vb = tap && TWO && val[2 * mm + 1];
                        ok |= (static_cast<unsigned>(va) << m) | (static_cast<unsigned>(vb) << (m + 8));
                        rq = masked(rq, va, vb);
                        e = masked(e, va, vb);
                    }
                    acc.add(m, e, rq);
                }
            }
            // The even lane flushes the pair's rows in the one-lane order
            // (row i0's even taps, its odd taps, then row i0 + 1's); the odd
            // lane's sums are not used.
            Acc16<CHECK> other;
            other.a1 = __shfl_xor_sync(pm, acc.a1, 1);
            other.a2 = __shfl_xor_sync(pm, acc.a2, 1);
            other.a3 = __shfl_xor_sync(pm, acc.a3, 1);
            if constexpr (CHECK) {
                other.a4 = __shfl_xor_sync(pm, acc.a4, 1);
                other.a5 = __shfl_xor_sync(pm, acc.a5, 1);
            }
            sum.flush(acc, false);
            sum.flush(other, false);
            if (TWO) {
                sum.flush(acc, true);
                sum.flush(other, true);
            }
            if constexpr (CHECK) count += __popc(ok);
        };
#pragma unroll 1
        for (int i0 = 0; i0 + 1 < SIDE; i0 += 2) row_pair(i0, std::true_type{});
        if constexpr (SIDE & 1) row_pair(SIDE - 1, std::false_type{});
        // Both lanes take the even lane's sums; the counts add up.
        const int src = threadIdx.x & 31 & ~1;
        sum.s1 = __shfl_sync(pm, sum.s1, src);
        sum.s2 = __shfl_sync(pm, sum.s2, src);
        sum.s3 = __shfl_sync(pm, sum.s3, src);
        if constexpr (CHECK) {
            sum.r1 = __shfl_sync(pm, sum.r1, src);
            sum.r2 = __shfl_sync(pm, sum.r2, src);
            count += __shfl_xor_sync(pm, count, 1);
        }
    }
    const float s1 = sum.s1, s2 = sum.s2, s3 = sum.s3;
    float n = static_cast<float>(N), dr, num;
    if (!CHECK || count == N) {
        // n*sum(r^2)-sum(r)^2 = n*ssd and the covariance numerator is n*s3 (sum(r - mean) = 0).
        dr = __fmul_rn(n, st.ssd);
        num = __fmul_rn(n, s3);
    } else {
        if (count < N / 2) return 2.0f;
        const float r1 = sum.r1, r2s = sum.r2;
        n = static_cast<float>(count);
        dr = __fmaf_rn(n, r2s, -__fmul_rn(r1, r1));
        num = __fmaf_rn(n, s3, -__fmul_rn(r1, s1));
    }
    const float ds = __fmaf_rn(n, s2, -__fmul_rn(s1, s1));
    if (dr < 1e-6f || ds < 1e-6f) return 2.0f;
    const float ncc = fmaxf(-1.0f, fminf(1.0f, __fmul_rn(__fmul_rn(num, rsqrtf(dr)), rsqrtf(ds))));
    return __fsub_rn(1.0f, ncc);
}

// Corner flags of the warped window against the valid source region (bit 0:
// inside with margin, 1: in front, 2..5: beyond the left / right / top /
// bottom edge by the margin), for corner c (0: top-left, 1: top-right, 2:
// bottom-left, 3: bottom-right).  Tested as w_x >= lo w_z etc. without a
// division.  A 0.05 px margin covers the rounding of the taps' coordinates.
template <int R, int ST>
__device__ __forceinline__ unsigned corner_flags(const Plane& P, float xa, float ya, int c, float lo, float fW,
                                                 float fH) {
    constexpr float SPAN = static_cast<float>((Win<R, ST, 1>::SIDE - 1) * ST);
    const float cxp = (c & 1) ? __fadd_rn(xa, SPAN) : xa, cyp = (c & 2) ? __fadd_rn(ya, SPAN) : ya;
    const float wz = __fmaf_rn(P.h[6], cxp, __fmaf_rn(P.h[7], cyp, P.h[8]));
    const float wxc = __fmaf_rn(P.h[0], cxp, __fmaf_rn(P.h[1], cyp, P.h[2]));
    const float wyc = __fmaf_rn(P.h[3], cxp, __fmaf_rn(P.h[4], cyp, P.h[5]));
    const float ulo = __fadd_rn(lo, 0.05f), uhi = __fsub_rn(__fadd_rn(fW, lo), 1.05f);
    const float vhi = __fsub_rn(__fadd_rn(fH, lo), 1.05f);
    const float olo = __fsub_rn(lo, 0.05f), ohi = __fadd_rn(__fadd_rn(fW, lo), -0.95f);
    const float ovhi = __fadd_rn(__fadd_rn(fH, lo), -0.95f);
    const bool front = wz > 1e-6f;
    const bool inside = front && wxc >= __fmul_rn(ulo, wz) && wxc < __fmul_rn(uhi, wz) &&
                        wyc >= __fmul_rn(ulo, wz) && wyc < __fmul_rn(vhi, wz);
    return static_cast<unsigned>(inside) | (static_cast<unsigned>(front) << 1) |
           (static_cast<unsigned>(wxc < __fmul_rn(olo, wz)) << 2) |
           (static_cast<unsigned>(wxc >= __fmul_rn(ohi, wz)) << 3) |
           (static_cast<unsigned>(wyc < __fmul_rn(olo, wz)) << 4) |
           (static_cast<unsigned>(wyc >= __fmul_rn(ovhi, wz)) << 5);
}

// Top-k mean NCC cost of plane (d, n) at pixel (x, y) over the view's sources.
template <int R, int ST, int L>
__device__ __forceinline__ float cost_f16(RefStats st, const __half2* s_win, const float* s_ref, int tw, int lx,
                                          int ly, int x, int y, float d, float cnx, float cny, float cnz,
                                          const ViewDesc* __restrict__ v, int topk, unsigned soft_mask, int h) {
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
        // Corner test (flags ANDed over the corners).  Inside: every tap is
        // valid, so the per-tap tests can be skipped.  Fully outside: in front
        // at every corner and every corner beyond the same edge, so every tap
        // is invalid, the count is 0 and the reference's rule makes the cost 2
        // without sampling.  L = 2 splits the corners over the pair.
        unsigned f;
        if constexpr (L == 1) {
            f = corner_flags<R, ST>(P, xa, ya, 0, lo, fW, fH) & corner_flags<R, ST>(P, xa, ya, 1, lo, fW, fH) &
                corner_flags<R, ST>(P, xa, ya, 2, lo, fW, fH) & corner_flags<R, ST>(P, xa, ya, 3, lo, fW, fH);
        } else {
            f = corner_flags<R, ST>(P, xa, ya, 2 * h, lo, fW, fH) & corner_flags<R, ST>(P, xa, ya, 2 * h + 1, lo, fW, fH);
            f &= __shfl_xor_sync(3u << (threadIdx.x & 30), f, 1);
        }
        const bool inside = f & 1u;
        const bool outside = (f & 2u) && (f & 0x3cu);
        // One form per warp for the lanes that sample: the checked form gives
        // the unchecked form's bits whenever every tap is valid.
        const bool all_inside = __all_sync(__activemask(), inside || outside);
        float c = 2.0f;
        if (outside) {
        } else if (soft) {
            const uint2* qb = soft_base(v->src_quad[s]);
            c = all_inside ? source_cost<R, ST, false, true, L>(P, 0, qb, st, s_win, s_ref, tw, lx, ly, x, y, fW, fH, h)
                           : source_cost<R, ST, true, true, L>(P, 0, qb, st, s_win, s_ref, tw, lx, ly, x, y, fW, fH, h);
        } else {
            const cudaTextureObject_t tex = v->src_tex16[s];
            c = all_inside
                    ? source_cost<R, ST, false, false, L>(P, tex, nullptr, st, s_win, s_ref, tw, lx, ly, x, y, fW, fH, h)
                    : source_cost<R, ST, true, false, L>(P, tex, nullptr, st, s_win, s_ref, tw, lx, ly, x, y, fW, fH, h);
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

// s_win column of thread t's pixel for this lane (its half of a pair's slot for L = 2).
template <int R, int ST, int L>
__device__ __forceinline__ const __half2* win_col(const __half2* s_win, int t, int h) {
    using Wn = Win<R, ST, L>;
    return s_win + t * Wn::COL + (L == 2 ? h * Wn::VEC : 0);
}

// Shared memory of the half-pass beyond the reference tile and window.
// The refinement phase (L = 2) reuses the neighbour phase's space: a warp's
// candidate planes overlay its own cost slots (lane l's plane covers lane l's
// four slots, which it has read by then), and the candidate costs overlay the
// item list, which nothing reads after the neighbour phase's last barrier.
struct PassSmem {
    union {
        float cost[WARPS][32 * 4];      // neighbour cost, slot (lane << 2 | cand) of the owner's warp
        float4 plane[WARPS][32];        // L = 2 refinement: the owners' candidate planes
    };
    union {
        unsigned short items[WARPS * 128];  // CTA item list: warp << 7 | lane << 2 | cand
        float rcost[WARPS][32];             // L = 2 refinement: the candidates' costs
    };
    float2 stat[CTA_THREADS];           // (mean, ssd) of each thread's pixel window
    int warp_total[WARPS];
};

// Initial cost of one tile.  L = 1: each thread scores its two pixels; L = 2:
// per column parity, every thread prepares its pixel's window, then each
// warp's lane pairs score the warp's 32 pixels, 16 at a time.
template <int R, int ST, int L>
__device__ __forceinline__ void tile_cost16(const ViewDesc* v, int tile_x, int tile_y, const SolveConsts& sc,
                                            float* s_ref, __half2* s_win) {
    constexpr int tw = TILE_W + 2 * R, th = TILE_H + 2 * R;
    const int x0 = tile_x * TILE_W, y0 = tile_y * TILE_H;
    load_ref_tile16(s_ref, tw, th, v, x0, y0, R);
    __syncthreads();
    const int ly = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = y0 + ly;
    if (y >= v->H) return;  // a whole warp (one row) leaves together
    for (int j = 0; j < 2; ++j) {
        if constexpr (L == 1) {
            const int lx = 2 * lane + j, x = x0 + lx;
            if (x >= v->W) continue;
            const RefStats st = load_window<R, ST, 1>(s_win, s_ref, tw, lx, ly);
            const size_t idx = static_cast<size_t>(y) * v->W + x;
            const float4 hh = v->hyp[idx];
            v->cost[idx] = cost_f16<R, ST, 1>(st, win_col<R, ST, 1>(s_win, threadIdx.x, 0), s_ref, tw, lx, ly, x, y,
                                              hh.x, hh.y, hh.z, hh.w, v, sc.top_k, sc.soft_mask, 0);
        } else {
            const RefStats own = load_window<R, ST, 2>(s_win, s_ref, tw, 2 * lane + j, ly);
            __syncwarp();
            const int h = lane & 1;
            for (int round = 0; round < 2; ++round) {
                const int o = 16 * round + (lane >> 1);  // owner lane of the pair's pixel
                const float mean = __shfl_sync(0xffffffffu, own.mean, o);
                const float ssd = __shfl_sync(0xffffffffu, own.ssd, o);
                const int lx = 2 * o + j, x = x0 + lx;
                if (x < v->W) {
                    const size_t idx = static_cast<size_t>(y) * v->W + x;
                    const float4 hh = v->hyp[idx];
                    const float c = cost_f16<R, ST, 2>(RefStats{mean, ssd},
                                                       win_col<R, ST, 2>(s_win, ly * 32 + o, h), s_ref, tw, lx, ly,
                                                       x, y, hh.x, hh.y, hh.z, hh.w, v, sc.top_k, sc.soft_mask, h);
                    if (h == 0) v->cost[idx] = c;
                }
            }
            __syncwarp();  // the next parity overwrites the warp's s_win columns
        }
    }
}

// One red-black half-pass.  The neighbour phase is compacted across the CTA:
// every lane lists the neighbour planes its pixel must score (duplicates of
// the current plane or of an earlier neighbour skipped), the lists of all
// eight warps are concatenated in shared memory, and the warps score the
// union (L = 1: 32 items per warp step; L = 2: 16, one per lane pair).  An
// item reads its owner pixel's window statistics and s_win column from shared
// memory and leaves its cost in the owner's slot, so owners then fold the
// costs in L, R, U, D order exactly as if they had scored them themselves:
// results do not depend on which lane scored what.
template <int R, int ST, int L>
__device__ __forceinline__ void tile_propagate16(const ViewDesc* v, int tile_x, int tile_y, const SolveConsts& sc,
                                                 int iteration, int color, float* s_ref, __half2* s_win,
                                                 PassSmem& sm) {
    constexpr int tw = TILE_W + 2 * R, th = TILE_H + 2 * R;
    const int x0 = tile_x * TILE_W, y0 = tile_y * TILE_H;
    load_ref_tile16(s_ref, tw, th, v, x0, y0, R);
    __syncthreads();
    const int W = v->W, H = v->H;
    const int ly = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int h = L == 2 ? (lane & 1) : 0;
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
        st = load_window<R, ST, L>(s_win, s_ref, tw, lx, ly);
        best = v->hyp[idx];
        best_cost = v->cost[idx];
#pragma unroll
        for (int cand = 0; cand < 4; ++cand) {
            const int nxp = x + (cand == 0 ? -1 : (cand == 1 ? 1 : 0));
            const int nyp = y + (cand == 2 ? -1 : (cand == 3 ? 1 : 0));
            if (nxp < 0 || nxp >= W || nyp < 0 || nyp >= H) continue;
            const float4 hn = v->hyp[static_cast<size_t>(nyp) * W + nxp];
            if (hn.x < dmin || hn.x > dmax) continue;
            bool dup = same_plane16(hn, best);
            for (int j = 0; j < cand && !dup; ++j) {
                if (need & (1u << j)) {
                    const int jx = x + (j == 0 ? -1 : (j == 1 ? 1 : 0));
                    const int jy = y + (j == 2 ? -1 : (j == 3 ? 1 : 0));
                    dup = same_plane16(hn, v->hyp[static_cast<size_t>(jy) * W + jx]);
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
    constexpr int PER_WARP = 32 / L;  // items a warp scores per step
    for (int base = ly * PER_WARP; base < total; base += WARPS * PER_WARP) {
        const int w = base + (L == 2 ? (lane >> 1) : lane);
        if (w < total) {
            const int item = sm.items[w];
            const int oly = item >> 7, owner = (item >> 2) & 31, cand = item & 3;
            const int oy = y0 + oly, olx = 2 * owner + ((oy + color) & 1), ox = x0 + olx;
            const float2 os = sm.stat[oly * 32 + owner];
            const int nxp = ox + (cand == 0 ? -1 : (cand == 1 ? 1 : 0));
            const int nyp = oy + (cand == 2 ? -1 : (cand == 3 ? 1 : 0));
            const float4 hn = v->hyp[static_cast<size_t>(nyp) * W + nxp];
            const float c = cost_f16<R, ST, L>(RefStats{os.x, os.y}, win_col<R, ST, L>(s_win, oly * 32 + owner, h),
                                               s_ref, tw, olx, oly, ox, oy, hn.x, hn.y, hn.z, hn.w, v, sc.top_k,
                                               sc.soft_mask, h);
            if (h == 0) sm.cost[oly][item & 127] = c;
        }
    }
    __syncthreads();  // every neighbour cost is in its owner's slot
    if (active) {
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
    }
    if constexpr (L == 1) {
        if (!active) return;
    } else {
        // Every lane of a warp stays for the refinement rounds (lane pairs span owners).
        if (y >= H) return;  // a whole warp
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
        float c;
        if constexpr (L == 1) {
            c = cost_f16<R, ST, 1>(st, win_col<R, ST, 1>(s_win, threadIdx.x, 0), s_ref, tw, lx, ly, x, y, cd, cn.x,
                                   cn.y, cn.z, v, sc.top_k, sc.soft_mask, 0);
        } else {
            // The warp's owners post their candidates; lane pairs score them 16 at a time.
            sm.plane[ly][lane] = make_float4(cd, cn.x, cn.y, cn.z);
            __syncwarp();
            for (int round = 0; round < 2; ++round) {
                const int o = 16 * round + (lane >> 1);
                const int olx = 2 * o + parity, ox = x0 + olx;
                if (ox < W) {
                    const float4 pl = sm.plane[ly][o];
                    const float2 os = sm.stat[ly * 32 + o];
                    const float cc = cost_f16<R, ST, 2>(RefStats{os.x, os.y}, win_col<R, ST, 2>(s_win, ly * 32 + o, h),
                                                        s_ref, tw, olx, ly, ox, y, pl.x, pl.y, pl.z, pl.w, v, sc.top_k,
                                                        sc.soft_mask, h);
                    if (h == 0) sm.rcost[ly][o] = cc;
                }
            }
            __syncwarp();
            c = sm.rcost[ly][lane];
            __syncwarp();  // read before the next step overwrites
        }
        if (active && c < best_cost) {
            best_cost = c;
            best = make_float4(cd, cn.x, cn.y, cn.z);
        }
        drange = __fmul_rn(drange, sc.step_decay);
        nrange = __fmul_rn(nrange, sc.step_decay);
    }
    if (!active) return;
    v->hyp[idx] = best;
    v->cost[idx] = best_cost;
}

template <int R, int ST, int L>
__global__ void __launch_bounds__(CTA_THREADS, HP_F16_MIN_BLOCKS) cost16_kernel(BatchList bl, SolveConsts sc) {
    __shared__ float s_ref[MAX_TW * MAX_TH];
    __shared__ __align__(16) __half2 s_win[Win<R, ST, L>::IN_SMEM ? WIN_PAIRS_MAX * CTA_THREADS : 1];
    int tile_x, tile_y;
    const ViewDesc* v = locate_tile16(bl, blockIdx.x, &tile_x, &tile_y);
    tile_cost16<R, ST, L>(v, tile_x, tile_y, sc, s_ref, s_win);
}

template <int R, int ST, int L>
__global__ void __launch_bounds__(CTA_THREADS, HP_F16_MIN_BLOCKS) propagate16_kernel(BatchList bl, SolveConsts sc,
                                                                                     int iteration, int color) {
    __shared__ float s_ref[MAX_TW * MAX_TH];
    __shared__ __align__(16) __half2 s_win[Win<R, ST, L>::IN_SMEM ? WIN_PAIRS_MAX * CTA_THREADS : 1];
    __shared__ PassSmem sm;
    int tile_x, tile_y;
    const ViewDesc* v = locate_tile16(bl, blockIdx.x, &tile_x, &tile_y);
    tile_propagate16<R, ST, L>(v, tile_x, tile_y, sc, iteration, color, s_ref, s_win, sm);
}

// Persistent form (see Schedule and the FP32 persistent kernel): the stage
// bodies are those of the per-stage kernels, so the results are bit-identical.
template <int R, int ST, int L>
__global__ void __launch_bounds__(CTA_THREADS, HP_F16_MIN_BLOCKS) persistent16_kernel(Schedule s) {
    __shared__ float s_ref[MAX_TW * MAX_TH];
    __shared__ __align__(16) __half2 s_win[Win<R, ST, L>::IN_SMEM ? WIN_PAIRS_MAX * CTA_THREADS : 1];
    __shared__ PassSmem sm;
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
        if (stage == 0) {
            tile_init(v, tx, ty);
            __syncthreads();
            tile_cost16<R, ST, L>(v, tx, ty, s.sc, s_ref, s_win);
        } else if (stage <= 2 * v->iterations) {
            const int k = stage - 1;
            tile_propagate16<R, ST, L>(v, tx, ty, s.sc, k >> 1, k & 1, s_ref, s_win, sm);
        } else if (is_filter_stage(v, stage)) {
            tile_filter(s.views, v, tx, ty, true);  // geometric check, then the maps
        } else {
            tile_unpack(v, tx, ty);
        }
        __syncthreads();
        if (threadIdx.x == 0) sched_publish(s, s_tile);
    }
}

// Launch or occupancy query of one lane layout, dispatched on (radius, stride).
// mode 0: cost kernel, 1: propagate half-pass, 2: persistent (occ: query only).
template <int L>
struct Dispatch {
    template <int R, int ST>
    static cudaError_t run(int mode, const BatchList* bl, const SolveConsts& sc, int iteration, int color,
                           const Schedule* s, int grid, cudaStream_t st, int* occ) {
        if (mode == 2) {
            if (occ)
                return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, persistent16_kernel<R, ST, L>, CTA_THREADS, 0);
            persistent16_kernel<R, ST, L><<<grid, CTA_THREADS, 0, st>>>(*s);
        } else if (mode == 0) {
            cost16_kernel<R, ST, L><<<bl->total_tiles, CTA_THREADS, 0, st>>>(*bl, sc);
        } else {
            propagate16_kernel<R, ST, L><<<bl->total_tiles, CTA_THREADS, 0, st>>>(*bl, sc, iteration, color);
        }
        return cudaGetLastError();
    }
    static cudaError_t go(int mode, int radius, int stride, const BatchList* bl, const SolveConsts& sc, int iteration,
                          int color, const Schedule* s, int grid, cudaStream_t st, int* occ) {
        if (stride != 1 && stride != 2) return cudaErrorInvalidValue;
#define HP_CASE(RR)                                                                                \
    case RR:                                                                                       \
        return stride == 1 ? run<RR, 1>(mode, bl, sc, iteration, color, s, grid, st, occ)          \
                           : run<RR, 2>(mode, bl, sc, iteration, color, s, grid, st, occ);
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

}  // namespace f16

// The FP16 launches of each lane layout (hp_kernels_f16.cu: L = 1,
// hp_kernels_f16x2.cu: L = 2); same arguments as f16::Dispatch<L>::go.
cudaError_t f16_dispatch_l1(int mode, int radius, int stride, const BatchList* bl, const SolveConsts& sc,
                            int iteration, int color, const Schedule* s, int grid, cudaStream_t st, int* occ);
cudaError_t f16_dispatch_l2(int mode, int radius, int stride, const BatchList* bl, const SolveConsts& sc,
                            int iteration, int color, const Schedule* s, int grid, cudaStream_t st, int* occ);

}  // namespace hp
