// Plain FP32 PatchMatch kernels for sm_100a: hypothesis initialisation, full-map
// NCC cost, and the fused red-black propagate + refine pass.
//
// Parity contract.  The reference's cost (computePixelCost,
// src/dense_recon/patchmatch_mvs.cu:222-343) samples sources through the
// texture unit's linear filter, whose weights carry only 8 fractional bits; a
// warped coordinate that moves by one ulp can flip a weight by 1/256 and the
// cost by ~1e-5.  To hold the 1e-5 bound this file reproduces the reference's
// per-tap rounding exactly - the operation sequence its --use_fast_math build
// executes, pinned with explicitly rounded intrinsics (see cost_f32) - and
// samples sources with tex2D on the same filter configuration; the per-pixel
// plane setup and the NCC finalisation keep the reference's expressions in a
// translation unit built with the same flags.  The result is bit-identical to
// the reference's compute_ncc_cost_kernel.  Everything around the arithmetic
// is this engine's own: packed float4 hypotheses, a shared-memory reference
// tile, red-black compaction (every thread owns a pixel of the active color),
// row-batched texture fetches, duplicate-candidate elimination, batched
// multi-view launches and counter-based RNG.  Engine-defined arithmetic
// outside the taps (initialisation, refinement) uses explicitly rounded
// intrinsics so the CPU restatement reproduces it bit for bit.
#include "hp_internal.h"
#include "hp_rng.cuh"
#include "hp_filter.cuh"
#include "hp_tile.cuh"

// Resident CTAs per SM the cost kernels are register-budgeted for.
#ifndef HP_F32_MIN_BLOCKS
#define HP_F32_MIN_BLOCKS 2
#endif

namespace hp {

#ifdef HP_COUNT_TAPS
// Instrumented builds only (make count): taps sampled.
__device__ unsigned long long g_taps32;
unsigned long long f32_taps() {
    unsigned long long v = 0, z = 0;
    cudaDeviceSynchronize();
    cudaMemcpyFromSymbol(&v, g_taps32, sizeof v);
    cudaMemcpyToSymbol(g_taps32, &z, sizeof z);
    return v;
}
#endif

namespace {

constexpr int MAX_TW = TILE_W + 2 * HP_MAX_RADIUS;
constexpr int MAX_TH = TILE_H + 2 * HP_MAX_RADIUS;

// Locate the view and tile of this CTA in a batch launch.
__device__ __forceinline__ const ViewDesc* locate_tile(const BatchList& bl, int t, int* tx, int* ty) {
    int lo = 0, hi = bl.n_active - 1;
    while (lo < hi) {  // last k with tile_prefix[k] <= t
        int mid = (lo + hi + 1) >> 1;
        if (bl.tile_prefix[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const ViewDesc* v = &bl.views[bl.active[lo]];
    int local = t - bl.tile_prefix[lo];
    *tx = local % v->tiles_x;
    *ty = local / v->tiles_x;
    return v;
}

// Reference window source: rows [y0-r, y0+TILE_H+r), cols [x0-r, x0+TILE_W+r),
// clamped to the image edge like the reference's clamp-addressed texel fetches
// (patchmatch_mvs.cu:275-276, :371-380).
__device__ __forceinline__ void load_ref_tile(float* s_ref, int tw, int th, const ViewDesc* v, int x0, int y0,
                                              int r) {
    const int W = v->W, H = v->H;
    for (int i = threadIdx.x; i < tw * th; i += CTA_THREADS) {
        int ty = i / tw, tx = i - ty * tw;
        int gx = min(max(x0 - r + tx, 0), W - 1);
        int gy = min(max(y0 - r + ty, 0), H - 1);
        s_ref[i] = __ldg(v->ref + static_cast<size_t>(gy) * v->ref_pitch + gx);
    }
}

// Approximate reciprocal (PTX rcp.approx.ftz.f32): the instruction the
// reference's fast-math build uses for 1.0f / w_z.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Cost of hypothesis (d, n) at pixel (x, y): per-source NCC over the window,
// top_k lowest of (1 - NCC) averaged (computePixelCost, :222-343).
//
// Per tap the warp arithmetic is pinned with explicitly rounded intrinsics to
// the operation sequence the reference compiles to (found by a bit-exact
// search against its kernels on B200):
//   q = fma(a0, x, a1*y) + a2,  f = s * inv(n.P),  w_z = fma(b2, f, q_z),
//   u = fma(b0, f, q_x) * rcp(w_z),  sums accumulated with fma in tap order.
// Because nothing is left to the compiler's reassociation, the taps can be
// restructured for throughput: each window row issues all its texture
// fetches before consuming any (SIDE fetches in flight per thread), the
// row-invariant products a1*y are computed once per row (the same rounded
// value), and samples are accumulated in tap order, skipping invalid taps
// exactly as the reference's `continue`s do.
template <int R, int ST>
__device__ __forceinline__ float cost_f32(const float* __restrict__ s_ref, int tw, int lx, int ly, int x, int y,
                                          float d, float cnx, float cny, float cnz, const ViewDesc* __restrict__ v,
                                          int topk) {
    constexpr int SIDE = (2 * R) / ST + 1;
    const float ki0 = v->kinv[0], ki1 = v->kinv[1], ki2 = v->kinv[2];
    const float ki3 = v->kinv[3], ki4 = v->kinv[4], ki5 = v->kinv[5];
    const float ki6 = v->kinv[6], ki7 = v->kinv[7], ki8 = v->kinv[8];
    const float fx = static_cast<float>(x);
    const float fy = static_cast<float>(y);
    // Plane through P = d K^-1 [x y 1] with normal n; nK = K^-T n.
    const float Px = d * (ki0 * fx + ki1 * fy + ki2);
    const float Py = d * (ki3 * fx + ki4 * fy + ki5);
    const float Pz = d * (ki6 * fx + ki7 * fy + ki8);
    const float n_dot_P = cnx * Px + cny * Py + cnz * Pz;
    if (fabsf(n_dot_P) < 1e-8f) return 2.0f;
    const float inv_n_dot_P = 1.0f / n_dot_P;
    const float nK0 = ki0 * cnx + ki3 * cny + ki6 * cnz;
    const float nK1 = ki1 * cnx + ki4 * cny + ki7 * cnz;
    const float nK2 = ki2 * cnx + ki5 * cny + ki8 * cnz;
    constexpr int min_count = (SIDE * SIDE) / 2;
    const float fw1 = static_cast<float>(v->W) - 1.0f;
    const float fh1 = static_cast<float>(v->H) - 1.0f;

    float top[3] = {2.0f, 2.0f, 2.0f};
    const int S = v->S;
    for (int s = 0; s < S; ++s) {
        const float* A = v->ab[s];
        const float a0 = A[0], a1 = A[1], a2 = A[2], a3 = A[3], a4 = A[4], a5 = A[5];
        const float a6 = A[6], a7 = A[7], a8 = A[8], b0 = A[9], b1 = A[10], b2 = A[11];
        const cudaTextureObject_t tex = v->src_tex[s];
        float sum_ref = 0.0f, sum_src = 0.0f, sum_ref2 = 0.0f, sum_src2 = 0.0f, sum_rs = 0.0f;
        int count = 0;
        // A window whose warp lies wholly beyond one edge of the source has no
        // valid tap, so the reference's count rule gives 2 for this source:
        // skip its taps.  The test runs on the plane-induced homography
        // H = A + b (K^-T n)^T / (n.P) at the window's corners, in front of
        // the camera (w_z > 1e-6, so the warped window is the convex quad of
        // its corners) and past the edge by 0.25 px, far above the rounding
        // differences between this and the per-tap arithmetic below.
        {
            const float m0 = nK0 * inv_n_dot_P, m1 = nK1 * inv_n_dot_P, m2 = nK2 * inv_n_dot_P;
            const float hz0 = fmaf(b2, m0, a6), hz1 = fmaf(b2, m1, a7), hz2 = fmaf(b2, m2, a8);
            const float hx0 = fmaf(b0, m0, a0), hx1 = fmaf(b0, m1, a1), hx2 = fmaf(b0, m2, a2);
            const float hy0 = fmaf(b1, m0, a3), hy1 = fmaf(b1, m1, a4), hy2 = fmaf(b1, m2, a5);
            bool front = true, left = true, right = true, top_ = true, bottom = true;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const float px = fx + static_cast<float>((c & 1) ? (SIDE - 1) * ST - R : -R);
                const float py = fy + static_cast<float>((c & 2) ? (SIDE - 1) * ST - R : -R);
                const float wz = fmaf(hz0, px, fmaf(hz1, py, hz2));
                const float wx = fmaf(hx0, px, fmaf(hx1, py, hx2));
                const float wy = fmaf(hy0, px, fmaf(hy1, py, hy2));
                front = front && wz > 1e-6f;
                left = left && wx < -0.25f * wz;
                right = right && wx >= (fw1 + 0.25f) * wz;
                top_ = top_ && wy < -0.25f * wz;
                bottom = bottom && wy >= (fh1 + 0.25f) * wz;
            }
            // Cost 2 would change nothing in the running top-3 (every entry is <= 2).
            if (front && (left || right || top_ || bottom)) continue;
        }
#ifdef HP_COUNT_TAPS
        atomicAdd(&g_taps32, static_cast<unsigned long long>(SIDE * SIDE));
#endif
#pragma unroll 1
        for (int i = 0; i < SIDE; ++i) {
            const float wpy = fy + static_cast<float>(i * ST - R);
            const float tqx = __fmul_rn(a1, wpy), tqy = __fmul_rn(a4, wpy), tqz = __fmul_rn(a7, wpy);
            const float tsv = __fmul_rn(nK1, wpy);
            float smp[SIDE];
            unsigned ok = 0;
#pragma unroll
            for (int j = 0; j < SIDE; ++j) {
                const float wpx = fx + static_cast<float>(j * ST - R);
                const float qx = __fadd_rn(__fmaf_rn(a0, wpx, tqx), a2);
                const float qy = __fadd_rn(__fmaf_rn(a3, wpx, tqy), a5);
                const float qz = __fadd_rn(__fmaf_rn(a6, wpx, tqz), a8);
                const float sval = __fadd_rn(__fmaf_rn(nK0, wpx, tsv), nK2);
                const float factor = __fmul_rn(sval, inv_n_dot_P);
                const float wz = __fmaf_rn(b2, factor, qz);
                const float iw = rcp_approx(wz);
                const float u = __fmul_rn(__fmaf_rn(b0, factor, qx), iw);
                const float vv = __fmul_rn(__fmaf_rn(b1, factor, qy), iw);
                const bool skip = fabsf(wz) < 1e-8f || u < 0.0f || u >= fw1 || vv < 0.0f || vv >= fh1;
                ok |= static_cast<unsigned>(!skip) << j;
                smp[j] = tex2D<float>(tex, __fadd_rn(u, 0.5f), __fadd_rn(vv, 0.5f));
            }
            const float* rrow = s_ref + (ly + i * ST) * tw + lx;
#pragma unroll
            for (int j = 0; j < SIDE; ++j) {
                if (ok & (1u << j)) {
                    const float rv = rrow[j * ST];
                    const float sv = smp[j];
                    sum_ref = __fadd_rn(sum_ref, rv);
                    sum_src = __fadd_rn(sum_src, sv);
                    sum_ref2 = __fmaf_rn(rv, rv, sum_ref2);
                    sum_src2 = __fmaf_rn(sv, sv, sum_src2);
                    sum_rs = __fmaf_rn(rv, sv, sum_rs);
                    count++;
                }
            }
        }
        float c;
        if (count < min_count) {
            c = 2.0f;
        } else {
            const float fc = static_cast<float>(count);
            const float num = fc * sum_rs - sum_ref * sum_src;
            const float den_r = fc * sum_ref2 - sum_ref * sum_ref;
            const float den_s = fc * sum_src2 - sum_src * sum_src;
            if (den_r < 1e-6f || den_s < 1e-6f) {
                c = 2.0f;
            } else {
                float ncc = num / (sqrtf(den_r) * sqrtf(den_s));
                ncc = fmaxf(-1.0f, fminf(1.0f, ncc));
                c = 1.0f - ncc;
            }
        }
        // Sorted insert into the running top-3 (lowest first).
        if (c < top[2]) {
            top[2] = c;
#pragma unroll
            for (int i = 1; i >= 0; --i) {
                if (top[i + 1] < top[i]) {
                    const float t = top[i];
                    top[i] = top[i + 1];
                    top[i + 1] = t;
                } else {
                    break;
                }
            }
        }
    }
    const int k = min(topk, S);
    float sum = 0.0f;
    for (int i = 0; i < k; ++i) sum += top[i];
    return sum / static_cast<float>(k);
}

__device__ __forceinline__ bool same_plane(float4 a, float4 b) {
    return __float_as_uint(a.x) == __float_as_uint(b.x) && __float_as_uint(a.y) == __float_as_uint(b.y) &&
           __float_as_uint(a.z) == __float_as_uint(b.z) && __float_as_uint(a.w) == __float_as_uint(b.w);
}

__global__ void __launch_bounds__(256) init_kernel(BatchList bl) {
    int tile_x, tile_y;
    const ViewDesc* v = locate_tile(bl, blockIdx.x, &tile_x, &tile_y);
    tile_init(v, tile_x, tile_y);
}

// Full-map cost of the current hypotheses of one tile (compute_ncc_cost_kernel,
// patchmatch_mvs.cu:349-513).  Each thread owns a horizontal pixel pair.
template <int R, int ST>
__device__ __forceinline__ void tile_cost(const ViewDesc* v, int tile_x, int tile_y, const SolveConsts& sc,
                                          float* s_ref) {
    constexpr int tw = TILE_W + 2 * R, th = TILE_H + 2 * R;
    const int x0 = tile_x * TILE_W, y0 = tile_y * TILE_H;
    load_ref_tile(s_ref, tw, th, v, x0, y0, R);
    __syncthreads();
    const int ly = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = y0 + ly;
    if (y >= v->H) return;
    for (int j = 0; j < 2; ++j) {
        const int lx = 2 * lane + j, x = x0 + lx;
        if (x >= v->W) continue;
        const size_t idx = static_cast<size_t>(y) * v->W + x;
        const float4 h = v->hyp[idx];
        v->cost[idx] = cost_f32<R, ST>(s_ref, tw, lx, ly, x, y, h.x, h.y, h.z, h.w, v, sc.top_k);
    }
}

template <int R, int ST>
__global__ void __launch_bounds__(CTA_THREADS, HP_F32_MIN_BLOCKS) cost_kernel(BatchList bl, SolveConsts sc) {
    __shared__ float s_ref[MAX_TW * MAX_TH];
    int tile_x, tile_y;
    const ViewDesc* v = locate_tile(bl, blockIdx.x, &tile_x, &tile_y);
    tile_cost<R, ST>(v, tile_x, tile_y, sc, s_ref);
}

// One red-black half-pass (propagate_and_refine_kernel, patchmatch_mvs.cu:519-655).
// Thread (ly, lane) owns pixel x0 + 2*lane + ((y + color) & 1) of row y0 + ly:
// every thread has work, where the reference idles half its grid.
//
// Neighbour phase (L, R, U, D; :551-580), compacted per warp.  Each lane lists
// the neighbour planes it must score: in range, and not bit-identical to its
// current plane or to an earlier listed neighbour (such a candidate cannot win:
// same pixel, same plane, same arithmetic, same cost).  Lanes skip different
// candidates, so scoring them lane by lane would leave warps half idle while
// every texture instruction still costs nearly a full warp's worth of filter
// throughput.  Instead the CTA's eight warps write the union of their (pixel,
// neighbour) items to one list in shared memory and score it 32 items at a
// time (warp w takes items [32 (w + 8 k), 32 (w + 8 k) + 32)), each cost
// landing in its owner's slot; then each owner folds its costs in L, R, U, D
// order with the same strict-less rule - the result is that of the
// sequential loop.  The refinement perturbations
// (:583-648) follow per lane: every lane has exactly refine_steps of them.
constexpr int WARPS = CTA_THREADS / 32;

// Shared memory of the half-pass beyond the reference tile.
struct PassSmem {
    float cost[WARPS][32 * 4];          // neighbour cost, slot (lane << 2 | cand) of the owner's warp
    unsigned short items[WARPS * 128];  // CTA item list: warp << 7 | lane << 2 | cand
    int warp_total[WARPS];
};

template <int R, int ST>
__device__ __forceinline__ void tile_propagate(const ViewDesc* v, int tile_x, int tile_y, const SolveConsts& sc,
                                               int iteration, int color, float* s_ref, PassSmem& sm) {
    constexpr int tw = TILE_W + 2 * R, th = TILE_H + 2 * R;
    const int x0 = tile_x * TILE_W, y0 = tile_y * TILE_H;
    load_ref_tile(s_ref, tw, th, v, x0, y0, R);
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

    float4 best = make_float4(0.f, 0.f, 0.f, 0.f);
    float best_cost = 0.f;
    unsigned need = 0;
    if (active) {
        best = v->hyp[idx];
        best_cost = v->cost[idx];
#pragma unroll
        for (int cand = 0; cand < 4; ++cand) {
            const int nxp = x + (cand == 0 ? -1 : (cand == 1 ? 1 : 0));
            const int nyp = y + (cand == 2 ? -1 : (cand == 3 ? 1 : 0));
            if (nxp < 0 || nxp >= W || nyp < 0 || nyp >= H) continue;
            const float4 h = v->hyp[static_cast<size_t>(nyp) * W + nxp];
            if (h.x < dmin || h.x > dmax) continue;
            bool dup = same_plane(h, best);
            for (int j = 0; j < cand && !dup; ++j) {
                if (need & (1u << j)) {
                    const int jx = x + (j == 0 ? -1 : (j == 1 ? 1 : 0));
                    const int jy = y + (j == 2 ? -1 : (j == 3 ? 1 : 0));
                    dup = same_plane(h, v->hyp[static_cast<size_t>(jy) * W + jx]);
                }
            }
            if (!dup) need |= 1u << cand;
        }
    }
    // Exclusive scan of the item counts over the warp, then over the CTA's warps; owners write their items.
    const int cnt = __popc(need);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) sm.warp_total[ly] = incl;
    __syncthreads();
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
    __syncthreads();
    for (int base = ly * 32; base < total; base += CTA_THREADS) {
        const int w = base + lane;
        if (w < total) {
            const int item = sm.items[w];
            const int oly = item >> 7, owner = (item >> 2) & 31, cand = item & 3;
            const int oy = y0 + oly, olx = 2 * owner + ((oy + color) & 1), ox = x0 + olx;
            const int nxp = ox + (cand == 0 ? -1 : (cand == 1 ? 1 : 0));
            const int nyp = oy + (cand == 2 ? -1 : (cand == 3 ? 1 : 0));
            const float4 h = v->hyp[static_cast<size_t>(nyp) * W + nxp];
            sm.cost[oly][item & 127] = cost_f32<R, ST>(s_ref, tw, olx, oly, ox, oy, h.x, h.y, h.z, h.w, v, sc.top_k);
        }
    }
    __syncthreads();
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

    // Random refinement around the running best.
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
        const float c = cost_f32<R, ST>(s_ref, tw, lx, ly, x, y, cd, cn.x, cn.y, cn.z, v, sc.top_k);
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

template <int R, int ST>
__global__ void __launch_bounds__(CTA_THREADS, HP_F32_MIN_BLOCKS) propagate_kernel(BatchList bl, SolveConsts sc,
                                                                                   int iteration, int color) {
    __shared__ float s_ref[MAX_TW * MAX_TH];
    __shared__ PassSmem sm;
    int tile_x, tile_y;
    const ViewDesc* v = locate_tile(bl, blockIdx.x, &tile_x, &tile_y);
    tile_propagate<R, ST>(v, tile_x, tile_y, sc, iteration, color, s_ref, sm);
}

// Persistent form: one launch runs every stage of every view of a solve
// (see Schedule), each CTA taking tiles until the tickets run out.  The stage
// bodies are the functions the per-stage kernels above run, so the results
// are bit-identical to the per-stage launch sequence.
template <int R, int ST>
__global__ void __launch_bounds__(CTA_THREADS, HP_F32_MIN_BLOCKS) persistent_kernel(Schedule s) {
    __shared__ float s_ref[MAX_TW * MAX_TH];
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
            tile_cost<R, ST>(v, tx, ty, s.sc, s_ref);
        } else if (stage <= 2 * v->iterations) {
            const int k = stage - 1;
            tile_propagate<R, ST>(v, tx, ty, s.sc, k >> 1, k & 1, s_ref, sm);
        } else if (is_filter_stage(v, stage)) {
            tile_filter(s.views, v, tx, ty, true);  // geometric check, then the maps
        } else {
            tile_unpack(v, tx, ty);
        }
        __syncthreads();
        if (threadIdx.x == 0) sched_publish(s, s_tile);
    }
}

template <int R, int ST>
cudaError_t launch_rs(const BatchList& bl, const SolveConsts& sc, int iteration, int color, bool full,
                      cudaStream_t st) {
    if (full)
        cost_kernel<R, ST><<<bl.total_tiles, CTA_THREADS, 0, st>>>(bl, sc);
    else
        propagate_kernel<R, ST><<<bl.total_tiles, CTA_THREADS, 0, st>>>(bl, sc, iteration, color);
    return cudaGetLastError();
}

cudaError_t dispatch_f32(const BatchList& bl, const SolveConsts& sc, int iteration, int color, bool full,
                         cudaStream_t st) {
    if (bl.total_tiles <= 0) return cudaSuccess;
    if (sc.stride != 1 && sc.stride != 2) return cudaErrorInvalidValue;
#define HP_CASE(RR)                                                                  \
    case RR:                                                                         \
        return sc.stride == 1 ? launch_rs<RR, 1>(bl, sc, iteration, color, full, st) \
                              : launch_rs<RR, 2>(bl, sc, iteration, color, full, st);
    switch (sc.radius) {
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

template <int R, int ST>
cudaError_t persistent_rs(const Schedule& s, int grid, cudaStream_t st, int* occ) {
    if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, persistent_kernel<R, ST>, CTA_THREADS, 0);
    persistent_kernel<R, ST><<<grid, CTA_THREADS, 0, st>>>(s);
    return cudaGetLastError();
}

cudaError_t persistent_dispatch(int radius, int stride, const Schedule* s, int grid, cudaStream_t st, int* occ) {
    if (stride != 1 && stride != 2) return cudaErrorInvalidValue;
#define HP_CASE(RR)                                                                              \
    case RR:                                                                                     \
        return stride == 1 ? persistent_rs<RR, 1>(*s, grid, st, occ) : persistent_rs<RR, 2>(*s, grid, st, occ);
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

}  // namespace

cudaError_t launch_persistent_f32(const Schedule& s, int grid, cudaStream_t st) {
    if (s.total <= 0 || grid <= 0) return cudaSuccess;
    Schedule k = s;
    if (!k.abort) k.abort = k.status + 1;
    return persistent_dispatch(k.sc.radius, k.sc.stride, &k, grid, st, nullptr);
}

cudaError_t persistent_occupancy_f32(int radius, int stride, int* blocks_per_sm) {
    Schedule dummy{};
    return persistent_dispatch(radius, stride, &dummy, 0, nullptr, blocks_per_sm);
}

cudaError_t launch_init(const BatchList& bl, int tile_h, cudaStream_t st) {
    if (bl.total_tiles <= 0) return cudaSuccess;
    init_kernel<<<bl.total_tiles, 32 * tile_h, 0, st>>>(bl);
    return cudaGetLastError();
}

cudaError_t launch_cost_f32(const BatchList& bl, const SolveConsts& sc, cudaStream_t st) {
    return dispatch_f32(bl, sc, 0, 0, true, st);
}

cudaError_t launch_propagate_f32(const BatchList& bl, const SolveConsts& sc, int iteration, int color,
                                 cudaStream_t st) {
    return dispatch_f32(bl, sc, iteration, color, false, st);
}

}  // namespace hp
