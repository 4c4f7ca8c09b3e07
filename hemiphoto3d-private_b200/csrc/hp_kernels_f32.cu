// Plain FP32 PatchMatch kernels for sm_100a: hypothesis initialisation, full-map
// NCC cost, and the fused red-black propagate + refine pass.
//
// Parity contract.  The reference's cost (computePixelCost,
// src/dense_recon/patchmatch_mvs.cu:222-343) samples sources through the
// texture unit's linear filter, whose weights carry only 8 fractional bits; a
// warped coordinate that moves by one ulp can flip a weight by 1/256 and the
// cost by ~1e-5.  To hold the 1e-5 bound this file keeps the reference's
// per-tap arithmetic - the same expressions in the same order, built with the
// reference's --use_fast_math - and samples sources with tex2D on the same
// filter configuration.  Everything around the taps is this engine's own:
// packed float4 hypotheses, a shared-memory reference tile, red-black
// compaction (every thread owns a pixel of the active color), duplicate-
// candidate elimination, batched multi-view launches and counter-based RNG.
// Engine-defined arithmetic outside the taps uses explicitly rounded
// intrinsics so the CPU restatement reproduces it bit for bit.
#include "hp_internal.h"
#include "hp_rng.cuh"

namespace hp {

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

// Cost of hypothesis (d, n) at pixel (x, y): per-source NCC over the window,
// top_k lowest of (1 - NCC) averaged.  One out-of-line body so the full-map
// kernel and the propagate kernel round identically.  The sampling stride ST
// is a compile-time constant: with a run-time stride the fast-math build
// reassociates the warp arithmetic differently from the reference's unit-
// stride loop and ~30% of costs move by an ulp-driven 1e-5; with ST = 1 the
// loop has the reference's shape and the costs are bit-identical to it.
template <int ST>
__device__ __noinline__ float cost_f32(const float* __restrict__ s_ref, int tw, int lx, int ly, int x, int y,
                                       float d, float cnx, float cny, float cnz, const ViewDesc* __restrict__ v,
                                       int r, int topk) {
    constexpr int st = ST;
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

    const int side = (2 * r) / st + 1;
    const int min_count = (side * side) / 2;
    const float fwidth = static_cast<float>(v->W);
    const float fheight = static_cast<float>(v->H);

    // Loop shape, coefficient reads and the top-k array are kept as the
    // reference writes them: the fast-math build then rounds every tap exactly
    // as the reference does (verified bit-for-bit on the GPU).
    float top[3] = {2.0f, 2.0f, 2.0f};
    const int S = v->S;
    for (int s = 0; s < S; ++s) {
        const float* A = v->ab[s];
        float sum_ref = 0.0f, sum_src = 0.0f, sum_ref2 = 0.0f, sum_src2 = 0.0f, sum_rs = 0.0f;
        int count = 0;
        for (int dy = -r; dy <= r; dy += st) {
            for (int dx = -r; dx <= r; dx += st) {
                const float ref_val = s_ref[(ly + r + dy) * tw + (lx + r + dx)];
                const float wpx = fx + static_cast<float>(dx);
                const float wpy = fy + static_cast<float>(dy);
                const float qx = A[0] * wpx + A[1] * wpy + A[2];
                const float qy = A[3] * wpx + A[4] * wpy + A[5];
                const float qz = A[6] * wpx + A[7] * wpy + A[8];
                const float sval = nK0 * wpx + nK1 * wpy + nK2;
                const float factor = sval * inv_n_dot_P;
                const float wz = qz + A[11] * factor;
                if (fabsf(wz) < 1e-8f) continue;
                const float inv_wz = 1.0f / wz;
                const float src_u = (qx + A[9] * factor) * inv_wz;
                const float src_v = (qy + A[10] * factor) * inv_wz;
                if (src_u < 0.0f || src_u >= fwidth - 1.0f || src_v < 0.0f || src_v >= fheight - 1.0f) continue;
                const float src_val = tex2D<float>(v->src_tex[s], src_u + 0.5f, src_v + 0.5f);
                sum_ref += ref_val;
                sum_src += src_val;
                sum_ref2 += ref_val * ref_val;
                sum_src2 += src_val * src_val;
                sum_rs += ref_val * src_val;
                count++;
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

// --------------------------------------------------------------------------
// Initial hypotheses: depth uniform in [dmin, dmax]; normal from theta in
// [0, 2pi) and cos(phi) in (0, 1), flipped to face the camera, normalised
// (init_depth_normal_kernel, patchmatch_mvs.cu:164-216).
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(CTA_THREADS) init_kernel(BatchList bl) {
    int tile_x, tile_y;
    const ViewDesc* v = locate_tile(bl, blockIdx.x, &tile_x, &tile_y);
    const int ly = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = tile_y * TILE_H + ly;
    if (y >= v->H) return;
    for (int j = 0; j < 2; ++j) {
        const int x = tile_x * TILE_W + j * 32 + lane;
        if (x >= v->W) continue;
        const uint32_t idx = static_cast<uint32_t>(y * v->W + x);
        const uint4 r = philox4x32_10(make_uint4(idx, v->view_id, 0u, 0u), v->seed_lo, v->seed_hi);
        const float depth = __fmaf_rn(u01(r.x), __fsub_rn(v->dmax, v->dmin), v->dmin);
        const float3 ray = view_ray(v->kinv, x, y);
        float st, ct;
        sincos_2pi(u01(r.y), &st, &ct);
        const float cp = u01(r.z);
        const float sp = __fsqrt_rn(fmaxf(0.0f, __fmaf_rn(-cp, cp, 1.0f)));
        float3 n = make_float3(__fmul_rn(sp, ct), __fmul_rn(sp, st), cp);
        if (dot3_rn(n, ray) > 0.0f) n = make_float3(-n.x, -n.y, -n.z);
        n = normalize3_rn(n.x, n.y, n.z);
        v->hyp[idx] = make_float4(depth, n.x, n.y, n.z);
    }
}

// Full-map cost of the current hypotheses (compute_ncc_cost_kernel,
// patchmatch_mvs.cu:349-513).  Each thread owns a horizontal pixel pair.
template <int ST>
__global__ void __launch_bounds__(CTA_THREADS) cost_kernel(BatchList bl, SolveConsts sc) {
    __shared__ float s_ref[MAX_TW * MAX_TH];
    int tile_x, tile_y;
    const ViewDesc* v = locate_tile(bl, blockIdx.x, &tile_x, &tile_y);
    const int r = sc.radius, tw = TILE_W + 2 * r, th = TILE_H + 2 * r;
    const int x0 = tile_x * TILE_W, y0 = tile_y * TILE_H;
    load_ref_tile(s_ref, tw, th, v, x0, y0, r);
    __syncthreads();
    const int ly = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = y0 + ly;
    if (y >= v->H) return;
    for (int j = 0; j < 2; ++j) {
        const int lx = 2 * lane + j, x = x0 + lx;
        if (x >= v->W) continue;
        const size_t idx = static_cast<size_t>(y) * v->W + x;
        const float4 h = v->hyp[idx];
        v->cost[idx] = cost_f32<ST>(s_ref, tw, lx, ly, x, y, h.x, h.y, h.z, h.w, v, r, sc.top_k);
    }
}

// One red-black half-pass (propagate_and_refine_kernel, patchmatch_mvs.cu:519-655).
// Thread (ly, lane) owns pixel x0 + 2*lane + ((y + color) & 1) of row y0 + ly:
// every thread has work, where the reference idles half its grid.
template <int ST>
__global__ void __launch_bounds__(CTA_THREADS) propagate_kernel(BatchList bl, SolveConsts sc, int iteration,
                                                                int color) {
    __shared__ float s_ref[MAX_TW * MAX_TH];
    int tile_x, tile_y;
    const ViewDesc* v = locate_tile(bl, blockIdx.x, &tile_x, &tile_y);
    const int r = sc.radius, tw = TILE_W + 2 * r, th = TILE_H + 2 * r;
    const int x0 = tile_x * TILE_W, y0 = tile_y * TILE_H;
    load_ref_tile(s_ref, tw, th, v, x0, y0, r);
    __syncthreads();
    const int W = v->W, H = v->H;
    const int ly = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = y0 + ly;
    const int lx = 2 * lane + ((y + color) & 1);
    const int x = x0 + lx;
    if (y >= H || x >= W) return;
    const size_t idx = static_cast<size_t>(y) * W + x;
    const float dmin = v->dmin, dmax = v->dmax;

    float4 best = v->hyp[idx];
    float best_cost = v->cost[idx];

    // Neighbour hypotheses, left, right, up, down (patchmatch_mvs.cu:551-580).
    // A candidate bit-identical to the current best or to one already tried
    // at this visit cannot win (its cost is the same number), so it is skipped.
    float4 tried[4];
    int n_tried = 0;
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        const int nxp = x + (n == 0 ? -1 : (n == 1 ? 1 : 0));
        const int nyp = y + (n == 2 ? -1 : (n == 3 ? 1 : 0));
        if (nxp < 0 || nxp >= W || nyp < 0 || nyp >= H) continue;
        const float4 h = v->hyp[static_cast<size_t>(nyp) * W + nxp];
        if (h.x < dmin || h.x > dmax) continue;
        bool dup = same_plane(h, best);
#pragma unroll
        for (int j = 0; j < 4; ++j) dup |= (j < n_tried) && same_plane(h, tried[j]);
        if (dup) continue;
        tried[n_tried++] = h;
        const float c = cost_f32<ST>(s_ref, tw, lx, ly, x, y, h.x, h.y, h.z, h.w, v, r, sc.top_k);
        if (c < best_cost) {
            best_cost = c;
            best = h;
        }
    }

    // Random refinement around the running best (patchmatch_mvs.cu:583-648).
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
        const float c = cost_f32<ST>(s_ref, tw, lx, ly, x, y, cd, cn.x, cn.y, cn.z, v, r, sc.top_k);
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

}  // namespace

cudaError_t launch_init(const BatchList& bl, cudaStream_t st) {
    if (bl.total_tiles <= 0) return cudaSuccess;
    init_kernel<<<bl.total_tiles, CTA_THREADS, 0, st>>>(bl);
    return cudaGetLastError();
}

cudaError_t launch_cost_f32(const BatchList& bl, const SolveConsts& sc, cudaStream_t st) {
    if (bl.total_tiles <= 0) return cudaSuccess;
    if (sc.stride == 1)
        cost_kernel<1><<<bl.total_tiles, CTA_THREADS, 0, st>>>(bl, sc);
    else if (sc.stride == 2)
        cost_kernel<2><<<bl.total_tiles, CTA_THREADS, 0, st>>>(bl, sc);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_propagate_f32(const BatchList& bl, const SolveConsts& sc, int iteration, int color,
                                 cudaStream_t st) {
    if (bl.total_tiles <= 0) return cudaSuccess;
    if (sc.stride == 1)
        propagate_kernel<1><<<bl.total_tiles, CTA_THREADS, 0, st>>>(bl, sc, iteration, color);
    else if (sc.stride == 2)
        propagate_kernel<2><<<bl.total_tiles, CTA_THREADS, 0, st>>>(bl, sc, iteration, color);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace hp
