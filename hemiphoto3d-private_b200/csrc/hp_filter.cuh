// Geometric-consistency check, device side (the rule of
// geometric_consistency_filter_kernel, src/dense_recon/patchmatch_mvs.cu:668-781,
// with this engine's own arithmetic; see FilterSource for the transforms).
//
// A reference pixel keeps its depth when at least min_consistent sources
// agree: the point lands in front of the source, inside it at the nearest
// pixel, that pixel holds a positive depth within depth_tol (relative to the
// point's source-camera depth), and the two world-frame normals have a cosine
// of at least normal_cos.  Otherwise its depth becomes 0 and its cost 2
// (confidence 0).  Every float operation is an explicitly rounded intrinsic,
// so the result does not depend on the including translation unit's flags:
// the fused stage (per-pass kernel, both persistent kernels) and the
// external-maps kernel give the same bits on the same inputs.
#pragma once

#include "hp_internal.h"

namespace hp {

// Number of sources that agree with the plane (d, n) at pixel (x, y).
// fetch(s, i) returns the source's (depth, camera-frame normal) at element i.
template <class Fetch>
__device__ __forceinline__ int filter_agreeing(const FilterStage* __restrict__ f, int W, int H, int x, int y,
                                               float d, float nx, float ny, float nz, Fetch fetch) {
    const float fx = static_cast<float>(x), fy = static_cast<float>(y);
    const int n = f->n;
    int agree = 0;
    for (int s = 0; s < n; ++s) {
        const FilterSource& q = f->src[s];
        const float z = __fmaf_rn(d, __fmaf_rn(q.m[0], fx, __fmaf_rn(q.m[1], fy, q.m[2])), q.cz);
        if (!(z > 0.0f)) continue;  // behind the source camera
        const float px = __fmaf_rn(d, __fmaf_rn(q.A[0], fx, __fmaf_rn(q.A[1], fy, q.A[2])), q.b[0]);
        const float py = __fmaf_rn(d, __fmaf_rn(q.A[3], fx, __fmaf_rn(q.A[4], fy, q.A[5])), q.b[1]);
        const float pz = __fmaf_rn(d, __fmaf_rn(q.A[6], fx, __fmaf_rn(q.A[7], fy, q.A[8])), q.b[2]);
        // Nearest source pixel (ties to even); NaN and overflow land out of range.
        const int ui = __float2int_rn(__fdiv_rn(px, pz));
        const int vi = __float2int_rn(__fdiv_rn(py, pz));
        if (ui < 0 || ui >= W || vi < 0 || vi >= H) continue;
        const float4 o = fetch(s, static_cast<size_t>(vi) * W + ui);
        if (!(o.x > 0.0f)) continue;  // no depth there (never solved, or filtered out)
        if (__fdiv_rn(fabsf(__fsub_rn(o.x, z)), z) > f->depth_tol) continue;
        const float rx = __fmaf_rn(q.Rn[0], nx, __fmaf_rn(q.Rn[1], ny, __fmul_rn(q.Rn[2], nz)));
        const float ry = __fmaf_rn(q.Rn[3], nx, __fmaf_rn(q.Rn[4], ny, __fmul_rn(q.Rn[5], nz)));
        const float rz = __fmaf_rn(q.Rn[6], nx, __fmaf_rn(q.Rn[7], ny, __fmul_rn(q.Rn[8], nz)));
        if (__fmaf_rn(rx, o.y, __fmaf_rn(ry, o.z, __fmul_rn(rz, o.w))) < f->normal_cos) continue;
        ++agree;
    }
    return agree;
}

// The filter stage of one tile of view v (a CTA of v->tile_h warps, one per
// tile row, two pixels a thread), in place on its packed state.  The
// sources' state is read through L2 (ld.global.cg): in a persistent launch it
// may have been written by other CTAs since this SM last cached it.  With
// write_out the tile's final maps go to v's out_* pointers too (the unpack).
__device__ __forceinline__ void tile_filter(const ViewDesc* __restrict__ views, const ViewDesc* __restrict__ v,
                                            int tile_x, int tile_y, bool write_out) {
    const int ly = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = tile_y * v->tile_h + ly;
    if (y >= v->H) return;
    const FilterStage* f = v->filter;
    const int W = v->W, H = v->H;
    auto fetch = [&](int s, size_t i) { return __ldcg(views[f->src[s].view].hyp + i); };
    for (int j = 0; j < 2; ++j) {
        const int x = tile_x * TILE_W + j * 32 + lane;
        if (x >= W) continue;
        const size_t i = static_cast<size_t>(y) * W + x;
        float4 h = __ldcg(v->hyp + i);
        float c = __ldcg(v->cost + i);
        const bool keep = h.x > 0.0f && filter_agreeing(f, W, H, x, y, h.x, h.y, h.z, h.w, fetch) >= f->min_consistent;
        if (!keep) {
            if (h.x > 0.0f) {
                h.x = 0.0f;
                v->hyp[i] = h;
            }
            c = 2.0f;
            v->cost[i] = c;
        }
        if (write_out) {
            v->out_depth[i] = h.x;
            v->out_normal[3 * i] = h.y;
            v->out_normal[3 * i + 1] = h.z;
            v->out_normal[3 * i + 2] = h.w;
            v->out_cost[i] = c;
            if (v->out_conf) v->out_conf[i] = __fsub_rn(1.0f, __fmul_rn(c, 0.5f));
        }
    }
}

}  // namespace hp
