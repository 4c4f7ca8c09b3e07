// Depth-map fusion into a dense point cloud (hp_fuse_depth_maps).
//
// The reference declares the stage's consumer, fuseDepthMaps(depth_maps,
// poses, images) -> DensePointCloud (src/dense_recon/point_cloud.h:7), and
// leaves it a stub (src/dense_recon/point_cloud.cu:4-8).  The rule fused here
// is stated in include/hpmvs.h: a pixel's back-projected point is checked in
// each neighbour view for depth, reprojection and normal agreement, the mean
// of the agreeing points is emitted once, by the lowest-index view that sees
// it.
//
// One thread per pixel of every view; the maps stay where the solve left them
// and neighbours are gathered straight from them.  The output is compacted in
// (view, row, column) order without atomics: a counting pass writes each
// CTA's number of points, one CTA scans those counts, and a writing pass
// recomputes its pixels and stores each point at its CTA's offset plus its
// rank in the CTA.  Every operation is an explicitly rounded intrinsic (no
// contraction into FMAs the source does not spell out), so the CPU oracle's
// plain-C restatement gives the same bits.
#include "hp_internal.h"

namespace hp {

namespace {

struct Fused {
    float px, py, pz, nx, ny, nz, c;
};

__device__ __forceinline__ int fuse_view_of(const FuseArgs& a, int block) {
    int lo = 0, hi = a.n_views - 1;
    while (lo < hi) {  // last view whose first CTA is at or before `block`
        const int mid = (lo + hi + 1) >> 1;
        if (a.view_block[mid] <= block) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// R^T (x, y, z): a camera-frame direction in the world frame.
__device__ __forceinline__ float3 rot_to_world(const float* R, float x, float y, float z) {
    return make_float3(__fmaf_rn(R[0], x, __fmaf_rn(R[3], y, __fmul_rn(R[6], z))),
                       __fmaf_rn(R[1], x, __fmaf_rn(R[4], y, __fmul_rn(R[7], z))),
                       __fmaf_rn(R[2], x, __fmaf_rn(R[5], y, __fmul_rn(R[8], z))));
}

// Pixel (fx, fy) of view v at depth d, in the world frame: R^T (d K^-1 [x y 1] - t).
__device__ __forceinline__ float3 to_world(const FuseView& v, float fx, float fy, float d) {
    const float* k = v.kinv;
    const float cx = __fmul_rn(d, __fmaf_rn(k[0], fx, __fmaf_rn(k[1], fy, k[2])));
    const float cy = __fmul_rn(d, __fmaf_rn(k[3], fx, __fmaf_rn(k[4], fy, k[5])));
    const float cz = __fmul_rn(d, __fmaf_rn(k[6], fx, __fmaf_rn(k[7], fy, k[8])));
    return rot_to_world(v.R, __fsub_rn(cx, v.t[0]), __fsub_rn(cy, v.t[1]), __fsub_rn(cz, v.t[2]));
}

// World point in view v's camera frame: R X + t.
__device__ __forceinline__ float3 to_camera(const FuseView& v, float3 X) {
    const float* R = v.R;
    return make_float3(__fmaf_rn(R[0], X.x, __fmaf_rn(R[1], X.y, __fmaf_rn(R[2], X.z, v.t[0]))),
                       __fmaf_rn(R[3], X.x, __fmaf_rn(R[4], X.y, __fmaf_rn(R[5], X.z, v.t[1]))),
                       __fmaf_rn(R[6], X.x, __fmaf_rn(R[7], X.y, __fmaf_rn(R[8], X.z, v.t[2]))));
}

// Homogeneous pixel K p of a camera-frame point.
__device__ __forceinline__ float3 to_pixel(const float* K, float3 p) {
    return make_float3(__fmaf_rn(K[0], p.x, __fmaf_rn(K[1], p.y, __fmul_rn(K[2], p.z))),
                       __fmaf_rn(K[3], p.x, __fmaf_rn(K[4], p.y, __fmul_rn(K[5], p.z))),
                       __fmaf_rn(K[6], p.x, __fmaf_rn(K[7], p.y, __fmul_rn(K[8], p.z))));
}

// Fuses pixel (x, y) of view i.  False when it emits no point (invalid,
// too few agreeing views, or a lower-index view emits this surface point).
__device__ bool fuse_pixel(const FuseArgs& a, int i, int x, int y, Fused* out) {
    const FuseView& v = a.views[i];
    const size_t idx = static_cast<size_t>(y) * v.W + x;
    const float d = v.depth[idx];
    if (!(d > 0.0f)) return false;
    if (v.conf && !(v.conf[idx] >= a.min_conf)) return false;
    const float fx = static_cast<float>(x), fy = static_cast<float>(y);
    const float3 X = to_world(v, fx, fy, d);
    const float3 n = rot_to_world(v.R, v.normal[3 * idx], v.normal[3 * idx + 1], v.normal[3 * idx + 2]);
    float sx = X.x, sy = X.y, sz = X.z, snx = n.x, sny = n.y, snz = n.z;
    float sc = v.gray ? v.gray[idx] : 0.0f;
    int count = 1;
    for (int k = 0; k < v.nb_count; ++k) {
        const int j = a.neighbors[v.nb_begin + k];
        const FuseView& w = a.views[j];
        const float3 p = to_camera(w, X);
        if (!(p.z > 0.0f)) continue;
        const float3 h = to_pixel(w.K, p);
        if (!(h.z > 0.0f)) continue;
        const float u = __fdiv_rn(h.x, h.z), vv = __fdiv_rn(h.y, h.z);
        // The loose range keeps the conversion below in range (and rejects NaN).
        if (!(u >= -0.5f && u <= static_cast<float>(w.W) && vv >= -0.5f && vv <= static_cast<float>(w.H)))
            continue;
        const int qx = __float2int_rn(u), qy = __float2int_rn(vv);
        if (qx < 0 || qx >= w.W || qy < 0 || qy >= w.H) continue;
        const size_t q = static_cast<size_t>(qy) * w.W + qx;
        const float dj = w.depth[q];
        if (!(dj > 0.0f)) continue;
        if (w.conf && !(w.conf[q] >= a.min_conf)) continue;
        if (!(fabsf(__fsub_rn(p.z, dj)) <= __fmul_rn(a.max_depth_rel, dj))) continue;
        const float3 Y = to_world(w, static_cast<float>(qx), static_cast<float>(qy), dj);
        const float3 r = to_camera(v, Y);
        if (!(r.z > 0.0f)) continue;
        const float3 g = to_pixel(v.K, r);
        if (!(g.z > 0.0f)) continue;
        const float du = __fsub_rn(__fdiv_rn(g.x, g.z), fx), dv = __fsub_rn(__fdiv_rn(g.y, g.z), fy);
        if (!(__fmaf_rn(du, du, __fmul_rn(dv, dv)) <= a.max_reproj_sq)) continue;
        const float3 m = rot_to_world(w.R, w.normal[3 * q], w.normal[3 * q + 1], w.normal[3 * q + 2]);
        if (!(__fmaf_rn(n.x, m.x, __fmaf_rn(n.y, m.y, __fmul_rn(n.z, m.z))) >= a.min_normal_cos)) continue;
        if (j < i) return false;  // the lower-index view emits this surface point
        sx = __fadd_rn(sx, Y.x);
        sy = __fadd_rn(sy, Y.y);
        sz = __fadd_rn(sz, Y.z);
        snx = __fadd_rn(snx, m.x);
        sny = __fadd_rn(sny, m.y);
        snz = __fadd_rn(snz, m.z);
        sc = __fadd_rn(sc, w.gray ? w.gray[q] : 0.0f);
        ++count;
    }
    if (count < a.min_views) return false;
    if (out) {
        const float c = static_cast<float>(count);
        out->px = __fdiv_rn(sx, c);
        out->py = __fdiv_rn(sy, c);
        out->pz = __fdiv_rn(sz, c);
        const float len = __fsqrt_rn(__fmaf_rn(snx, snx, __fmaf_rn(sny, sny, __fmul_rn(snz, snz))));
        const bool unit = len > 0.0f;
        out->nx = unit ? __fdiv_rn(snx, len) : 0.0f;
        out->ny = unit ? __fdiv_rn(sny, len) : 0.0f;
        out->nz = unit ? __fdiv_rn(snz, len) : 0.0f;
        out->c = __fdiv_rn(sc, c);
    }
    return true;
}

__device__ __forceinline__ bool locate(const FuseArgs& a, int* view, int* x, int* y) {
    const int i = fuse_view_of(a, blockIdx.x);
    const FuseView& v = a.views[i];
    const long long p = static_cast<long long>(blockIdx.x - a.view_block[i]) * FUSE_THREADS + threadIdx.x;
    *view = i;
    if (p >= static_cast<long long>(v.W) * v.H) return false;
    *y = static_cast<int>(p / v.W);
    *x = static_cast<int>(p - static_cast<long long>(*y) * v.W);
    return true;
}

__global__ void __launch_bounds__(FUSE_THREADS) fuse_count_kernel(FuseArgs a, int* block_counts) {
    int i = 0, x = 0, y = 0;
    const bool emit = locate(a, &i, &x, &y) && fuse_pixel(a, i, x, y, nullptr);
    const int n = __syncthreads_count(emit);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = n;
}

// One CTA: exclusive prefix of the per-CTA counts, and their total.
constexpr int SCAN_THREADS = 1024;
__global__ void __launch_bounds__(SCAN_THREADS) fuse_scan_kernel(const int* counts, int n, long long* offsets,
                                                                 long long* total) {
    __shared__ long long part[SCAN_THREADS];
    const int t = threadIdx.x;
    const int per = (n + SCAN_THREADS - 1) / SCAN_THREADS;
    const int lo = min(n, t * per), hi = min(n, lo + per);
    long long s = 0;
    for (int k = lo; k < hi; ++k) s += counts[k];
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < SCAN_THREADS; o <<= 1) {  // inclusive scan of the chunk sums
        const long long add = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += add;
        __syncthreads();
    }
    long long run = t > 0 ? part[t - 1] : 0;
    for (int k = lo; k < hi; ++k) {
        offsets[k] = run;
        run += counts[k];
    }
    if (t == SCAN_THREADS - 1) *total = part[t];
}

__global__ void __launch_bounds__(FUSE_THREADS) fuse_write_kernel(FuseArgs a, const long long* offsets,
                                                                  float* positions, float* normals, float* colors,
                                                                  long long capacity) {
    __shared__ int warp_n[FUSE_THREADS / 32];
    int i = 0, x = 0, y = 0;
    Fused f;
    const bool emit = locate(a, &i, &x, &y) && fuse_pixel(a, i, x, y, &f);
    const unsigned bal = __ballot_sync(0xffffffffu, emit);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_n[w] = __popc(bal);
    __syncthreads();
    if (!emit) return;
    int rank = __popc(bal & ((1u << lane) - 1u));
    for (int k = 0; k < w; ++k) rank += warp_n[k];
    const long long o = offsets[blockIdx.x] + rank;
    if (o >= capacity) return;
    if (positions) {
        positions[3 * o] = f.px;
        positions[3 * o + 1] = f.py;
        positions[3 * o + 2] = f.pz;
    }
    if (normals) {
        normals[3 * o] = f.nx;
        normals[3 * o + 1] = f.ny;
        normals[3 * o + 2] = f.nz;
    }
    if (colors) {
        colors[3 * o] = f.c;
        colors[3 * o + 1] = f.c;
        colors[3 * o + 2] = f.c;
    }
}

}  // namespace

cudaError_t launch_fuse_count(const FuseArgs& a, int blocks, int* block_counts, cudaStream_t st) {
    if (blocks <= 0) return cudaSuccess;
    fuse_count_kernel<<<blocks, FUSE_THREADS, 0, st>>>(a, block_counts);
    return cudaGetLastError();
}

cudaError_t launch_fuse_scan(const int* block_counts, int blocks, long long* block_offsets, long long* total,
                             cudaStream_t st) {
    fuse_scan_kernel<<<1, SCAN_THREADS, 0, st>>>(block_counts, blocks, block_offsets, total);
    return cudaGetLastError();
}

cudaError_t launch_fuse_write(const FuseArgs& a, int blocks, const long long* block_offsets, float* positions,
                              float* normals, float* colors, long long capacity, cudaStream_t st) {
    if (blocks <= 0) return cudaSuccess;
    fuse_write_kernel<<<blocks, FUSE_THREADS, 0, st>>>(a, block_offsets, positions, normals, colors, capacity);
    return cudaGetLastError();
}

}  // namespace hp
