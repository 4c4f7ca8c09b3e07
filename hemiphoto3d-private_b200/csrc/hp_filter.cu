// Geometric-consistency filter kernels: the fused stage of a solve (one
// view's tiles, in place on its packed plane state) and the same check on
// caller-owned maps (hp_geometric_filter).  The per-pixel rule lives in
// hp_filter.cuh, shared with the persistent kernels.
//
// The reference packs every source's depth and normal map on the host and
// uploads them per view (src/dense_recon/patchmatch_mvs.cu:1290-1340); here
// the sources are read where they lie - the solve's packed state, or the
// caller's device maps - so no map crosses the host.
#include "hp_filter.cuh"

namespace hp {

namespace {

__global__ void __launch_bounds__(256) filter_view_kernel(const ViewDesc* __restrict__ views, int view,
                                                                  bool write_out) {
    const ViewDesc* v = &views[view];
    const int tx = blockIdx.x % v->tiles_x, ty = blockIdx.x / v->tiles_x;
    tile_filter(views, v, tx, ty, write_out);
}

// One thread per pixel of caller maps: depth and confidence updated in place
// (depth 0 and confidence 0 where too few sources agree; confidence 0 where
// the depth is not positive).
__global__ void __launch_bounds__(256) filter_maps_kernel(FilterMaps a, float* __restrict__ depth,
                                                          const float* __restrict__ normal,
                                                          float* __restrict__ conf) {
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (x >= a.W || y >= a.H) return;
    const size_t i = static_cast<size_t>(y) * a.W + x;
    const float d = depth[i];
    if (!(d > 0.0f)) {
        conf[i] = 0.0f;
        return;
    }
    auto fetch = [&](int s, size_t k) {
        const float* n = a.src_normal[s] + 3 * k;
        return make_float4(__ldg(a.src_depth[s] + k), __ldg(n), __ldg(n + 1), __ldg(n + 2));
    };
    const int agree = filter_agreeing(&a.f, a.W, a.H, x, y, d, normal[3 * i], normal[3 * i + 1], normal[3 * i + 2],
                                      fetch);
    if (agree < a.f.min_consistent) {
        depth[i] = 0.0f;
        conf[i] = 0.0f;
    }
}

}  // namespace

cudaError_t launch_filter_view(const ViewDesc* views, int view, int tiles, int tile_h, bool write_out,
                               cudaStream_t st) {
    if (tiles <= 0) return cudaSuccess;
    filter_view_kernel<<<tiles, 32 * tile_h, 0, st>>>(views, view, write_out);
    return cudaGetLastError();
}

cudaError_t launch_filter_maps(const FilterMaps& a, float* depth, const float* normal, float* conf,
                               cudaStream_t st) {
    dim3 grid((a.W + 31) / 32, (a.H + 7) / 8);
    filter_maps_kernel<<<grid, 256, 0, st>>>(a, depth, normal, conf);
    return cudaGetLastError();
}

}  // namespace hp
