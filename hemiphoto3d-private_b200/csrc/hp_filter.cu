// Geometric-consistency filter over device-resident depth maps
// (geometric_consistency_filter_kernel, src/dense_recon/patchmatch_mvs.cu:668-781).
//
// The reference packs every source's depth and normal map on the host and
// uploads them per view (:1290-1340); here each source map is read in place
// through its own pointer, so a solve's outputs feed the filter without a host
// round trip.  Built with the reference's --use_fast_math and the same
// expression order, so pixel decisions match it at the rounding boundaries.
#include "hp_internal.h"

namespace hp {


namespace {

__global__ void __launch_bounds__(256) geometric_filter_kernel(FilterArgs a, float* __restrict__ depth,
                                                               const float* __restrict__ normal,
                                                               float* __restrict__ conf) {
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (x >= a.W || y >= a.H) return;
    const size_t idx = static_cast<size_t>(y) * a.W + x;
    const float d = depth[idx];
    if (d <= 0.0f) {
        conf[idx] = 0.0f;
        return;
    }
    const float* ki = a.ref_kinv;
    const float* R = a.ref_R;
    const float fx = static_cast<float>(x), fy = static_cast<float>(y);
    const float pcx = d * (ki[0] * fx + ki[1] * fy + ki[2]);
    const float pcy = d * (ki[3] * fx + ki[4] * fy + ki[5]);
    const float pcz = d * (ki[6] * fx + ki[7] * fy + ki[8]);
    const float ax = pcx - a.ref_t[0], ay = pcy - a.ref_t[1], az = pcz - a.ref_t[2];
    const float pwx = R[0] * ax + R[3] * ay + R[6] * az;
    const float pwy = R[1] * ax + R[4] * ay + R[7] * az;
    const float pwz = R[2] * ax + R[5] * ay + R[8] * az;
    const float ncx = normal[3 * idx], ncy = normal[3 * idx + 1], ncz = normal[3 * idx + 2];
    const float nwx = R[0] * ncx + R[3] * ncy + R[6] * ncz;
    const float nwy = R[1] * ncx + R[4] * ncy + R[7] * ncz;
    const float nwz = R[2] * ncx + R[5] * ncy + R[8] * ncz;
    int consistent = 0;
    for (int s = 0; s < a.S; ++s) {
        const FilterCam& c = a.src[s];
        const float psx = c.R[0] * pwx + c.R[1] * pwy + c.R[2] * pwz + c.t[0];
        const float psy = c.R[3] * pwx + c.R[4] * pwy + c.R[5] * pwz + c.t[1];
        const float psz = c.R[6] * pwx + c.R[7] * pwy + c.R[8] * pwz + c.t[2];
        if (psz <= 0.0f) continue;
        const float prx = c.K[0] * psx + c.K[1] * psy + c.K[2] * psz;
        const float pry = c.K[3] * psx + c.K[4] * psy + c.K[5] * psz;
        const float prz = c.K[6] * psx + c.K[7] * psy + c.K[8] * psz;
        const float u = prx / prz;
        const float v = pry / prz;
        const int ui = __float2int_rn(u), vi = __float2int_rn(v);
        if (ui < 0 || ui >= a.W || vi < 0 || vi >= a.H) continue;
        const size_t sp = static_cast<size_t>(vi) * a.W + ui;
        const float ds = __ldg(a.src_depth[s] + sp);
        if (ds <= 0.0f) continue;
        const float err = fabsf(ds - psz) / psz;
        if (err > a.depth_tol) continue;
        const float* sn = a.src_normal[s] + 3 * sp;
        const float nsx = __ldg(sn), nsy = __ldg(sn + 1), nsz = __ldg(sn + 2);
        const float qx = c.R[0] * nsx + c.R[3] * nsy + c.R[6] * nsz;
        const float qy = c.R[1] * nsx + c.R[4] * nsy + c.R[7] * nsz;
        const float qz = c.R[2] * nsx + c.R[5] * nsy + c.R[8] * nsz;
        const float cos_angle = nwx * qx + nwy * qy + nwz * qz;
        if (cos_angle < a.normal_tol_cos) continue;
        consistent++;
    }
    if (consistent < a.min_consistent) {
        depth[idx] = 0.0f;
        conf[idx] = 0.0f;
    }
}

}  // namespace

cudaError_t launch_geometric_filter(const FilterArgs& a, float* depth, const float* normal, float* conf,
                                    cudaStream_t st) {
    dim3 grid((a.W + 31) / 32, (a.H + 7) / 8);
    geometric_filter_kernel<<<grid, 256, 0, st>>>(a, depth, normal, conf);
    return cudaGetLastError();
}

}  // namespace hp
