// Layout kernels: image conversion on upload and hypothesis (un)packing
// between the engine's packed float4 planes and the caller's depth / AoS
// normal / cost maps.  All are HBM-bound streaming kernels: grid-stride loops
// over a grid sized to the SM count.
#include "hp_internal.h"

namespace hp {

namespace {

int g_grid_cache = 0;
int stream_grid() {
    if (g_grid_cache == 0) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        g_grid_cache = sms * 8;
    }
    return g_grid_cache;
}

// u8 / f16 / f32 (tightly packed) -> FP32 and FP16 pitched planes, values in [0, 1].
__global__ void to_planes_kernel(const void* __restrict__ src, int dtype, int W, int H, float* __restrict__ dst,
                                 int pitch, __half* __restrict__ dst16, int pitch16) {
    const size_t n = static_cast<size_t>(W) * H;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int y = static_cast<int>(i / W), x = static_cast<int>(i - static_cast<size_t>(y) * W);
        float v;
        __half h;
        if (dtype == HP_DTYPE_U8) {
            v = __fdiv_rn(static_cast<float>(static_cast<const unsigned char*>(src)[i]), 255.0f);
            h = __float2half_rn(v);
        } else if (dtype == HP_DTYPE_F16) {
            h = static_cast<const __half*>(src)[i];
            v = __half2float(h);
        } else {
            v = static_cast<const float*>(src)[i];
            h = __float2half_rn(v);
        }
        dst[static_cast<size_t>(y) * pitch + x] = v;
        dst16[static_cast<size_t>(y) * pitch16 + x] = h;
    }
}

// Quad plane of the FP16 software sampler.  Quad (x, y) holds the bilinear
// patch of texels t00 = t(x,y), t10 = t(x+1,y), t01 = t(x,y+1), t11 =
// t(x+1,y+1) (right and bottom neighbours clamped) in difference form:
//   .x = (t00 - 0.5, t01 - t00), .y = (t10 - t00, t11 - t10 - t01 + t00),
// each formed exactly in FP32 from the FP16 texels and rounded once to FP16,
// so a sample is t00 + fx (t10 - t00) + fy ((t01 - t00) + fx dxy): two FP16
// FMAs.  The -0.5 shift keeps the interpolated values within [-0.5, 0.5].
// Quad (x, y) is stored at x_lo | y_lo << 8 | x_hi << 16 | y_hi << 24 (bytes of
// x and y): 256 x 256 blocks, the layout the sampler addresses with one byte
// permute (hpx::QuadPlane).
__global__ void quads_kernel(const __half* __restrict__ src, int pitch16, int W, int H, uint2* __restrict__ quads) {
    const size_t n = static_cast<size_t>(W) * H;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int y = static_cast<int>(i / W), x = static_cast<int>(i - static_cast<size_t>(y) * W);
        const int x1 = min(x + 1, W - 1), y1 = min(y + 1, H - 1);
        const __half* r0 = src + static_cast<size_t>(y) * pitch16;
        const __half* r1 = src + static_cast<size_t>(y1) * pitch16;
        const float t00 = __half2float(r0[x]), t10 = __half2float(r0[x1]);
        const float t01 = __half2float(r1[x]), t11 = __half2float(r1[x1]);
        const __half2 a = __floats2half2_rn(__fsub_rn(t00, 0.5f), __fsub_rn(t01, t00));
        const __half2 b = __floats2half2_rn(__fsub_rn(t10, t00), __fadd_rn(__fsub_rn(t11, t10), __fsub_rn(t00, t01)));
        uint2 q;
        memcpy(&q.x, &a, sizeof q.x);
        memcpy(&q.y, &b, sizeof q.y);
        quads[static_cast<size_t>(x & 255) | (static_cast<size_t>(y & 255) << 8) |
              (static_cast<size_t>(x >> 8) << 16) | (static_cast<size_t>(y >> 8) << 24)] = q;
    }
}

// SfM seeding: for every pixel, the largest index of a seed whose (2r+1)^2
// square covers it (atomicMax keeps the last-listed seed, as painting the
// squares in list order would).  One CTA per seed.  The initialisation stage
// (tile_init) then takes the seed's plane instead of a random one.
__global__ void seed_map_kernel(const hp_seed* __restrict__ seeds, int radius, int W, int H, int* __restrict__ map) {
    const int k = blockIdx.x;
    const hp_seed s = seeds[k];
    const int side = 2 * radius + 1;
    const long long x0 = static_cast<long long>(s.x) - radius, y0 = static_cast<long long>(s.y) - radius;
    for (int t = threadIdx.x; t < side * side; t += blockDim.x) {
        const long long x = x0 + t % side, y = y0 + t / side;
        if (x < 0 || x >= W || y < 0 || y >= H) continue;
        atomicMax(map + y * W + x, k);
    }
}


// Packed state -> caller maps; confidence is 1 - cost / 2, the reference's
// host-side conversion (patchmatch_mvs.cu:1246-1252), formed on the device.
__global__ void unpack_kernel(const float4* __restrict__ hyp, const float* __restrict__ cost_in, size_t n,
                              float* __restrict__ depth, float* __restrict__ normal, float* __restrict__ cost,
                              float* __restrict__ conf) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float4 h = hyp[i];
        if (depth) depth[i] = h.x;
        if (normal) {
            normal[3 * i] = h.y;
            normal[3 * i + 1] = h.z;
            normal[3 * i + 2] = h.w;
        }
        if (cost || conf) {
            const float c = cost_in[i];
            if (cost) cost[i] = c;
            if (conf) conf[i] = __fsub_rn(1.0f, __fmul_rn(c, 0.5f));
        }
    }
}

__global__ void pack_kernel(const float* __restrict__ depth, const float* __restrict__ normal,
                            const float* __restrict__ cost, size_t n, float4* __restrict__ hyp,
                            float* __restrict__ cost_out) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        if (depth && normal) hyp[i] = make_float4(depth[i], normal[3 * i], normal[3 * i + 1], normal[3 * i + 2]);
        if (cost) cost_out[i] = cost[i];
    }
}

}  // namespace

cudaError_t launch_to_f32(const void* src, int dtype, int W, int H, float* dst, int dst_pitch, __half* dst16,
                          int dst16_pitch, cudaStream_t st) {
    to_planes_kernel<<<stream_grid(), 256, 0, st>>>(src, dtype, W, H, dst, dst_pitch, dst16, dst16_pitch);
    return cudaGetLastError();
}

cudaError_t launch_quads(const __half* src16, int pitch16, int W, int H, uint2* quads, cudaStream_t st) {
    quads_kernel<<<stream_grid(), 256, 0, st>>>(src16, pitch16, W, H, quads);
    return cudaGetLastError();
}

cudaError_t launch_seed_map(const hp_seed* seeds, int num_seeds, int radius, int W, int H, int* map,
                            cudaStream_t st) {
    const size_t n = static_cast<size_t>(W) * H;
    cudaError_t e = cudaMemsetAsync(map, 0xff, n * sizeof(int), st);
    if (e != cudaSuccess || num_seeds <= 0) return e;
    seed_map_kernel<<<num_seeds, 256, 0, st>>>(seeds, radius, W, H, map);
    return cudaGetLastError();
}

cudaError_t launch_unpack(const ViewDesc* vh, int view, float* depth, float* normal, float* cost, float* conf,
                          cudaStream_t st) {
    const ViewDesc& v = vh[view];
    unpack_kernel<<<stream_grid(), 256, 0, st>>>(v.hyp, v.cost, static_cast<size_t>(v.W) * v.H, depth, normal,
                                                 cost, conf);
    return cudaGetLastError();
}

cudaError_t launch_pack(const ViewDesc* vh, int view, const float* depth, const float* normal, const float* cost,
                        cudaStream_t st) {
    const ViewDesc& v = vh[view];
    pack_kernel<<<stream_grid(), 256, 0, st>>>(depth, normal, cost, static_cast<size_t>(v.W) * v.H, v.hyp,
                                               v.cost);
    return cudaGetLastError();
}

}  // namespace hp
