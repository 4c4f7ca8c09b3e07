// On-chip peak microbenchmarks for the roofline of the PatchMatch kernels.
//
// The cost kernels are bound by the SM, not HBM: every window tap is one
// bilinear texture fetch plus ~25 FP32 operations, and the compulsory DRAM
// traffic is ~1% of HBM bandwidth.  These kernels measure, on the running GPU,
// the ceilings those taps run into:
//   - bilinear texture fetches per second from an L1-resident FP32 or FP16
//     texture (the texture-filter pipe),
//   - shared-memory read bandwidth (128-bit loads),
//   - FP32 FMA throughput.
// Each is a grid of SM-count x 8 CTAs x 256 threads with independent work per
// thread; results are written out so nothing is dead code.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int THREADS = 256;

__global__ void __launch_bounds__(THREADS) tex_rate_kernel(cudaTextureObject_t tex, int iters, float* out) {
    const int tid = blockIdx.x * THREADS + threadIdx.x;
    float u = 3.3f + (threadIdx.x & 31) * 1.7f, v = 5.1f + (threadIdx.x >> 5) * 2.3f + (blockIdx.x & 7);
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f, acc3 = 0.f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            acc0 += tex2D<float>(tex, u, v);
            acc1 += tex2D<float>(tex, u + 0.37f, v + 0.21f);
            acc2 += tex2D<float>(tex, u + 0.71f, v + 0.53f);
            acc3 += tex2D<float>(tex, u + 1.13f, v + 0.87f);
            u += 0.173f;
            v += 0.071f;
        }
        if (u > 100.f) u -= 90.f;
        if (v > 100.f) v -= 90.f;
    }
    out[tid] = acc0 + acc1 + acc2 + acc3;
}

__global__ void __launch_bounds__(THREADS) smem_rate_kernel(int iters, float* out) {
    __shared__ float4 buf[THREADS * 4];
    for (int i = threadIdx.x; i < THREADS * 4; i += THREADS)
        buf[i] = make_float4(i * 0.5f, i * 0.25f, i * 0.125f, i * 0.0625f);
    __syncthreads();
    float4 acc = make_float4(0, 0, 0, 0);
    int idx = threadIdx.x;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float4 a = buf[(idx + k * 97) & (THREADS * 4 - 1)];
            acc.x += a.x; acc.y += a.y; acc.z += a.z; acc.w += a.w;
        }
        idx = (idx + 33) & (THREADS * 4 - 1);
    }
    out[blockIdx.x * THREADS + threadIdx.x] = acc.x + acc.y + acc.z + acc.w;
}

__global__ void __launch_bounds__(THREADS) fma_rate_kernel(int iters, float* out) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = threadIdx.x * 1e-3f + k;
    const float m = 0.999f, c = 1e-4f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int r = 0; r < 16; ++r)
#pragma unroll
            for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    out[blockIdx.x * THREADS + threadIdx.x] = s;
}

int grid_size() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms * 8;
}

template <class F>
int time_ms(F&& launch, float* ms) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    launch();  // warm-up
    cudaEventRecord(a);
    launch();
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace

extern "C" {

// Bilinear texture fetches per second (FP16 texture when half_texels != 0).
int hpk_tex_fetch_rate(int half_texels, double* fetches_per_s) {
    const int n = 128;
    const int grid = grid_size();
    cudaChannelFormatDesc d = half_texels ? cudaCreateChannelDescHalf() : cudaCreateChannelDesc<float>();
    cudaArray_t arr = nullptr;
    if (cudaMallocArray(&arr, &d, n, n) != cudaSuccess) return 1;
    // Fill with a ramp (content does not matter for the rate).
    if (half_texels) {
        __half h[n * n];
        for (int i = 0; i < n * n; ++i) h[i] = __float2half(static_cast<float>(i % 97) / 97.f);
        cudaMemcpy2DToArray(arr, 0, 0, h, n * sizeof(__half), n * sizeof(__half), n, cudaMemcpyHostToDevice);
    } else {
        static float f[n * n];
        for (int i = 0; i < n * n; ++i) f[i] = static_cast<float>(i % 97) / 97.f;
        cudaMemcpy2DToArray(arr, 0, 0, f, n * sizeof(float), n * sizeof(float), n, cudaMemcpyHostToDevice);
    }
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    cudaTextureObject_t tex = 0;
    float* out = nullptr;
    int rc = 1;
    if (cudaCreateTextureObject(&tex, &rd, &td, nullptr) == cudaSuccess &&
        cudaMalloc(&out, static_cast<size_t>(grid) * THREADS * sizeof(float)) == cudaSuccess) {
        const int iters = 64;
        float ms = 0.f;
        rc = time_ms([&] { tex_rate_kernel<<<grid, THREADS>>>(tex, iters, out); }, &ms);
        *fetches_per_s = static_cast<double>(grid) * THREADS * iters * 32 / (ms * 1e-3);
    }
    if (out) cudaFree(out);
    if (tex) cudaDestroyTextureObject(tex);
    cudaFreeArray(arr);
    return rc;
}

// Shared-memory read bandwidth in bytes per second.
int hpk_smem_read_rate(double* bytes_per_s) {
    const int grid = grid_size(), iters = 512;
    float* out = nullptr;
    if (cudaMalloc(&out, static_cast<size_t>(grid) * THREADS * sizeof(float)) != cudaSuccess) return 1;
    float ms = 0.f;
    int rc = time_ms([&] { smem_rate_kernel<<<grid, THREADS>>>(iters, out); }, &ms);
    *bytes_per_s = static_cast<double>(grid) * THREADS * iters * 8 * 16 / (ms * 1e-3);
    cudaFree(out);
    return rc;
}

// FP32 FMA operations (2 flops each) per second.
int hpk_fma_rate(double* fma_per_s) {
    const int grid = grid_size(), iters = 256;
    float* out = nullptr;
    if (cudaMalloc(&out, static_cast<size_t>(grid) * THREADS * sizeof(float)) != cudaSuccess) return 1;
    float ms = 0.f;
    int rc = time_ms([&] { fma_rate_kernel<<<grid, THREADS>>>(iters, out); }, &ms);
    *fma_per_s = static_cast<double>(grid) * THREADS * iters * 16 * 8 / (ms * 1e-3);
    cudaFree(out);
    return rc;
}

}  // extern "C"
