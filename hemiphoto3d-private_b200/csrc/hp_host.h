// Host-side internals shared by the C ABI translation units: the context,
// its images and scratch buffers, error reporting, and the helpers that turn
// jobs into device descriptors.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "hp_internal.h"

namespace hpx {

// Block-tiled FP16 software-sampler quad plane in sparsely backed virtual
// memory (hp_quads.cpp): quad (x, y) at element quad_block_offset(x, y).
struct QuadPlane {
    uint2* base = nullptr;       // start of the reserved span
    size_t reserved = 0;         // bytes of virtual address space
    size_t physical = 0;         // bytes of device memory mapped under it
    std::vector<unsigned long long> handles;  // one physical allocation per 256-row block row
    std::vector<size_t> offsets, sizes;
    std::vector<char> mapped;
};
cudaError_t alloc_quads(int device, int W, int H, QuadPlane* q);
void free_quads(QuadPlane* q);
size_t quad_block_offset(int x, int y);

struct Image {
    int W = 0, H = 0;
    float* f32 = nullptr;
    size_t pitch32 = 0;  // bytes
    __half* f16 = nullptr;
    size_t pitch16 = 0;  // bytes
    cudaArray_t arr32 = nullptr, arr16 = nullptr;
    cudaTextureObject_t tex32 = 0, tex16 = 0;
    // Software-sampler plane: quad (x, y) holds the 2x2 FP16 block
    // {t(x,y), t(x+1,y)}, {t(x,y+1), t(x+1,y+1)} in difference form shifted by
    // -0.5 (edges clamped), block-tiled (QuadPlane).
    QuadPlane quads;
};

// Grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess) cap = bytes;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

}  // namespace hpx

struct hp_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    std::map<int, hpx::Image> images;
    int next_id = 1;
    hpx::DevBuf state;   // hypotheses + costs of all jobs of a solve
    hpx::DevBuf descs;   // ViewDesc array
    hpx::DevBuf lists;   // active-view lists and tile prefixes
    hpx::DevBuf staging; // host-memory results pass through here
    hpx::DevBuf seedbuf; // SfM seeds of one job and their W*H index map
    hpx::DevBuf upload;  // host images land here before conversion
    hpx::DevBuf filters; // FilterStage per filtered job of a solve
    // Released images kept for reuse by the next upload of the same size
    // (their planes, arrays, texture objects and quad plane), oldest first,
    // up to image_cache_limit bytes.
    std::vector<hpx::Image> image_cache;
    size_t image_cache_bytes = 0;
    size_t image_cache_limit = size_t(4) << 30;
    // Profiler: launch counts always; with profiling on, CUDA events bracket
    // each launch and are read back at the next synchronisation point.
    bool profiling = false;
    hp_profile prof{};
    std::vector<cudaEvent_t> events;
    std::vector<std::pair<int, size_t>> pending;  // (kind, index of the start event)
    size_t events_used = 0;
};

namespace hpx {

// Run one launch, counted under `kind` and, when profiling, bracketed by events.
template <class F>
cudaError_t counted(hp_ctx* ctx, int kind, F&& launch) {
    ctx->prof.launches[kind]++;
    if (!ctx->profiling) return launch();
    while (ctx->events.size() < ctx->events_used + 2) {
        cudaEvent_t e;
        cudaError_t err = cudaEventCreate(&e);
        if (err != cudaSuccess) return err;
        ctx->events.push_back(e);
    }
    const size_t i = ctx->events_used;
    ctx->events_used += 2;
    cudaEventRecord(ctx->events[i], ctx->stream);
    cudaError_t err = launch();
    cudaEventRecord(ctx->events[i + 1], ctx->stream);
    ctx->pending.emplace_back(kind, i);
    return err;
}

// Fold completed event pairs into the profile (call after a stream sync).
inline void flush_profile(hp_ctx* ctx) {
    for (auto& pk : ctx->pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ctx->events[pk.second], ctx->events[pk.second + 1]) == cudaSuccess) {
            ctx->prof.device_ms[pk.first] += ms;
            ctx->prof.timed[pk.first]++;
        }
    }
    ctx->pending.clear();
    ctx->events_used = 0;
}

inline hp_status fail(hp_ctx* c, hp_status s, const char* fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return s;
}

#define HP_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? HP_ERR_OUT_OF_MEMORY : HP_ERR_CUDA, \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);       \
    } while (0)

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

hp_status check_params(hp_ctx* ctx, const hp_params* p);
hp::SolveConsts consts_of(const hp_params* p);
// Validate a job and fill the image/camera part of its descriptor (tiles of
// TILE_W x tile_h pixels).
hp_status fill_desc(hp_ctx* ctx, const hp_job* j, int jobno, hp::ViewDesc* d, int tile_h);
// SfM seeds of a job: validation, the device bytes its seed list and W x H
// index map take, and staging them (upload + map build on `st`) into `area`,
// which sets d->seeds / d->seed_map (left null for a job without seeds).
hp_status check_seeds(hp_ctx* ctx, const hp_job* j, int jobno);
size_t seed_area_bytes(const hp_job* j, int W, int H);
cudaError_t stage_seeds(const hp_job* j, void* area, hp::ViewDesc* d, cudaStream_t st);
// Geometric-consistency stages of a batch (hp_params.filter_*): for each job
// the FilterStage it runs after its last half-pass, or none (has[k] = 0);
// order lists the filtered jobs in job order, the order the stages run in.
// Source views are the jobs that solved the job's source images (the last
// such job when several did), of the same size, the job itself excluded.
void filter_stages(const hp_job* jobs, int n, const hp_params* p, const std::vector<hp::ViewDesc>& descs,
                   std::vector<hp::FilterStage>* stages, std::vector<char>* has, std::vector<int>* order);
// One source's FP64-composed transforms (hp::FilterSource) from the two cameras.
bool filter_source_of(const hp_camera& ref, const hp_camera& src, hp::FilterSource* q);
void free_image(Image& im);
// Device bytes an image holds (planes, arrays, quad plane).
size_t image_bytes(const Image& im);
cudaError_t make_linear_texture(cudaArray_t arr, cudaTextureObject_t* tex);

}  // namespace hpx
