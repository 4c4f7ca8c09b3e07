// hp_solve_static: the single-view FP32 solve without any device allocation.
//
// Who needs it: callers that must not allocate device memory from inside the
// library - a host application whose device memory is owned by its own pool
// or arena (a framework's caching allocator, a fixed budget per process), or
// a latency-critical loop where cudaMalloc / cudaFree and the device
// synchronisation they imply are not acceptable.  hp_solve keeps its plane
// state, descriptors and launch lists in context-owned buffers that grow with
// cudaMalloc; this entry point runs the same kernels with all of that scratch
// in one statically sized device array instead.
//
// The scratch is `g_static_scratch` below: a file-scope __device__ array of
// HP_STATIC_SCRATCH_BYTES, created when the library's device code is loaded
// on a GPU and held by every GPU that loads it until the process exits.  Host
// code may not use the array's name as a device address (on the host it is
// only a stand-in symbol), so the first call in each CUDA context looks up the
// real address with cudaGetSymbolAddress while that context is current and
// caches it under the context's process-unique id (cuCtxGetId); that first
// call therefore does the set-up and should come before any stream capture.
// A context created later on the same device - after cudaDeviceReset, or a
// driver-API context the caller made current - has a new id, so its first
// call looks the address up again instead of using a stale one.
//
// Every call shares the one array and overwrites it: the state a call needs
// is fully written before it is read (the init kernel writes every plane, the
// cost kernel every cost, descriptors are copied in), so nothing needs to
// start at zero.  The call waits for its own work before returning, also when
// it fails after queuing some of it, but two calls running at the same time
// (from different host threads, on any streams) would use the same array and
// corrupt each other: callers must serialise them.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "hp_internal.h"

namespace {

constexpr size_t kHeaderBytes = 4096;  // ViewDesc + launch lists
constexpr size_t kPlaneBytes = static_cast<size_t>(HP_STATIC_MAX_PIXELS) * sizeof(float4);
constexpr size_t kCostBytes = static_cast<size_t>(HP_STATIC_MAX_PIXELS) * sizeof(float);
constexpr size_t HP_STATIC_SCRATCH_BYTES = kHeaderBytes + kPlaneBytes + kCostBytes;

static __device__ __align__(256) unsigned char g_static_scratch[HP_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
struct ScratchSlot {
    unsigned long long ctx_id = 0;  // cuCtxGetId of the context the address belongs to (0: none yet)
    void* addr = nullptr;
};
ScratchSlot g_scratch[kMaxDevices];

// Driver entry points for the current context's id, reached through the
// runtime so the library does not link libcuda.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

template <class F>
F driver_entry(const char* name) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
        return nullptr;
    return reinterpret_cast<F>(p);
}

// Id of the context current on this thread; 0 when it cannot be told (then the
// address is looked up on every call rather than cached).
unsigned long long current_context_id() {
    static const CtxGetCurrentFn get_current = driver_entry<CtxGetCurrentFn>("cuCtxGetCurrent");
    static const CtxGetIdFn get_id = driver_entry<CtxGetIdFn>("cuCtxGetId");
    if (!get_current || !get_id) return 0;
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of g_static_scratch in the context current on `device`.
cudaError_t scratch_address(int device, unsigned char** out) {
    // Before the runtime has made a context current the id reads 0, and the
    // lookup below (which makes one current) is simply repeated next call.
    const unsigned long long id = current_context_id();
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    ScratchSlot& slot = g_scratch[device];
    if (id == 0 || slot.ctx_id != id) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        slot.addr = p;
        slot.ctx_id = id;
    }
    *out = static_cast<unsigned char*>(slot.addr);
    return cudaSuccess;
}

hp_status fail(cudaError_t e) { return e == cudaErrorMemoryAllocation ? HP_ERR_OUT_OF_MEMORY : HP_ERR_CUDA; }

}  // namespace

extern "C" hp_status hp_solve_static(int device, void* stream, const hp_job* job, const float* ref_image,
                                     int ref_pitch, int width, int height, const unsigned long long* src_textures,
                                     const hp_params* params, hp_maps* out) {
    if (!job || !ref_image || !src_textures || !params || !out) return HP_ERR_INVALID_ARG;
    if (device < 0 || device >= kMaxDevices) return HP_ERR_INVALID_ARG;
    if (width < 2 || height < 2 || ref_pitch < width) return HP_ERR_INVALID_ARG;
    if (static_cast<long long>(width) * height > HP_STATIC_MAX_PIXELS) return HP_ERR_UNSUPPORTED;  // over the fixed scratch
    if (out->memory != HP_MEMORY_DEVICE || !out->depth || !out->normal || !out->cost) return HP_ERR_INVALID_ARG;
    if (params->precision != HP_PRECISION_F32) return HP_ERR_UNSUPPORTED;
    if (params->radius < 1 || params->radius > HP_MAX_RADIUS || (params->stride != 1 && params->stride != 2) ||
        params->top_k < 1 || params->top_k > HP_MAX_TOP_K || params->refine_steps < 0 || params->refine_steps > 4)
        return HP_ERR_INVALID_ARG;
    if (job->num_seeds != 0) return HP_ERR_UNSUPPORTED;  // the seed index map would need scratch
    if (job->num_sources < 1 || job->num_sources > HP_MAX_SOURCES || !(job->depth_min > 0.f) ||
        !(job->depth_max > job->depth_min) || !std::isfinite(job->depth_max) || job->iterations < 0 ||
        job->iterations > 1000)
        return HP_ERR_INVALID_ARG;

    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return HP_ERR_CUDA;
    if (prev != device && cudaSetDevice(device) != cudaSuccess) return HP_ERR_CUDA;
    struct Restore {
        int dev;
        ~Restore() { if (dev >= 0) cudaSetDevice(dev); }
    } restore{prev != device ? prev : -1};

    unsigned char* base = nullptr;
    const cudaError_t se = scratch_address(device, &base);
    if (se != cudaSuccess) return fail(se);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Descriptor, built on the host and copied into the scratch header.
    hp::ViewDesc d;
    std::memset(&d, 0, sizeof d);
    d.ref = ref_image;
    d.ref_pitch = ref_pitch;
    d.W = width;
    d.H = height;
    d.S = job->num_sources;
    for (int s = 0; s < job->num_sources; ++s) d.src_tex[s] = static_cast<cudaTextureObject_t>(src_textures[s]);
    if (job->use_coeffs) {
        std::memcpy(d.kinv, job->kinv, sizeof d.kinv);
        for (int s = 0; s < job->num_sources; ++s) std::memcpy(d.ab[s], job->ab[s], sizeof d.ab[s]);
    } else {
        double kinv[9], ab[HP_MAX_SOURCES * 12];
        hp_status hs = hp_setup_homographies(&job->ref_cam, job->src_cams, job->num_sources, kinv, ab);
        if (hs != HP_OK) return hs;
        for (int i = 0; i < 9; ++i) d.kinv[i] = static_cast<float>(kinv[i]);
        for (int s = 0; s < job->num_sources; ++s)
            for (int i = 0; i < 12; ++i) d.ab[s][i] = static_cast<float>(ab[12 * s + i]);
    }
    d.tile_h = hp::TILE_H;
    d.tiles_x = (width + hp::TILE_W - 1) / hp::TILE_W;
    d.tiles_y = (height + hp::TILE_H - 1) / hp::TILE_H;
    d.dmin = job->depth_min;
    d.dmax = job->depth_max;
    d.seed_lo = static_cast<uint32_t>(job->seed);
    d.seed_hi = static_cast<uint32_t>(job->seed >> 32);
    d.view_id = job->view_id;
    d.iterations = job->iterations;
    d.hyp = reinterpret_cast<float4*>(base + kHeaderBytes);
    d.cost = reinterpret_cast<float*>(base + kHeaderBytes + kPlaneBytes);

    // Header layout: ViewDesc at 0, then the launch list {active view 0, tile prefix 0, total}.
    static_assert(sizeof(hp::ViewDesc) + 64 <= kHeaderBytes, "scratch header too small");
    const size_t list_off = (sizeof(hp::ViewDesc) + 255) & ~size_t(255);
    const int list[3] = {0, 0, d.tiles_x * d.tiles_y};
    // Once anything is queued, a failure still waits for what was queued (it
    // may be using the shared array) before returning.
    auto bail = [st](cudaError_t err) {
        cudaStreamSynchronize(st);
        return fail(err);
    };
    cudaError_t e = cudaMemcpyAsync(base, &d, sizeof d, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return bail(e);
    if ((e = cudaMemcpyAsync(base + list_off, list, sizeof list, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return bail(e);

    hp::BatchList bl;
    bl.views = reinterpret_cast<const hp::ViewDesc*>(base);
    bl.active = reinterpret_cast<const int*>(base + list_off);
    bl.tile_prefix = bl.active + 1;
    bl.n_active = 1;
    bl.total_tiles = list[2];
    hp::SolveConsts sc;
    sc.radius = params->radius;
    sc.stride = params->stride;
    sc.top_k = params->top_k;
    sc.refine_steps = params->refine_steps;
    sc.iter_decay = params->iter_decay;
    sc.step_decay = params->step_decay;
    sc.soft_mask = 0;
    sc.tile_h = hp::TILE_H;
    sc.staging = 4;

    if ((e = hp::launch_init(bl, hp::TILE_H, st)) != cudaSuccess) return bail(e);
    if ((e = hp::launch_cost_f32(bl, sc, st)) != cudaSuccess) return bail(e);
    for (int it = 0; it < job->iterations; ++it)
        for (int color = 0; color < 2; ++color)
            if ((e = hp::launch_propagate_f32(bl, sc, it, color, st)) != cudaSuccess) return bail(e);
    if ((e = hp::launch_unpack(&d, 0, out->depth, out->normal, out->cost, out->confidence, st)) != cudaSuccess) return bail(e);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e);
    return HP_OK;
}
