// Quad planes of the FP16 software sampler in block-tiled, sparsely backed
// virtual memory.
//
// The sampler turns a warped coordinate pair into the quad's element offset
// with one byte permute of the two fixed-point coordinates (hp_kernels_f16.cu,
// soft_offset): offset = lo(x) | lo(y) << 8 | hi(x) << 16 | hi(y) << 24, where
// lo/hi are the low and high bytes of 0x4000 + x.  That is a layout of
// 256 x 256-quad blocks (512 KB each) whose block columns are 2^16 quads apart
// and whose block rows are 2^24 quads (128 MB) apart.  Only the first
// ceil(W / 256) blocks of each block row are ever addressed, so the span is
// reserved as virtual address space and physical memory is mapped under those
// blocks alone: ~W * H * 8 bytes, rounded up to the allocation granularity per
// block row.  The driver's virtual-memory calls are reached through
// cudaGetDriverEntryPoint, so the library does not link libcuda.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "hp_host.h"

namespace hpx {

namespace {

struct VmmApi {
    decltype(&cuMemGetAllocationGranularity) granularity = nullptr;
    decltype(&cuMemAddressReserve) reserve = nullptr;
    decltype(&cuMemAddressFree) address_free = nullptr;
    decltype(&cuMemCreate) create = nullptr;
    decltype(&cuMemRelease) release = nullptr;
    decltype(&cuMemMap) map = nullptr;
    decltype(&cuMemUnmap) unmap = nullptr;
    decltype(&cuMemSetAccess) set_access = nullptr;
    bool ok = false;
};

template <class F>
bool entry(const char* name, F* fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess ||
        !p)
        return false;
    *fn = reinterpret_cast<F>(p);
    return true;
}

const VmmApi& vmm() {
    static VmmApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        api.ok = entry("cuMemGetAllocationGranularity", &api.granularity) &&
                 entry("cuMemAddressReserve", &api.reserve) && entry("cuMemAddressFree", &api.address_free) &&
                 entry("cuMemCreate", &api.create) && entry("cuMemRelease", &api.release) &&
                 entry("cuMemMap", &api.map) && entry("cuMemUnmap", &api.unmap) &&
                 entry("cuMemSetAccess", &api.set_access);
    });
    return api;
}

cudaError_t to_cuda(CUresult r) {
    if (r == CUDA_SUCCESS) return cudaSuccess;
    return r == CUDA_ERROR_OUT_OF_MEMORY ? cudaErrorMemoryAllocation : cudaErrorUnknown;
}

size_t round_up(size_t x, size_t g) { return (x + g - 1) / g * g; }

}  // namespace

size_t quad_block_offset(int x, int y) {
    return static_cast<size_t>(x & 255) | (static_cast<size_t>(y & 255) << 8) | (static_cast<size_t>(x >> 8) << 16) |
           (static_cast<size_t>(y >> 8) << 24);
}

void free_quads(QuadPlane* q) {
    const VmmApi& api = vmm();
    if (q->base && api.ok) {
        const CUdeviceptr base = reinterpret_cast<CUdeviceptr>(q->base);
        for (size_t i = 0; i < q->handles.size(); ++i) {
            if (q->mapped[i]) api.unmap(base + q->offsets[i], q->sizes[i]);
            api.release(static_cast<CUmemGenericAllocationHandle>(q->handles[i]));
        }
        api.address_free(base, q->reserved);
    }
    *q = QuadPlane();
}

cudaError_t alloc_quads(int device, int W, int H, QuadPlane* q) {
    *q = QuadPlane();
    const VmmApi& api = vmm();
    if (!api.ok) return cudaErrorNotSupported;
    CUmemAllocationProp prop{};
    prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
    prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
    prop.location.id = device;
    size_t g = 0;
    cudaError_t e = to_cuda(api.granularity(&g, &prop, CU_MEM_ALLOC_GRANULARITY_MINIMUM));
    if (e != cudaSuccess) return e;
    const int block_rows = ((H - 1) >> 8) + 1;
    const size_t row_bytes = round_up((static_cast<size_t>((W - 1) >> 8) + 1) * (size_t(1) << 16) * sizeof(uint2), g);
    const size_t row_stride = (size_t(1) << 24) * sizeof(uint2);
    q->reserved = static_cast<size_t>(block_rows - 1) * row_stride + row_bytes;
    CUdeviceptr base = 0;
    if ((e = to_cuda(api.reserve(&base, q->reserved, 0, 0, 0))) != cudaSuccess) {
        *q = QuadPlane();
        return e;
    }
    q->base = reinterpret_cast<uint2*>(base);
    CUmemAccessDesc access{};
    access.location = prop.location;
    access.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
    for (int r = 0; r < block_rows; ++r) {
        CUmemGenericAllocationHandle h = 0;
        if ((e = to_cuda(api.create(&h, row_bytes, &prop, 0))) != cudaSuccess) break;
        q->handles.push_back(static_cast<unsigned long long>(h));
        q->offsets.push_back(static_cast<size_t>(r) * row_stride);
        q->sizes.push_back(row_bytes);
        q->mapped.push_back(0);
        if ((e = to_cuda(api.map(base + q->offsets.back(), row_bytes, 0, h, 0))) != cudaSuccess) break;
        q->mapped.back() = 1;
        if ((e = to_cuda(api.set_access(base + q->offsets.back(), row_bytes, &access, 1))) != cudaSuccess) break;
        q->physical += row_bytes;
    }
    if (e != cudaSuccess) free_quads(q);
    return e;
}

}  // namespace hpx
