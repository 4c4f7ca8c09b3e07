// Self-checking builds (make check, -DHP_SELF_CHECK): range checks on the
// global accesses of the tile stages whose indices come from data or from
// descriptors.  A failed check records its first occurrence in this
// translation unit's g_check and the access is skipped (a quad load falls
// back to quad 0, a store is dropped), so a bad index shows up as a record
// instead of a fault.  In ordinary builds HP_CHECK is `true` and compiles away.
#pragma once

#include <cuda_runtime.h>

#ifdef HP_SELF_CHECK
namespace hp {
namespace {

// First failed check: kind, six integers and four floats describing it, and
// the number of failed checks since the last read.
struct CheckRec {
    int hits;
    int kind;
    int a[6];
    float f[4];
};
__device__ CheckRec g_check;

__device__ __noinline__ void check_fail(int kind, int a0, int a1, int a2, int a3, int a4, int a5, float f0,
                                        float f1, float f2, float f3) {
    if (atomicAdd(&g_check.hits, 1) != 0) return;
    volatile CheckRec* r = &g_check;
    r->kind = kind;
    r->a[0] = a0;
    r->a[1] = a1;
    r->a[2] = a2;
    r->a[3] = a3;
    r->a[4] = a4;
    r->a[5] = a5;
    r->f[0] = f0;
    r->f[1] = f1;
    r->f[2] = f2;
    r->f[3] = f3;
    __threadfence();
}

// Host: this translation unit's record (12 ints: hits, kind, a[6], f[4] as
// bits), then cleared.
inline cudaError_t check_read_reset(int* out) {
    CheckRec r{};
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpyFromSymbol(&r, g_check, sizeof r);
    if (e != cudaSuccess) return e;
    static_assert(sizeof(CheckRec) == 12 * sizeof(int), "record layout");
    __builtin_memcpy(out, &r, sizeof r);
    const CheckRec z{};
    return cudaMemcpyToSymbol(g_check, &z, sizeof z);
}

}  // namespace
}  // namespace hp
#define HP_CHECK(cond, kind, a0, a1, a2, a3, a4, a5, f0, f1, f2, f3) \
    ((cond) ? true : (::hp::check_fail((kind), (a0), (a1), (a2), (a3), (a4), (a5), (f0), (f1), (f2), (f3)), false))
#else
#define HP_CHECK(cond, kind, a0, a1, a2, a3, a4, a5, f0, f1, f2, f3) true
#endif

// Kinds of HP_CHECK records.
#define HP_CHECK_QUAD 1        // a quad load outside the source (x, y, xi, yi, checked form, tap; wx, wy, wz)
#define HP_CHECK_STATE 2       // a view's state pointers null or its size non-positive (W, H, stage, tile)
#define HP_CHECK_NEIGHBOUR 3   // a neighbour read outside the view (x, y, nx, ny, W, H)
#define HP_CHECK_TICKET 4      // a claimed tile or stage outside its view (view, stage, tile, tiles, iterations)
#define HP_CHECK_OUTPUT 5      // an output map pointer null at unpack (W, H, tile)
