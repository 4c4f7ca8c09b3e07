// FP16-storage / FP32-accumulate PatchMatch kernels for sm_100a: the 64 x 8
// tile instantiation of hp_f16.cuh and the launchers of both tile heights
// (64 x 4 is instantiated in hp_kernels_f16t4.cu).
#include "hp_f16.cuh"

namespace hp {

#ifdef HP_COUNT_TAPS
unsigned long long f16_taps_th8() { return f16::taps_read_reset(); }
#endif
#ifdef HP_SELF_CHECK
cudaError_t f16_check_th8(int* out) { return check_read_reset(out); }
#endif

cudaError_t f16_dispatch_th8(int mode, int radius, int stride, int staging, const BatchList* bl,
                             const SolveConsts& sc, int iteration, int color, const Schedule* s, int grid,
                             cudaStream_t st, int* occ) {
    return f16::Dispatch<8>::go(mode, radius, stride, staging, bl, sc, iteration, color, s, grid, st, occ);
}

namespace {

cudaError_t dispatch(int mode, int tile_h, const SolveConsts& sc, const BatchList* bl, int iteration, int color,
                     const Schedule* s, int grid, cudaStream_t st, int* occ) {
    if (tile_h == 8)
        return f16_dispatch_th8(mode, sc.radius, sc.stride, sc.staging, bl, sc, iteration, color, s, grid, st, occ);
    if (tile_h == 4)
        return f16_dispatch_th4(mode, sc.radius, sc.stride, sc.staging, bl, sc, iteration, color, s, grid, st, occ);
    return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_cost_f16(const BatchList& bl, const SolveConsts& sc, cudaStream_t st) {
    if (bl.total_tiles <= 0) return cudaSuccess;
    return dispatch(0, sc.tile_h, sc, &bl, 0, 0, nullptr, 0, st, nullptr);
}

cudaError_t launch_propagate_f16(const BatchList& bl, const SolveConsts& sc, int iteration, int color,
                                 cudaStream_t st) {
    if (bl.total_tiles <= 0) return cudaSuccess;
    return dispatch(1, sc.tile_h, sc, &bl, iteration, color, nullptr, 0, st, nullptr);
}

cudaError_t launch_persistent_f16(const Schedule& s, int grid, cudaStream_t st) {
    if (s.total <= 0 || grid <= 0) return cudaSuccess;
    Schedule k = s;
    if (!k.abort) k.abort = k.status + 1;
    return dispatch(2, k.sc.tile_h, k.sc, nullptr, 0, 0, &k, grid, st, nullptr);
}

cudaError_t persistent_occupancy_f16(const SolveConsts& sc, int* blocks_per_sm) {
    return dispatch(2, sc.tile_h, sc, nullptr, 0, 0, nullptr, 0, nullptr, blocks_per_sm);
}

}  // namespace hp

#ifdef HP_SELF_CHECK
namespace hp {
cudaError_t f16_check_th4(int* out);
}
// Self-checking builds only: the first failed range check of the FP16 kernels
// of each tile height since the last call (12 ints each: hits, kind, six
// integers, four floats as bits; hits 0 = none), then cleared.
extern "C" int hp_debug_check(int* th8, int* th4) {
    if (hp::f16_check_th8(th8) != cudaSuccess) return 1;
    return hp::f16_check_th4(th4) != cudaSuccess ? 1 : 0;
}
#endif

#ifdef HP_COUNT_TAPS
// Instrumented builds only: taps sampled by the FP32 and FP16 kernels since
// the last call (both counters are reset).
extern "C" int hp_debug_taps(unsigned long long* f32, unsigned long long* f16) {
    *f32 = hp::f32_taps();
    *f16 = hp::f16_taps_th8() + hp::f16_taps_th4();
    return 0;
}
#endif
