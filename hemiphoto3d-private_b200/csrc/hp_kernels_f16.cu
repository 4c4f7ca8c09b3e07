// FP16-storage / FP32-accumulate PatchMatch kernels for sm_100a: the
// one-lane-per-item layout and the launchers of both layouts (the device code
// is in hp_f16.cuh; the two-lane layout is instantiated in hp_kernels_f16x2.cu).
#include "hp_f16.cuh"

namespace hp {

cudaError_t f16_dispatch_l1(int mode, int radius, int stride, const BatchList* bl, const SolveConsts& sc,
                            int iteration, int color, const Schedule* s, int grid, cudaStream_t st, int* occ) {
    return f16::Dispatch<1>::go(mode, radius, stride, bl, sc, iteration, color, s, grid, st, occ);
}

namespace {

cudaError_t dispatch(int mode, int lanes, int radius, int stride, const BatchList* bl, const SolveConsts& sc,
                     int iteration, int color, const Schedule* s, int grid, cudaStream_t st, int* occ) {
    if (lanes != 1 && lanes != 2) return cudaErrorInvalidValue;
    return lanes == 2 ? f16_dispatch_l2(mode, radius, stride, bl, sc, iteration, color, s, grid, st, occ)
                      : f16_dispatch_l1(mode, radius, stride, bl, sc, iteration, color, s, grid, st, occ);
}

}  // namespace

cudaError_t launch_cost_f16(const BatchList& bl, const SolveConsts& sc, cudaStream_t st) {
    if (bl.total_tiles <= 0) return cudaSuccess;
    return dispatch(0, sc.lanes, sc.radius, sc.stride, &bl, sc, 0, 0, nullptr, 0, st, nullptr);
}

cudaError_t launch_propagate_f16(const BatchList& bl, const SolveConsts& sc, int iteration, int color,
                                 cudaStream_t st) {
    if (bl.total_tiles <= 0) return cudaSuccess;
    return dispatch(1, sc.lanes, sc.radius, sc.stride, &bl, sc, iteration, color, nullptr, 0, st, nullptr);
}

cudaError_t launch_persistent_f16(const Schedule& s, int grid, cudaStream_t st) {
    if (s.total <= 0 || grid <= 0) return cudaSuccess;
    return dispatch(2, s.sc.lanes, s.sc.radius, s.sc.stride, nullptr, s.sc, 0, 0, &s, grid, st, nullptr);
}

cudaError_t persistent_occupancy_f16(int radius, int stride, int lanes, int* blocks_per_sm) {
    const SolveConsts none{};
    return dispatch(2, lanes, radius, stride, nullptr, none, 0, 0, nullptr, 0, nullptr, blocks_per_sm);
}

}  // namespace hp
