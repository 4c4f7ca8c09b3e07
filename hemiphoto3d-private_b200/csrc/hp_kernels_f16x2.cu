// FP16-storage / FP32-accumulate PatchMatch kernels for sm_100a, two lanes
// per (pixel, candidate) item (hp_f16.cuh, L = 2).  A separate translation
// unit so both layouts compile in parallel.
#include "hp_f16.cuh"

namespace hp {

cudaError_t f16_dispatch_l2(int mode, int radius, int stride, const BatchList* bl, const SolveConsts& sc,
                            int iteration, int color, const Schedule* s, int grid, cudaStream_t st, int* occ) {
    return f16::Dispatch<2>::go(mode, radius, stride, bl, sc, iteration, color, s, grid, st, occ);
}

}  // namespace hp
