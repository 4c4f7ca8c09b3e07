// FP16-storage / FP32-accumulate PatchMatch kernels for sm_100a: the 64 x 4
// tile instantiation of hp_f16.cuh (128 threads, 4 warps per CTA; same
// results as 64 x 8), in its own translation unit so both compile in parallel.
#include "hp_f16.cuh"

namespace hp {

#ifdef HP_COUNT_TAPS
unsigned long long f16_taps_th4() { return f16::taps_read_reset(); }
#endif
#ifdef HP_SELF_CHECK
cudaError_t f16_check_th4(int* out) { return check_read_reset(out); }
#endif

cudaError_t f16_dispatch_th4(int mode, int radius, int stride, int staging, const BatchList* bl,
                             const SolveConsts& sc, int iteration, int color, const Schedule* s, int grid,
                             cudaStream_t st, int* occ) {
    return f16::Dispatch<4>::go(mode, radius, stride, staging, bl, sc, iteration, color, s, grid, st, occ);
}

}  // namespace hp
