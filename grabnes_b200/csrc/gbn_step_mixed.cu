// Instantiations of the recursion's sparse-product kernels in mixed precision (complex64 vectors, FP32 values): real or complex
// values, rows per group 1, 2, 4, every split of the tile's right-hand sides over a row group's threads,
// the plain and the staged kernel and their variants (gbn_step.cuh).  One file per precision, so that
// the two halves compile in parallel.
#include "gbn_step.cuh"

namespace gbn {

StepFn step_kernel_mixed(bool cplx, int G, int rpt, int tpr, bool staged, StepVariant v)
{
    return cplx ? step_pick<float, true>(G, rpt, tpr, staged, v) : step_pick<float, false>(G, rpt, tpr, staged, v);
}

StepFn tiled_kernel_mixed(int G, int rpt, int tpr, int min_blocks)
{
    if (G == 1) return tiled_pick_g<float, 1>(rpt, tpr, min_blocks);
    if (G == 2) return tiled_pick_g<float, 2>(rpt, tpr, min_blocks);
    if (G == 4) return tiled_pick_g<float, 4>(rpt, tpr, min_blocks);
    return nullptr;
}

}  // namespace gbn
