// FP64 throughput stage kernel (dtype BOLT_F64_FAST): the fused RK stage of
// qpair_kernel.cuh on FP64, one q-row per thread, built with FMA contraction
// (no -fmad=false) and Newton-refined reciprocals instead of IEEE divisions.  Its results
// differ from the reference-order FP64 kernels in rounding only.
#include "launch.h"
#include "qpair_kernel.cuh"

namespace bolt {

cudaError_t launch_qpair_f64(const QStageArgs& a, int bgk, int recon, dim3 grid, size_t smem,
                             cudaStream_t st) {
    return launch_qpair<double>(a, bgk, recon, grid, smem, st);
}

}  // namespace bolt
