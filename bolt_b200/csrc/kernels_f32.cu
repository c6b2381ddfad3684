// FP32 kernels: f and stencil arithmetic in FP32 with FMA and approximate
// reciprocals; moments, the BGK Maxwellian and the divergence check in FP64.
#define BOLT_T float
#define BOLT_EXACT false
#define BOLT_SUFFIX f32
#include "kernels_impl.cuh"
#include "qpair_kernel.cuh"

namespace bolt {

cudaError_t launch_qpair_f32(const QStageArgs& a, int bgk, int recon, dim3 grid, size_t smem,
                             cudaStream_t st) {
    return launch_qpair<float>(a, bgk, recon, grid, smem, st);
}

}  // namespace bolt
