// FP32 kernels: f and stencil arithmetic in FP32 with FMA and approximate
// reciprocals; moments, the BGK Maxwellian and the divergence check in FP64.
#define BOLT_T float
#define BOLT_EXACT false
#define BOLT_SUFFIX f32
#include "kernels_impl.cuh"
#include "qpair_kernel.cuh"

namespace bolt {

cudaError_t launch_qpair_f32(const QStageArgs& a, int bgk, dim3 grid, size_t smem,
                             cudaStream_t st) {
    const bool has2 = a.out2 != nullptr;
    // first RK4 stage: base1 (and base2) are the stage input
    const bool bx = a.base1 == a.fs && (!has2 || a.base2 == a.fs);
    void (*k)(QStageArgs);
    if (bx)
        k = bgk ? (has2 ? qpair_kernel<true, true, true> : qpair_kernel<true, false, true>)
                : (has2 ? qpair_kernel<false, true, true> : qpair_kernel<false, false, true>);
    else
        k = bgk ? (has2 ? qpair_kernel<true, true, false> : qpair_kernel<true, false, false>)
                : (has2 ? qpair_kernel<false, true, false> : qpair_kernel<false, false, false>);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, NTHREADS, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace bolt
