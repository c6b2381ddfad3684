// FP32 kernels: f and stencil arithmetic in FP32 with FMA and approximate
// reciprocals; moments, the BGK Maxwellian and the divergence check in FP64.
#define BOLT_T float
#define BOLT_EXACT false
#define BOLT_SUFFIX f32
#include "kernels_impl.cuh"
#include "qpair_kernel.cuh"

namespace bolt {

template <int R>
static void (*pick_qpair(int bgk, int mode))(QStageArgs) {
    switch (mode) {
        case QP_X1: return bgk ? qpair_kernel<true, QP_X1, R> : qpair_kernel<false, QP_X1, R>;
        case QP_X2: return bgk ? qpair_kernel<true, QP_X2, R> : qpair_kernel<false, QP_X2, R>;
        case QP_B1: return bgk ? qpair_kernel<true, QP_B1, R> : qpair_kernel<false, QP_B1, R>;
        case QP_K: return bgk ? qpair_kernel<true, QP_K, R> : qpair_kernel<false, QP_K, R>;
        default: return bgk ? qpair_kernel<true, QP_B1R2, R> : qpair_kernel<false, QP_B1R2, R>;
    }
}

cudaError_t launch_qpair_f32(const QStageArgs& a, int bgk, int recon, dim3 grid, size_t smem,
                             cudaStream_t st) {
    const bool has2 = a.out2 != nullptr;
    // first RK4 / RK2 stage: the bases are the stage input
    const bool bx = a.base1 == a.fs && (!has2 || a.base2 == a.fs);
    int mode;
    if (a.base1 == nullptr && !has2) mode = QP_K;
    else if (bx) mode = has2 ? QP_X2 : QP_X1;
    else if (!has2) mode = QP_B1;
    else if (a.base2 == a.out2) mode = QP_B1R2;
    else return cudaErrorInvalidValue;        // excluded by the host's dispatch
    void (*k)(QStageArgs);
    switch (recon) {
        case BOLT_RECON_MINMOD: k = pick_qpair<BOLT_RECON_MINMOD>(bgk, mode); break;
        case BOLT_RECON_PPM: k = pick_qpair<BOLT_RECON_PPM>(bgk, mode); break;
        case BOLT_RECON_PC: k = pick_qpair<BOLT_RECON_PC>(bgk, mode); break;
        default: k = pick_qpair<BOLT_RECON_WENO5>(bgk, mode); break;
    }
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, NTHREADS, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace bolt
