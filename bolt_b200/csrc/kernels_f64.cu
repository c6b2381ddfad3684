// FP64 kernels in the reference's operation order.  Built with -fmad=false so
// that no multiply-add is contracted (the reference evaluates every product
// and sum separately).
#define BOLT_T double
#define BOLT_EXACT true
#define BOLT_SUFFIX f64
#include "kernels_impl.cuh"
#include "fdtd_kernels.cuh"

namespace bolt {

static unsigned field_blocks(const FieldArgs& a) {
    long long n = (long long)a.Nq1g * a.Nq2g;
    long long b = (n + 255) / 256;
    return (unsigned)(b < 1 ? 1 : (b > 1184 ? 1184 : b));
}

cudaError_t launch_field_halo(const FieldArgs& a, cudaStream_t st) {
    fdtd_halo_kernel<<<field_blocks(a), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_fdtd(const FieldArgs& a, cudaStream_t st, long long* launches) {
    const unsigned nb = field_blocks(a);
    fdtd_prepare_kernel<<<nb, 256, 0, st>>>(a);
    fdtd_halo_kernel<<<nb, 256, 0, st>>>(a);
    fdtd_e_kernel<<<nb, 256, 0, st>>>(a);
    fdtd_halo_kernel<<<nb, 256, 0, st>>>(a);
    fdtd_b_kernel<<<nb, 256, 0, st>>>(a);
    fdtd_to_cell_kernel<<<nb, 256, 0, st>>>(a);
    if (launches) *launches += 6;
    return cudaGetLastError();
}

}  // namespace bolt
