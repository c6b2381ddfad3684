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
    for (int part = 0; part < 3; ++part) {
        const cudaError_t e = launch_fdtd_part(a, part, st, launches);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// the FDTD update in three parts, each ending where the Yee ghosts of a
// block's external axes must come from its neighbours: 0 the currents and the
// halo before the E update, 1 the E update and the halo before the B update,
// 2 the B update and the cell-centred fields
cudaError_t launch_fdtd_part(const FieldArgs& a, int part, cudaStream_t st, long long* launches) {
    const unsigned nb = field_blocks(a);
    if (part == 0) {
        fdtd_prepare_kernel<<<nb, 256, 0, st>>>(a);
        fdtd_halo_kernel<<<nb, 256, 0, st>>>(a);
    } else if (part == 1) {
        fdtd_e_kernel<<<nb, 256, 0, st>>>(a);
        fdtd_halo_kernel<<<nb, 256, 0, st>>>(a);
    } else {
        fdtd_b_kernel<<<nb, 256, 0, st>>>(a);
        fdtd_to_cell_kernel<<<nb, 256, 0, st>>>(a);
    }
    if (launches) *launches += 2;
    return cudaGetLastError();
}

}  // namespace bolt
