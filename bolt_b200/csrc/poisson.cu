// poisson.cu - electrostatic fields of one df/dt argument (FP64).
//
// Bolt's electrostatic model re-solves the fields at every df/dt evaluation
// (df_dt_fvm.py:234-242): rho = sum_s charge_s * density_s(f), then the
// periodic FFT Poisson solve of fft.py:9-78 on the interior q-grid:
//   rho_hat = fft2(rho - mean(rho))
//   phi_hat = rho_hat / (4 pi^2 (k1^2 + k2^2)),  phi_hat[0, 0] = 0
//   E_d     = real(ifft2(-i 2 pi k_d phi_hat)) / (N_q1 N_q2) / eps,  d = 1, 2
// with k_d = numpy.fft.fftfreq(N_qd, dq_d), written into the cell-centred
// E1, E2 and their periodic ghost images (communicate_fields +
// apply_bcs_fields for periodic axes).  E3 and B keep their initial values.
//
// The two transforms are cuFFT double-complex plans over the (N_q2, N_q1)
// row-major q-grid (q1 fastest); the three small kernels around them read the
// species-density partial sums of moments5_kernel (split 0 of the
// [5][Ns][Nq2][Nq1] layout).

#include <cufft.h>

#include "launch.h"

namespace bolt {

namespace {

constexpr int kRhoThreads = 1024;

// rho of every interior q-cell minus its mean, as complex values.  One block:
// the q-grids of the electrostatic runs are small (N_q1 N_q2 <= a few 1e5).
__global__ void __launch_bounds__(kRhoThreads)
poisson_rho_kernel(PoissonArgs a) {
    __shared__ double red[kRhoThreads / 32];
    const int n = a.Nq1 * a.Nq2;
    double local = 0.0;
    for (int q = threadIdx.x; q < n; q += kRhoThreads) {
        double r = 0.0;
        for (int s = 0; s < a.Ns; ++s) {
            // charge * density; the density times initial_mu on the polar2D
            // grid (mom_scale; 1 on the cartesian grid, an exact product)
            const double dens = a.measure[s] * a.part[(long long)s * n + q];
            r += a.charge[s] * (a.mom_scale * dens);
        }
        a.rho_hat[q] = make_double2(r, 0.0);
        local += r;
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < kRhoThreads / 32 ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) red[0] = v;
    }
    __syncthreads();
    const double mean = red[0] / n;
    for (int q = threadIdx.x; q < n; q += kRhoThreads) a.rho_hat[q].x -= mean;
}

// numpy.fft.fftfreq(n, d)[k]
__device__ __forceinline__ double fft_freq(int k, int n, double d) {
    const int kk = k < (n + 1) / 2 ? k : k - n;
    return double(kk) * (1.0 / (double(n) * d));
}

// E1_hat, E2_hat of every mode from rho_hat
__global__ void poisson_spectral_kernel(PoissonArgs a) {
    const int n = a.Nq1 * a.Nq2;
    const double two_pi = 2.0 * 3.141592653589793;
    const double four_pi2 = 4.0 * (3.141592653589793 * 3.141592653589793);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int k1 = q % a.Nq1, k2 = q / a.Nq1;
        const double f1 = fft_freq(k1, a.Nq1, a.dq1), f2 = fft_freq(k2, a.Nq2, a.dq2);
        double2 ph = make_double2(0.0, 0.0);
        if (q != 0) {
            const double den = four_pi2 * (f1 * f1 + f2 * f2);
            ph = make_double2(a.rho_hat[q].x / den, a.rho_hat[q].y / den);
        }
        // -i 2 pi k phi_hat = 2 pi k (Im phi_hat, -Re phi_hat)
        const double c1 = two_pi * f1, c2 = two_pi * f2;
        a.e_hat[q] = make_double2(c1 * ph.y, -(c1 * ph.x));
        a.e_hat[n + q] = make_double2(c2 * ph.y, -(c2 * ph.x));
    }
}

// E1, E2 of every cell of the ghosted grid (ghosts: periodic images)
__global__ void poisson_fields_kernel(PoissonArgs a) {
    const int n = a.Nq1 * a.Nq2;
    const int Nq1g = a.Nq1 + 2 * a.Ng, Nq2g = a.Nq2 + 2 * a.Ng;
    const long long plane = (long long)Nq1g * Nq2g;
    const double scale = double(n);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < Nq1g * Nq2g;
         c += gridDim.x * blockDim.x) {
        const int g1 = c % Nq1g, g2 = c / Nq1g;
        const int i = ((g1 - a.Ng) % a.Nq1 + a.Nq1) % a.Nq1;
        const int j = ((g2 - a.Ng) % a.Nq2 + a.Nq2) % a.Nq2;
        const int q = j * a.Nq1 + i;
        a.cell[c] = (a.e_hat[q].x / scale) / a.eps;
        a.cell[plane + c] = (a.e_hat[n + q].x / scale) / a.eps;
    }
}

}  // namespace

int poisson_plans_create(int Nq1, int Nq2, int* fwd, int* inv) {
    cufftHandle p1 = 0, p2 = 0;
    if (cufftPlan2d(&p1, Nq2, Nq1, CUFFT_Z2Z) != CUFFT_SUCCESS) return 1;
    int dims[2] = {Nq2, Nq1};
    if (cufftPlanMany(&p2, 2, dims, nullptr, 1, Nq1 * Nq2, nullptr, 1, Nq1 * Nq2, CUFFT_Z2Z,
                      2) != CUFFT_SUCCESS) {
        cufftDestroy(p1);
        return 1;
    }
    *fwd = (int)p1;
    *inv = (int)p2;
    return 0;
}

void poisson_plans_destroy(int fwd, int inv) {
    if (fwd) cufftDestroy((cufftHandle)fwd);
    if (inv) cufftDestroy((cufftHandle)inv);
}

cudaError_t launch_poisson(const PoissonArgs& a, int fwd, int inv, cudaStream_t st,
                           long long* launches) {
    const int n = a.Nq1 * a.Nq2;
    poisson_rho_kernel<<<1, kRhoThreads, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cufftHandle pf = (cufftHandle)fwd, pi = (cufftHandle)inv;
    if (cufftSetStream(pf, st) != CUFFT_SUCCESS || cufftSetStream(pi, st) != CUFFT_SUCCESS)
        return cudaErrorUnknown;
    if (cufftExecZ2Z(pf, reinterpret_cast<cufftDoubleComplex*>(a.rho_hat),
                     reinterpret_cast<cufftDoubleComplex*>(a.rho_hat), CUFFT_FORWARD) !=
        CUFFT_SUCCESS)
        return cudaErrorUnknown;
    const int blocks = (n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8;
    poisson_spectral_kernel<<<blocks, 256, 0, st>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (cufftExecZ2Z(pi, reinterpret_cast<cufftDoubleComplex*>(a.e_hat),
                     reinterpret_cast<cufftDoubleComplex*>(a.e_hat), CUFFT_INVERSE) !=
        CUFFT_SUCCESS)
        return cudaErrorUnknown;
    const int ng = (a.Nq1 + 2 * a.Ng) * (a.Nq2 + 2 * a.Ng);
    const int fb = (ng + 255) / 256 < 148 * 8 ? (ng + 255) / 256 : 148 * 8;
    poisson_fields_kernel<<<fb, 256, 0, st>>>(a);
    *launches += 3;
    return cudaGetLastError();
}

}  // namespace bolt
