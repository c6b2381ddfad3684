// fdtd_kernels.cuh - Yee-grid FDTD kernels (FP64), included by kernels_f64.cu only.
#pragma once

#include "fvm_common.cuh"
#include "fvm_args.h"

namespace bolt {

// ---------------------------------------------------------------------------
// Yee-grid FDTD (fdtd_explicit.py:9-177, fields.py:527-647).  Field arrays are
// [6][Nq2g][Nq1g] FP64; af.shift(a,0,0,s1,s2) neighbours wrap over the ghosted
// extent like the reference's circular shifts.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int wrapi(int x, int n) { return ((x % n) + n) % n; }

// J from partial sums (or the caller's J); copy of the cell-centred E before the update
__global__ void fdtd_prepare_kernel(FieldArgs a) {
    const int n = a.Nq1g * a.Nq2g;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int g1 = t % a.Nq1g, g2 = t / a.Nq1g;
        const int i = g1 - a.Ng, j = g2 - a.Ng;
        for (int c = 0; c < 3; ++c) {
            double v = 0.0;
            if (a.j_given) {
                v = a.j_given[c * n + t];
            } else if (i >= 0 && i < a.Nq1 && j >= 0 && j < a.Nq2) {
                // per species: charge * moment, the moment sum * measure
                // (times initial_mu on the polar2D grid); then the species sum
                for (int s = 0; s < a.Ns; ++s) {
                    double sum = 0.0;
                    for (int sp = 0; sp < a.nsplit; ++sp)
                        sum += a.jpart[(((long long)sp * 3 + c) * a.Ns + s) * a.Nq2 * a.Nq1
                                       + (long long)j * a.Nq1 + i];
                    const double mom = sum * a.measure[s];
                    v += a.charge[s] * (a.mom_scale * mom);
                }
            }
            a.J[c * n + t] = v;
            a.ebefore[c * n + t] = a.cell[c * n + t];
        }
    }
}

// periodic refresh of the 6 Yee components' halos (communicate_fields); the
// ghosts of an external axis (a block's cut), corners included, are the
// caller's: it exchanges them with the neighbouring blocks afterwards
__global__ void fdtd_halo_kernel(FieldArgs a) {
    const int n = a.Nq1g * a.Nq2g;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int g1 = t % a.Nq1g, g2 = t / a.Nq1g;
        const int i = g1 - a.Ng, j = g2 - a.Ng;
        const bool in1 = i >= 0 && i < a.Nq1, in2 = j >= 0 && j < a.Nq2;
        if (in1 && in2) continue;
        if ((!in1 && a.ext1) || (!in2 && a.ext2)) continue;
        const int si = wrapi(i, a.Nq1) + a.Ng, sj = wrapi(j, a.Nq2) + a.Ng;
        for (int c = 0; c < 6; ++c) a.yee[c * n + t] = a.yee[c * n + sj * a.Nq1g + si];
    }
}

// E += (dt/(mu eps)) curl B - J dt / eps   (fdtd_explicit.py:29-66)
__global__ void fdtd_e_kernel(FieldArgs a) {
    const int n = a.Nq1g * a.Nq2g;
    const double* B1 = a.yee + 3 * n;
    const double* B2 = a.yee + 4 * n;
    const double* B3 = a.yee + 5 * n;
    const double cf = a.dt / (a.mu * a.eps);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int g1 = t % a.Nq1g, g2 = t / a.Nq1g;
        const int p1 = g2 * a.Nq1g + wrapi(g1 + 1, a.Nq1g);     // shift(.., -1, 0)
        const int p2 = wrapi(g2 + 1, a.Nq2g) * a.Nq1g + g1;     // shift(.., 0, -1)
        const double curl1 = (B3[p2] - B3[t]) / a.dq2;
        const double curl2 = -(B3[p1] - B3[t]) / a.dq1;
        const double curl3 = (B2[p1] - B2[t]) / a.dq1 - (B1[p2] - B1[t]) / a.dq2;
        a.yee[0 * n + t] = a.yee[0 * n + t] + (cf * curl1 - (a.J[0 * n + t] * a.dt) / a.eps);
        a.yee[1 * n + t] = a.yee[1 * n + t] + (cf * curl2 - (a.J[1 * n + t] * a.dt) / a.eps);
        a.yee[2 * n + t] = a.yee[2 * n + t] + (cf * curl3 - (a.J[2 * n + t] * a.dt) / a.eps);
    }
}

// B -= dt curl E   (fdtd_explicit.py:100-129)
__global__ void fdtd_b_kernel(FieldArgs a) {
    const int n = a.Nq1g * a.Nq2g;
    const double* E1 = a.yee;
    const double* E2 = a.yee + n;
    const double* E3 = a.yee + 2 * n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int g1 = t % a.Nq1g, g2 = t / a.Nq1g;
        const int m1 = g2 * a.Nq1g + wrapi(g1 - 1, a.Nq1g);     // shift(.., 1, 0)
        const int m2 = wrapi(g2 - 1, a.Nq2g) * a.Nq1g + g1;     // shift(.., 0, 1)
        const double curl1 = (E3[t] - E3[m2]) / a.dq2;
        const double curl2 = -(E3[t] - E3[m1]) / a.dq1;
        const double curl3 = (E2[t] - E2[m1]) / a.dq1 - (E1[t] - E1[m2]) / a.dq2;
        a.yee[3 * n + t] = a.yee[3 * n + t] + -a.dt * curl1;
        a.yee[4 * n + t] = a.yee[4 * n + t] + -a.dt * curl2;
        a.yee[5 * n + t] = a.yee[5 * n + t] + -a.dt * curl3;
    }
}

// Yee -> cell centres; E becomes the average of the old and new values
// (the reference's three cell-centred arrays alias one object, so its
// E_at_n_plus_half write lands in the array that get_fields returns)
__global__ void fdtd_to_cell_kernel(FieldArgs a) {
    const int n = a.Nq1g * a.Nq2g;
    const double* y = a.yee;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int g1 = t % a.Nq1g, g2 = t / a.Nq1g;
        const int p1 = g2 * a.Nq1g + wrapi(g1 + 1, a.Nq1g);
        const int p2 = wrapi(g2 + 1, a.Nq2g) * a.Nq1g + g1;
        const int p12 = wrapi(g2 + 1, a.Nq2g) * a.Nq1g + wrapi(g1 + 1, a.Nq1g);
        const double e1 = 0.5 * (y[0 * n + t] + y[0 * n + p1]);
        const double e2 = 0.5 * (y[1 * n + t] + y[1 * n + p2]);
        const double e3 = y[2 * n + t];
        a.cell[0 * n + t] = 0.5 * (a.ebefore[0 * n + t] + e1);
        a.cell[1 * n + t] = 0.5 * (a.ebefore[1 * n + t] + e2);
        a.cell[2 * n + t] = 0.5 * (a.ebefore[2 * n + t] + e3);
        a.cell[3 * n + t] = 0.5 * (y[3 * n + t] + y[3 * n + p2]);
        a.cell[4 * n + t] = 0.5 * (y[4 * n + t] + y[4 * n + p1]);
        a.cell[5 * n + t] = 0.25 * (((y[5 * n + t] + y[5 * n + p2]) + y[5 * n + p1]) + y[5 * n + p12]);
    }
}

}  // namespace bolt
