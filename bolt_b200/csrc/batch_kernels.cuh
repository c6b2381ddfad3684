// batch_kernels.cuh - ragged batch of independent 1D1V runs (sm_100a, FP32 f,
// FP64 moments).
//
// Every run r keeps its own ghosted distribution f_r[q1g][p1] (N_g = 3,
// periodic in q1, p1 fastest) at element offset f_off in one packed buffer;
// the RK stage buffers use the same packing.  A stage is ONE launch over all
// runs: persistent CTAs take work items (run, q-tile of 4 cells per warp)
// from a queue, and each item walks all p-chunks of its tile, so its
// q-cells' velocity moments are complete when the item ends (no partial sums,
// no atomics on data).  The tile height (warps per CTA), the CTAs per SM and
// the queue order are the schedule the batch's autotuner chooses; every
// schedule computes each cell with the same operations in the same order.
//
// Per item and 32-wide p-chunk (one p per lane):
//   * the tile's rows plus 3 halo rows each side are staged in shared memory
//     by coalesced 128-byte row loads;
//   * warp w walks the faces of cells 4w..4w+3 with the sliding WENO5 walker
//     (upwind side per lane), -(F_i+1/2 - F_i-1/2)/dq1 (df_dt_fvm.py:56-89);
//   * BGK to the Maxwellian of the stage input (collision_operator.py:16-128,
//     p_dim = 1): parameters per q-cell in FP64 from the input moments, the
//     exponential per cell at FP32 accuracy;
//   * out1 = base1 + c1 dt k, out2 = base2 + c2 dt k (RK4 stage combine,
//     integrators.py:15-28), periodic ghost images of out1, FP64 moments of
//     out1 accumulated per thread across chunks, non-finite check.
#pragma once

#include "fvm_args.h"
#include "fvm_common.cuh"

namespace bolt {

constexpr int kBatchNg = 3;          // ghost width (WENO5 stencil +-2 and the face shift)
// a work item is a q-tile of 4 cells per warp; CTAs of 2, 4, 8 or 16 warps
constexpr int kBatchCellsPerWarp = 4;

struct BatchRunDev {
    long long f_off;       // element offset of the run's ghosted f in every packed buffer
    int mom_off;           // first q-cell of the run in the packed moment arrays
    int Nq1, Np1;
    double p1_start, dp1;  // p1 cell centres p1_start + (i + 1/2) dp1
    double v2c, v3c;       // the single p2 / p3 cell centre
    double measure;        // dp1 dp2 dp3
    double mass, kB;
    double dt, inv_dq1, inv_tau;
};

struct BatchStageArgs {
    const BatchRunDev* runs;
    const int2* items;     // (run, tile) in queue order
    int nitems;
    int* counter;          // work-queue head (zeroed before the launch)
    const float* fs;       // stage input (ghosted)
    const float* base1;    // out1 = base1 + a1 dt k
    const float* base2;    // out2 = base2 + a2 dt k (null: no out2)
    float* out1;
    float* out2;
    const double* mom_in;  // moments of fs [packed q-cell][5] (raw sums over p)
    double* mom_out;       // moments of out1, same layout
    int* flag;             // non-finite flag or null
    double a1, a2;
    int source;            // BGK on
};

// e^x to FP32 accuracy: Cody-Waite reduction x = n ln2 + r, |r| <= ln2/2, in
// FP64, then 2^(r/ln2) by the hardware base-2 exponential (ex2.approx,
// relative error ~2^-22) scaled by 2^n built from its exponent bits.  Results
// below the FP32 normal range are flushed to zero, above it are infinite.
__device__ __forceinline__ float batch_exp(double x) {
    if (x < -87.0) return 0.0f;
    if (x > 88.0) return __int_as_float(0x7f800000);
    const double log2e = 1.4426950408889634, ln2 = 0.6931471805599453;
    const double n = rint(x * log2e);
    const double r = fma(-n, ln2, x);
    float e;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(float(r * log2e)));
    return e * __int_as_float((int(n) + 127) << 23);
}

// Maxwellian parameters of one q-cell from its raw moment sums
// (collision_operator.py:102-118, f0 :49-65 with p_dim = 1):
// {n A, u1, -m / (2 kB T)}
__device__ __forceinline__ void batch_maxwell(const BatchRunDev& R, const double* mm,
                                              double* out) {
    const double eps = 1e-30;
    const double m = R.mass, kB = R.kB;
    const double n = mm[0] * R.measure;
    const double u1 = (mm[1] * R.measure) / (n + eps);
    const double u2 = (mm[2] * R.measure) / (n + eps);
    const double u3 = (mm[3] * R.measure) / (n + eps);
    const double E = mm[4] * R.measure;
    const double nm = n * m;
    const double T = ((((2.0 * (E * m) - nm * (u1 * u1)) - nm * (u2 * u2)) - nm * (u3 * u3)))
                     / (n + eps) + eps;                     // (1/p_dim) with p_dim = 1
    const double twokT = (2.0 * kB) * T;
    const double A = sqrt(m / ((2.0 * 3.141592653589793 * kB) * T));
    out[0] = n * A;
    out[1] = u1;
    out[2] = -m / twokT;
}

__device__ __forceinline__ void batch_moments_out(const BatchRunDev& R, double m0, double m1,
                                                  double e1, double* dst) {
    dst[0] = m0;
    dst[1] = m1;
    dst[2] = R.v2c * m0;
    dst[3] = R.v3c * m0;
    dst[4] = e1 + 0.5 * (R.v2c * R.v2c + R.v3c * R.v3c) * m0;
}

template <int NW>
__global__ void __launch_bounds__(NW * 32)
batch_stage_kernel(const BatchStageArgs a) {
    constexpr int TQ = NW * kBatchCellsPerWarp;
    constexpr int ROWS = TQ + 2 * kBatchNg;
    __shared__ float X[2][ROWS][PW];      // chunk c in X[c & 1]; chunk c+1 loads meanwhile
    __shared__ double par[TQ][3];
    __shared__ int item_s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    bool nonfinite = false;

    for (;;) {
        if (tid == 0) item_s = atomicAdd(a.counter, 1);
        __syncthreads();
        const int it = item_s;
        if (it >= a.nitems) break;
        const int2 rt = a.items[it];
        const BatchRunDev& R = a.runs[rt.x];
        const int Nq1 = R.Nq1, Np1 = R.Np1;
        const int i0 = rt.y * TQ;
        const int ncell = min(TQ, Nq1 - i0);
        const float* fs = a.fs + R.f_off;

        // Maxwellian parameters of the tile's cells (stage input's moments)
        if (a.source && tid < ncell) {
            const double* mm = a.mom_in + (long long)(R.mom_off + i0 + tid) * kNumMom;
            batch_maxwell(R, mm, par[tid]);
        }

        const int j0 = 4 * warp;                  // this warp's first local cell
        const bool active = j0 < ncell;           // N_q1 % 4 == 0: whole 4-cell segments
        const float inv_dq = float(R.inv_dq1);
        const float inv_tau = float(R.inv_tau);
        const float c1 = float(a.a1 * R.dt), c2 = float(a.a2 * R.dt);
        double acc[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};

        // the tile's rows of one p-chunk -> X[b], asynchronously (one group)
        auto issue = [&](int c, int b) {
            for (int row = warp; row < ncell + 2 * kBatchNg; row += NW)
                cp_async4(&X[b][row][lane], fs + (long long)(i0 + row) * Np1 + c * PW + lane);
            cp_async_commit();
        };
        const int nch = Np1 / PW;
        __syncthreads();                          // the previous item is done with X
        issue(0, 0);
        for (int c = 0; c < nch; ++c) {
            const int p = c * PW + lane;
            const int b = c & 1;
            // X[b ^ 1] was last read in chunk c-1, before its closing barrier
            if (c + 1 < nch) {
                issue(c + 1, b ^ 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();                      // chunk c's rows landed for every thread
            if (active) {
                const double V = R.p1_start + (0.5 + p) * R.dp1;
                const float v = float(V);
                const bool right = v > 0.0f;
                Weno5Side<float> S;
                S.set(right);
                Weno5Walker<false, float> W;
                const float (*Xb)[PW] = X[b];
                // the combine bases of this warp's 4 cells, loaded before the
                // stencil so that their latency overlaps it
                float b1v[4], b2v[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const long long o = R.f_off + (long long)(i0 + j0 + q + kBatchNg) * Np1 + p;
                    b1v[q] = a.base1[o];
                    b2v[q] = a.out2 ? a.base2[o] : 0.0f;
                }
                // face between local cells f and f+1 reads rows f+1+off .. f+5+off
                const int r0 = j0 + (right ? 0 : 1);
                float y0 = Xb[r0][lane], y1 = Xb[r0 + 1][lane], y2 = Xb[r0 + 2][lane];
                float y3 = Xb[r0 + 3][lane], y4 = Xb[r0 + 4][lane];
                float Fprev = v * W.first(y0, y1, y2, y3, y4, S);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int j = j0 + q;             // local cell
                    y0 = y1; y1 = y2; y2 = y3; y3 = y4;
                    y4 = Xb[r0 + 5 + q][lane];
                    const float Fn = v * W.next(y0, y1, y2, y3, y4, S);
                    float k = (Fprev - Fn) * inv_dq;
                    Fprev = Fn;
                    const float fc = Xb[j + kBatchNg][lane];
                    if (a.source) {
                        const double dv = V - par[j][1];
                        const float f0 = float(par[j][0]) * batch_exp(par[j][2] * (dv * dv));
                        k = fmaf(f0 - fc, inv_tau, k);
                    }
                    const long long o = R.f_off + (long long)(i0 + j + kBatchNg) * Np1 + p;
                    const float o1 = fmaf(k, c1, b1v[q]);
                    a.out1[o] = o1;
                    if (a.out2) a.out2[o] = fmaf(k, c2, b2v[q]);
                    // periodic images of the border cells (2 N_g <= N_q1)
                    const int ii = i0 + j;
                    if (ii < kBatchNg) a.out1[o + (long long)Nq1 * Np1] = o1;
                    else if (ii >= Nq1 - kBatchNg) a.out1[o - (long long)Nq1 * Np1] = o1;
                    nonfinite |= !isfinite(o1);
                    const double od = o1;
                    acc[q][0] += od;
                    acc[q][1] = fma(od, V, acc[q][1]);
                    acc[q][2] = fma(0.5 * od, V * V, acc[q][2]);
                }
            }
            __syncthreads();                      // X[b] reads done before it is refilled
        }
        if (active) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double m0 = warp_sum(acc[q][0]), m1 = warp_sum(acc[q][1]);
                const double e1 = warp_sum(acc[q][2]);
                if (lane == 0)
                    batch_moments_out(R, m0, m1, e1,
                                      a.mom_out + (long long)(R.mom_off + i0 + j0 + q) * kNumMom);
            }
        }
        __syncthreads();                          // item_s and par are reused
    }
    if (__syncthreads_or(nonfinite) && tid == 0 && a.flag) atomicOr(a.flag, 1);
}

// velocity moments of f for every run (the first stage after f is set)
template <int NW>
__global__ void __launch_bounds__(NW * 32)
batch_moments_kernel(const BatchRunDev* runs, const int2* items, int nitems, int* counter,
                     const float* f, double* mom) {
    constexpr int TQ = NW * kBatchCellsPerWarp;
    __shared__ int item_s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (;;) {
        if (tid == 0) item_s = atomicAdd(counter, 1);
        __syncthreads();
        const int it = item_s;
        if (it >= nitems) break;
        const int2 rt = items[it];
        const BatchRunDev& R = runs[rt.x];
        const int i0 = rt.y * TQ, ncell = min(TQ, R.Nq1 - i0);
        const int j0 = 4 * warp;
        if (j0 < ncell) {
            double acc[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (int p = lane; p < R.Np1; p += PW) {
                const double V = R.p1_start + (0.5 + p) * R.dp1;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const double o = f[R.f_off + (long long)(i0 + j0 + q + kBatchNg) * R.Np1 + p];
                    acc[q][0] += o;
                    acc[q][1] = fma(o, V, acc[q][1]);
                    acc[q][2] = fma(0.5 * o, V * V, acc[q][2]);
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double m0 = warp_sum(acc[q][0]), m1 = warp_sum(acc[q][1]);
                const double e1 = warp_sum(acc[q][2]);
                if (lane == 0)
                    batch_moments_out(R, m0, m1, e1,
                                      mom + (long long)(R.mom_off + i0 + j0 + q) * kNumMom);
            }
        }
        __syncthreads();
    }
}

// periodic ghost rows of every run (communicate_f + apply_bcs_f for periodic q1)
__global__ void batch_ghost_kernel(const BatchRunDev* runs, int nruns, float* f) {
    const int r = blockIdx.y;
    if (r >= nruns) return;
    const BatchRunDev& R = runs[r];
    const int n = 2 * kBatchNg * R.Np1;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int g = e / R.Np1, p = e % R.Np1;
        const int row = g < kBatchNg ? g : R.Nq1 + g;          // ghost row (ghosted index)
        const int src = g < kBatchNg ? row + R.Nq1 : row - R.Nq1;
        f[R.f_off + (long long)row * R.Np1 + p] = f[R.f_off + (long long)src * R.Np1 + p];
    }
}

}  // namespace bolt
