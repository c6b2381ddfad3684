// asl_kernels.cuh - advective semi-Lagrangian step in q (sm_100a), FP64 / FP32.
//
// Bolt's ASL solver in q (asl_operators.py:20-83, interpolation_routines.py:
// 9-56) splits two operators by Strang, Lie, SWSS or Jia splitting (timestep.py,
// operator_splitting_methods.py):
//   op_advect_q  every cell takes the value at the foot of its characteristic,
//                q - A_q dt with A_q = (p1, p2) (advection_terms.py:29-61): one
//                bicubic interpolation over the ghosted q-plane per p-cell;
//   op_solve_src f <- f_MB (instantaneous collisions) or one RK2 step
//                (integrators.py:6-13) of the BGK source -(f - f_MB)/tau.
// The interpolation is ArrayFire's approx2 with BICUBIC_SPLINE, a third-party
// kernel absent here: it is restated as the tensor product of 1-D Catmull-Rom
// cubics (Catmull and Rom 1974), the neighbouring samples clamped to the
// ghosted array and 0 where a foot lies outside it.  The displacement
// (p1 dt / dq1, p2 dt / dq2) depends on p only, so consecutive lanes (p) of a
// warp gather from nearby cells of the same rows.
#pragma once

#include "fvm_kernels.cuh"

namespace bolt {

// weights of the Catmull-Rom cubic through samples -1, 0, 1, 2 at t in [0, 1)
__device__ __forceinline__ void catmull_rom_w(double t, double (&w)[4]) {
    const double t2 = t * t, t3 = t * t * t;
    w[0] = 0.5 * ((-t + 2.0 * t2) - t3);
    w[1] = 0.5 * ((2.0 - 5.0 * t2) + 3.0 * t3);
    w[2] = 0.5 * ((t + 4.0 * t2) - 3.0 * t3);
    w[3] = 0.5 * (t3 - t2);
}

// a position in sample units on an axis of n samples: first sample, weights
// (0 weights when the position lies off the samples)
__device__ __forceinline__ bool catmull_rom_axis(double x, int n, int& i0, double (&w)[4]) {
    const bool off = !(x >= 0.0 && x <= double(n - 1));
    const double xs = fmin(fmax(x, 0.0), double(n - 1));
    const double fl = floor(xs);
    i0 = (int)fl;
    catmull_rom_w(xs - fl, w);
    return off;
}

// the q2 row, species and p-cell of thread e (see asl_q_kernel); true if a
// written value is not finite
template <typename T>
__device__ __forceinline__ bool asl_q_row(const AslArgs& a, long long e) {
    bool bad = false;
    const int p = (int)(e % a.Np);
    const long long r = e / a.Np;
    const int s = (int)(r % a.Ns), j = (int)(r / a.Ns);
    const int Ng = a.Ng, Nq1 = a.Nq1, Nq1g = a.Nq1 + 2 * Ng, Nq2g = a.Nq2 + 2 * Ng;
    const int ip1 = p % a.Np1, ip2 = (p / a.Np1) % a.Np2;
    const double v1 = a.sg.p1_start[s] + (0.5 + ip1) * a.sg.dp1[s];
    const double v2 = a.sg.p2_start[s] + (0.5 + ip2) * a.sg.dp2[s];
    // cell centres of the ghosted grid (calculate_q.py:7-41) and the foot of
    // the characteristic in sample units, as approx2's xp / yp mapping
    // computes it: ((q - A dt) - q_0) / (q_1 - q_0)
    const double q10 = a.q1_start + (0.5 - Ng) * a.dq1, q11 = a.q1_start + (1.5 - Ng) * a.dq1;
    const double q20 = a.q2_start + (0.5 - Ng) * a.dq2, q21 = a.q2_start + (1.5 - Ng) * a.dq2;
    const double qj = a.q2_start + (0.5 + j) * a.dq2;
    const double y = ((qj - v2 * a.dt) - q20) / (q21 - q20);
    int j0;
    double wyd[4];
    const bool offy = catmull_rom_axis(y, Nq2g, j0, wyd);
    // the foot of the row's first cell, its sample and weights
    const double x0 = ((a.q1_start + 0.5 * a.dq1 - v1 * a.dt) - q10) / (q11 - q10);
    const double fl0 = floor(x0);
    const int i00 = (int)fl0;
    double wxd[4];
    catmull_rom_w(x0 - fl0, wxd);
    T wx[4], wy[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        wx[c] = T(wxd[c]);
        wy[c] = T(wyd[c]);
    }
    const long long rowstride = (long long)a.Ns * a.Np;
    const long long colstride = rowstride * Nq1g;
    const T* f = static_cast<const T*>(a.f) + (long long)s * a.Np + p;
    const T* rows[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) rows[b] = f + min(max(j0 - 1 + b, 0), Nq2g - 1) * colstride;
    T* __restrict__ out = static_cast<T*>(a.out) + (j + Ng) * colstride +
                          (long long)Ng * rowstride + (long long)s * a.Np + p;
    // column c of the ghosted row, clamped
    auto col = [&](int b, int c) { return rows[b][min(max(c, 0), Nq1g - 1) * rowstride]; };
    // the cell's value from the window (0 where the foot lies off the array)
    auto cell = [&](const T (&w)[4][4], int i) {
        const double x = x0 + i;
        const bool off = offy || !(x >= 0.0 && x <= double(Nq1g - 1));
        T acc = T(0);
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            T row = T(0);
#pragma unroll
            for (int c = 0; c < 4; ++c) row = row + wx[c] * w[b][c];
            acc = acc + wy[b] * row;
        }
        return off ? T(0) : acc;
    };
    // window[b][c]: row b, column clamp(i00 + i - 1 + c) of cell i
    T win[4][4];
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) win[b][c + 1] = col(b, i00 - 1 + c);
    int i = 0;
    // G cells per round (8 in FP32, 4 in FP64): their 4 G new samples are all
    // loaded before the first of the G cells is computed and stored (the
    // interpolation is latency-bound: many loads in flight per thread pay
    // more than occupancy)
    constexpr int G = sizeof(T) == 4 ? 8 : 4;
    for (; i + G <= Nq1; i += G) {
        T nc[G][4];
#pragma unroll
        for (int u = 0; u < G; ++u)
#pragma unroll
            for (int b = 0; b < 4; ++b) nc[u][b] = col(b, i00 + i + u + 2);
#pragma unroll
        for (int u = 0; u < G; ++u) {
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                win[b][0] = win[b][1];
                win[b][1] = win[b][2];
                win[b][2] = win[b][3];
                win[b][3] = nc[u][b];
            }
            const T v = cell(win, i + u);
            out[(long long)(i + u) * rowstride] = v;
            bad |= !isfinite(double(v));
        }
    }
    for (; i < Nq1; ++i) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            win[b][0] = win[b][1];
            win[b][1] = win[b][2];
            win[b][2] = win[b][3];
            win[b][3] = col(b, i00 + i + 2);
        }
        const T v = cell(win, i);
        out[(long long)i * rowstride] = v;
        bad |= !isfinite(double(v));
    }
    return bad;
}

// One thread per (interior q2 row j, species s, p-cell p), p fastest across
// lanes, walking the row's q1 cells.  The feet of a thread's cells are its
// first foot plus 0, 1, 2, ... samples (the displacement depends on p only),
// so the weights are computed once and the 4 x 4 source window slides along
// q1: each cell loads one new column of 4 samples (neighbours clamped to the
// ghosted array; a foot off the array gives 0).  Arithmetic in T.  A written
// value that is not finite sets *flag (one atomic per warp that saw one).
template <typename T>
__global__ void __launch_bounds__(256) asl_q_kernel(const AslArgs a, int* flag) {
    const long long nthr = (long long)a.Nq2 * a.Ns * a.Np;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool bad = e < nthr && asl_q_row<T>(a, e);
    if (flag && __any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// the BGK source of one interior q-cell of species blockIdx.y (blockIdx.x =
// q-cell): mode 0, out = base + c * (-(in - f_MB) / tau) with f_MB from the
// moments of `in` (a.mom_in, one partial slot); mode 1, out = f_MB.  The
// Maxwellian is the product of its per-axis factors, tabulated once per
// q-cell (the p1 factor carries n times the normalisation).  With mom_out,
// the five moment sums of the written values go to that partial slot (the
// next source evaluation needs no separate moment pass).  The p-block is
// streamed in 16-byte vectors when N_p1 is a multiple of the vector width and
// the buffers are 16-byte aligned; four CTAs per SM (at most 64 registers)
// overlap one CTA's Maxwellian set-up with the others' streaming.
constexpr int kAslMaxTab = 768;
template <typename T>
__global__ void __launch_bounds__(256, 4) asl_src_kernel(const QStageArgs a, const void* in,
                                                         const void* base, void* out, double c,
                                                         int mode, int* flag, double* mom_out) {
    __shared__ double qq[5];
    __shared__ double vg[kAslMaxTab];
    __shared__ double tab[kAslMaxTab];
    __shared__ double red[8][kNumMom];
    const int cell = blockIdx.x, s = blockIdx.y, tid = threadIdx.x;
    const int ii = cell % a.Nq1, jj = cell / a.Nq1;
    const int Np1 = a.Np1, Np2 = a.Np2, Np3 = a.Np3;
    const int ntab = Np1 + Np2 + Np3;             // <= kAslMaxTab (checked by the host)
    const long long rowstride = (long long)a.Ns * a.Np;
    const long long colstride = rowstride * a.Nq1g;
    const long long o = (jj + a.Ng) * colstride + (ii + a.Ng) * rowstride + (long long)s * a.Np;
    const T* fi = static_cast<const T*>(in) + o;
    const T* fb = static_cast<const T*>(base) + o;
    T* fo = static_cast<T*>(out) + o;
    typedef Vec16<T> VT;
    typedef typename VT::V V;
    constexpr int VN = VT::n;
    const bool vec = Np1 % VN == 0 &&
                     ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(base) |
                       reinterpret_cast<uintptr_t>(out)) & 15) == 0;
    const V* vi = reinterpret_cast<const V*>(fi);
    const V* vb = reinterpret_cast<const V*>(fb);
    const int nv = a.Np / VN;
    if (tid == 0) bgk_cell_params(a, s, ii, jj, qq);
    for (int q = tid; q < ntab; q += blockDim.x) {
        if (q < Np1) vg[q] = a.sg.p1_start[s] + (0.5 + q) * a.sg.dp1[s];
        else if (q < Np1 + Np2) vg[q] = a.sg.p2_start[s] + (0.5 + (q - Np1)) * a.sg.dp2[s];
        else vg[q] = a.sg.p3_start[s] + (0.5 + (q - Np1 - Np2)) * a.sg.dp3[s];
    }
    __syncthreads();
    const double m = a.sg.mass[s];
    for (int q = tid; q < ntab; q += blockDim.x) tab[q] = bgk_table_entry(a, qq, vg, q, m);
    __syncthreads();
    const double inv_tau = 1.0 / a.tau;
    const double dp1 = a.sg.dp1[s];
    bool bad = false;
    double acc[kNumMom] = {0, 0, 0, 0, 0};
    // the value written at p-cell (i1, i2, i3) from its input and base values
    auto value = [&](double f0, double vin, double vbase) -> T {
        return mode == 1 ? T(f0) : T(vbase + (-(vin - f0) * inv_tau) * c);
    };
    if (vec) {
        V* vo = reinterpret_cast<V*>(fo);
        // two vectors of input and base per round, loaded before either is
        // written (out may be base: every element is read, then written, by
        // one thread)
        for (int c0 = tid; c0 < nv; c0 += 2 * 256) {
            V ci[2], cb[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                if (c0 + u * 256 < nv && mode != 1) {
                    ci[u] = vi[c0 + u * 256];
                    cb[u] = fb == fi ? ci[u] : vb[c0 + u * 256];
                }
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int cv = c0 + u * 256;
                if (cv >= nv) break;
                const int p = cv * VN;
                const int ip1 = p % Np1, ip2 = (p / Np1) % Np2, ip3 = p / (Np1 * Np2);
                double di[VN], db[VN], ov[VN];
                if (mode != 1) {
                    VT::get(ci[u], di);
                    VT::get(cb[u], db);
                }
                T w[VN];
#pragma unroll
                for (int t = 0; t < VN; ++t) {
                    const double f0 = (tab[ip1 + t] * tab[Np1 + ip2]) * tab[Np1 + Np2 + ip3];
                    w[t] = value(f0, mode == 1 ? 0.0 : di[t], mode == 1 ? 0.0 : db[t]);
                    ov[t] = double(w[t]);
                    bad |= !isfinite(ov[t]);
                }
                V wv;
                if constexpr (VN == 4) wv = make_float4(w[0], w[1], w[2], w[3]);
                else wv = make_double2(w[0], w[1]);
                vo[cv] = wv;
                if (mom_out)
                    add_moment_run<VN>(ov, vg[ip1], dp1, vg[Np1 + ip2], vg[Np1 + Np2 + ip3], acc);
            }
        }
    } else {
        for (int p = tid; p < a.Np; p += blockDim.x) {
            const int ip1 = p % Np1, ip2 = (p / Np1) % Np2, ip3 = p / (Np1 * Np2);
            const double f0 = (tab[ip1] * tab[Np1 + ip2]) * tab[Np1 + Np2 + ip3];
            const T v = value(f0, mode == 1 ? 0.0 : double(fi[p]), mode == 1 ? 0.0 : double(fb[p]));
            fo[p] = v;
            const double ov[1] = {double(v)};
            bad |= !isfinite(ov[0]);
            if (mom_out)
                add_moment_run<1>(ov, vg[ip1], dp1, vg[Np1 + ip2], vg[Np1 + Np2 + ip3], acc);
        }
    }
    if (flag && __any_sync(0xffffffffu, bad) && (tid & 31) == 0) atomicOr(flag, 1);
    if (mom_out) {
#pragma unroll
        for (int q = 0; q < kNumMom; ++q) {
            const double v = warp_sum(acc[q]);
            if ((tid & 31) == 0) red[tid >> 5][q] = v;
        }
        __syncthreads();
        if (tid < kNumMom) {
            double v = 0.0;
            for (int w = 0; w < 8; ++w) v += red[w][tid];
            mom_out[((long long)tid * a.Ns + s) * a.Nq2 * a.Nq1 + (long long)jj * a.Nq1 + ii] = v;
        }
    }
}

}  // namespace bolt
