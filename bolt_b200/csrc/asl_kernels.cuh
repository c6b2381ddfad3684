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

// q2 rows per interpolation thread: consecutive output rows of one p-cell
// have feet one sample apart in q2 (the displacement depends on p only), so
// R rows share R + 3 source rows.  G cells' samples are loaded together.
// Measured on 128^2 x 24^3 (the walk is latency-bound: more rows per thread
// cost registers and occupancy): FP32 2 rows, 4 cells as fast as 1 row, 8
// cells, 10 % ahead of 1 row, 4 or 6 cells and 2 rows, 2 cells; FP64 2 rows,
// 2 cells 11 % ahead of 1 row, 4 cells.
template <typename T> struct AslRows {
    static constexpr int R = 2;
    static constexpr int G = sizeof(T) == 4 ? 4 : 2;
};

// the q2 rows [R jb, R jb + R), species and p-cell of thread e (see
// asl_q_kernel); true if a written value is not finite.  I: the type of the
// element offsets from the thread's own (species, p) base -- int when the
// ghosted array holds fewer than 2^31 elements (fewer registers and no 64-bit
// multiplies in the walk), else long long
template <typename T, typename I>
__device__ __forceinline__ bool asl_q_rows(const AslArgs& a, long long e) {
    constexpr int R = AslRows<T>::R, NS = R + 3, G = AslRows<T>::G;
    bool bad = false;
    const int p = (int)(e % a.Np);
    const long long r = e / a.Np;
    const int s = (int)(r % a.Ns), jb = R * (int)(r / a.Ns);
    const int Ng = a.Ng, Nq1 = a.Nq1, Nq1g = a.Nq1 + 2 * Ng, Nq2g = a.Nq2 + 2 * Ng;
    const int nr = min(R, a.Nq2 - jb);                   // rows of this thread
    const int ip1 = p % a.Np1, ip2 = (p / a.Np1) % a.Np2;
    const double v1 = a.sg.p1_start[s] + (0.5 + ip1) * a.sg.dp1[s];
    const double v2 = a.sg.p2_start[s] + (0.5 + ip2) * a.sg.dp2[s];
    // cell centres of the ghosted grid (calculate_q.py:7-41) and the foot of
    // the characteristic in sample units, as approx2's xp / yp mapping
    // computes it: ((q - A dt) - q_0) / (q_1 - q_0); row jb + k has its foot
    // at y + k, cell i at x0 + i
    const double q10 = a.q1_start + (0.5 - Ng) * a.dq1, q11 = a.q1_start + (1.5 - Ng) * a.dq1;
    const double q20 = a.q2_start + (0.5 - Ng) * a.dq2, q21 = a.q2_start + (1.5 - Ng) * a.dq2;
    const double qj = a.q2_start + (0.5 + jb) * a.dq2;
    const double y = ((qj - v2 * a.dt) - q20) / (q21 - q20);
    const double x0 = ((a.q1_start + 0.5 * a.dq1 - v1 * a.dt) - q10) / (q11 - q10);
    // first samples and weights; the positions are clamped a few samples
    // beyond the ranges where some row or cell of the thread lies on the
    // array (beyond them every value is 0), which keeps the sample indices
    // exact where they matter and finite everywhere
    const double yc = fmin(fmax(y, -double(R + 4)), double(Nq2g + 4));
    const double xc = fmin(fmax(x0, -double(Nq1 + 4)), double(Nq1g + 4));
    const double fy = floor(yc), fl0 = floor(xc);
    const int j0 = (int)fy, i00 = (int)fl0;
    double wyd[4], wxd[4];
    catmull_rom_w(yc - fy, wyd);
    catmull_rom_w(xc - fl0, wxd);
    T wx[4], wy[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        wx[c] = T(wxd[c]);
        wy[c] = T(wyd[c]);
    }
    // an output row whose foot lies off the ghosted rows is 0
    bool offy[R];
#pragma unroll
    for (int k = 0; k < R; ++k) offy[k] = !(y + k >= 0.0 && y + k <= double(Nq2g - 1));
    const I rowstride = I(a.Ns) * I(a.Np);
    const I colstride = rowstride * I(Nq1g);
    const T* f = static_cast<const T*>(a.f) + (long long)s * a.Np + p;
    // source rows j0 - 1 .. j0 + R + 1, clamped to the ghosted array
    I rows[NS];
#pragma unroll
    for (int b = 0; b < NS; ++b) rows[b] = I(min(max(j0 - 1 + b, 0), Nq2g - 1)) * colstride;
    T* __restrict__ out = static_cast<T*>(a.out) + (long long)(jb + Ng) * colstride +
                          (long long)Ng * rowstride + (long long)s * a.Np + p;
    auto col = [&](int b, int c) { return f[rows[b] + I(min(max(c, 0), Nq1g - 1)) * rowstride]; };
    if constexpr (sizeof(T) == 4 && R == 2) {
        // FP32: the q1 cubics of source rows (0, 1) and (2, 3) as f32x2 pairs
        // (two FMAs per instruction, each lane the same operations in the
        // same order as the scalar form below, so the values are identical);
        // row 4 scalar
        float2 w01[4], w23[4];
        float w4[4];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            w01[c + 1] = make_float2(col(0, i00 - 1 + c), col(1, i00 - 1 + c));
            w23[c + 1] = make_float2(col(2, i00 - 1 + c), col(3, i00 - 1 + c));
            w4[c + 1] = col(4, i00 - 1 + c);
        }
        auto cell2 = [&](int i, float2 n01, float2 n23, float n4) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                w01[c] = w01[c + 1];
                w23[c] = w23[c + 1];
                w4[c] = w4[c + 1];
            }
            w01[3] = n01;
            w23[3] = n23;
            w4[3] = n4;
            float2 x01 = make_float2(0.0f, 0.0f), x23 = make_float2(0.0f, 0.0f);
            float x4 = 0.0f;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const float2 wc = make_float2(wx[c], wx[c]);
                x01 = __ffma2_rn(wc, w01[c], x01);
                x23 = __ffma2_rn(wc, w23[c], x23);
                x4 = x4 + wx[c] * w4[c];
            }
            const float xs[5] = {x01.x, x01.y, x23.x, x23.y, x4};
            const double x = x0 + i;
            const bool offx = !(x >= 0.0 && x <= double(Nq1g - 1));
#pragma unroll
            for (int k = 0; k < R; ++k) {
                if (k < nr) {
                    float acc = 0.0f;
#pragma unroll
                    for (int b = 0; b < 4; ++b) acc = acc + wy[b] * xs[k + b];
                    const float v = (offx || offy[k]) ? 0.0f : acc;
                    out[I(k) * colstride + I(i) * rowstride] = v;
                    bad |= !isfinite(v);
                }
            }
        };
        int i = 0;
        for (; i + G <= Nq1; i += G) {
            float2 n01[G], n23[G];
            float n4[G];
#pragma unroll
            for (int u = 0; u < G; ++u) {
                const int c = i00 + i + u + 2;
                n01[u] = make_float2(col(0, c), col(1, c));
                n23[u] = make_float2(col(2, c), col(3, c));
                n4[u] = col(4, c);
            }
#pragma unroll
            for (int u = 0; u < G; ++u) cell2(i + u, n01[u], n23[u], n4[u]);
        }
        for (; i < Nq1; ++i) {
            const int c = i00 + i + 2;
            cell2(i, make_float2(col(0, c), col(1, c)), make_float2(col(2, c), col(3, c)),
                  col(4, c));
        }
        return bad;
    }
    // win[b][c]: source row b, column clamp(i00 + i - 1 + c) of cell i
    T win[NS][4];
#pragma unroll
    for (int b = 0; b < NS; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) win[b][c + 1] = col(b, i00 - 1 + c);
    // cell i of every row: the window slid by one column, the q1 sums of the
    // source rows, then per output row k the q2 sum over rows k .. k+3
    auto cell = [&](int i, const T (&nc)[NS]) {
#pragma unroll
        for (int b = 0; b < NS; ++b) {
            win[b][0] = win[b][1];
            win[b][1] = win[b][2];
            win[b][2] = win[b][3];
            win[b][3] = nc[b];
        }
        T xs[NS];
#pragma unroll
        for (int b = 0; b < NS; ++b) {
            T row = T(0);
#pragma unroll
            for (int c = 0; c < 4; ++c) row = row + wx[c] * win[b][c];
            xs[b] = row;
        }
        const double x = x0 + i;
        const bool offx = !(x >= 0.0 && x <= double(Nq1g - 1));
#pragma unroll
        for (int k = 0; k < R; ++k) {
            if (k < nr) {
                T acc = T(0);
#pragma unroll
                for (int b = 0; b < 4; ++b) acc = acc + wy[b] * xs[k + b];
                const T v = (offx || offy[k]) ? T(0) : acc;
                out[I(k) * colstride + I(i) * rowstride] = v;
                bad |= !isfinite(v);
            }
        }
    };
    int i = 0;
    // G cells per round: their new samples are loaded before any is computed
    for (; i + G <= Nq1; i += G) {
        T nc[G][NS];
#pragma unroll
        for (int u = 0; u < G; ++u)
#pragma unroll
            for (int b = 0; b < NS; ++b) nc[u][b] = col(b, i00 + i + u + 2);
#pragma unroll
        for (int u = 0; u < G; ++u) cell(i + u, nc[u]);
    }
    for (; i < Nq1; ++i) {
        T nc[NS];
#pragma unroll
        for (int b = 0; b < NS; ++b) nc[b] = col(b, i00 + i + 2);
        cell(i, nc);
    }
    return bad;
}

// One thread per (block of R interior q2 rows, species s, p-cell p), p
// fastest across lanes, walking the rows' q1 cells.  The feet of a thread's
// cells are its first foot plus whole samples in q1 and q2 (the displacement
// depends on p only), so the weights are computed once, the R rows share
// R + 3 source rows, and the source window slides along q1: each cell loads
// one new column of R + 3 samples (neighbours clamped to the ghosted array;
// a foot off the array gives 0).  Arithmetic in T: per source row the q1
// cubic, then per output row the q2 cubic, the order of a tensor-product
// evaluation row by row.  A written value that is not finite sets *flag (one
// atomic per warp that saw one).
template <typename T, typename I>
__global__ void __launch_bounds__(256) asl_q_kernel(const AslArgs a, int* flag) {
    constexpr int R = AslRows<T>::R;
    const long long nthr = (long long)((a.Nq2 + R - 1) / R) * a.Ns * a.Np;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool bad = e < nthr && asl_q_rows<T, I>(a, e);
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
    // the first round's input and base vectors are loaded before the
    // Maxwellian set-up, so that their latency overlaps it
    V ci[2], cb[2];
    if (vec && mode != 1) {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            if (tid + u * 256 < nv) {
                ci[u] = vi[tid + u * 256];
                cb[u] = fb == fi ? ci[u] : vb[tid + u * 256];
            }
        }
    }
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
        // the vectors cv = tid, tid + 256, ... in that order: p-cell cv * VN
        PCellWalk pw(tid * VN, 256 * VN, Np1, Np2);
        for (int c0 = tid; c0 < nv; c0 += 2 * 256) {
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                if (c0 != tid && c0 + u * 256 < nv && mode != 1) {
                    ci[u] = vi[c0 + u * 256];
                    cb[u] = fb == fi ? ci[u] : vb[c0 + u * 256];
                }
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int cv = c0 + u * 256;
                if (cv >= nv) break;
                const int ip1 = pw.i1, ip2 = pw.i2, ip3 = pw.i3;
                pw.advance();
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
