// adjoint_kernels.cuh - 1D1V forward RK4 and its hand-written adjoint
// (sm_100a; T = float or double).
//
// Problem: f[i][p] on N_q1 periodic q-cells x N_p1 p-cells (no ghost storage:
// neighbours wrap), p_dim = 1, one species, fields off.
//   L(g)_i,p = -(v_p/dq) (phi_i+1/2 - phi_i-1/2) + (f0[g]_i,p - g_i,p) / tau
// phi the reference's WENO5 face value on the upwind side of v_p
// (weno5.py:4-98 with eps = 1e-17 (1 + |a| + |b| + |c|); riemann.py:46-49 --
// the LLF flux with alpha = |v_p| reduces to it), f0 the Maxwellian of g's
// velocity moments (collision_operator.py:16-128, p_dim = 1, moments FP64).
// RK4 (integrators.py:15-28): k1 = L(f), k2 = L(f + dt/2 k1),
// k3 = L(f + dt/2 k2), k4 = L(f + dt k3), f' = f + dt/6 (k1 + 2k2 + 2k3 + k4).
//
// phi may also be the reference's minmod face (minmod.py:4-71: the theta = 2
// limited slope of the upwind cell, sign(0) = +1), differentiated by a
// subgradient: where the limiter's three arguments share a sign it passes the
// smallest magnitude and that argument (the first of equal magnitudes) gets
// derivative 1, elsewhere the slope is 0 and so is its derivative -- the
// one-sided derivative at every kink, hence an element of the Clarke
// subdifferential.
// The adjoint of a stage applies L'(g)^T to an adjoint field a:
//   * advection: phi_F enters L_F with -v/dq and L_F+1 with +v/dq, so
//     phibar_F = -(v/dq)(a_F - a_F+1); cell j receives phibar_F dphi_F/dy_j
//     for every face whose five-point window holds j, with the WENO weights
//     differentiated exactly, w_k = c_k / beta_k^2:
//     dphi/dy = sum_k [w_k du_k/dy + (u_k - phi) dw_k/dy] / sum_k w_k,
//     dw_k/dy = -2 c_k / beta_k^3 dbeta_k/dy (d|y|/dy = sign y, 0 at 0);
//     the upwind choice and alpha = |v| do not depend on f;
//   * BGK: -a/tau directly, plus (1/tau) dM/dg . G with G = sum_p a_p df0_p/dM
//     through n, u, T of the moments M = (sum g, sum g v, sum g v^2/2) dp;
//   * tau: sum a (-(f0 - g) / tau^2).
// One CTA per q-cell, threads over p (block reductions in FP64).
#pragma once

#include <cooperative_groups.h>

#include "fvm_common.cuh"

namespace bolt {

constexpr int kAdjThreads = 256;
constexpr int kAdjMaxNp = 2048;
// face reconstructions of the adjoint (the BOLT_RECON_* values)
constexpr int kAdjMinmod = 1;
constexpr int kAdjWeno5 = 3;

struct Adj1DArgs {
    int Nq1, Np1;
    double p1_start, dp1, inv_dq, dq1;
    double mass, kB, tau, measure;
};

template <typename T>
__device__ __forceinline__ T adj_sgn(T x) { return x > T(0) ? T(1) : (x < T(0) ? T(-1) : T(0)); }

// Smoothness indicator of (a, b, c).  FP64 evaluates the reference's expanded
// polynomial; FP32 the identical sum of squares 13/12 (a-2b+c)^2 +
// 1/4 (a-4b+3c)^2, because the expanded form cancels catastrophically in FP32
// on smooth data (it can fall to or below zero, where the weight derivative
// 1/beta is unbounded).
template <typename T>
__device__ __forceinline__ T adj_beta(T a, T b, T c) {
    const T eps = T(1e-17);
    const T floor_ = eps * (((T(1) + fabs(a)) + fabs(b)) + fabs(c));
    if (sizeof(T) == 4) {
        const T d1 = (a - T(2) * b) + c, d2 = (a - T(4) * b) + T(3) * c;
        return (T(13) / T(12)) * d1 * d1 + T(0.25) * d2 * d2 + floor_;
    }
    return (((((T(4) / T(3)) * a * a - (T(19) / T(3)) * a * b) + (T(25) / T(3)) * b * b)
             + (T(11) / T(3)) * a * c) - (T(31) / T(3)) * b * c) + (T(10) / T(3)) * c * c
           + floor_;
}

// d beta / d(a, b, c), in the same form as adj_beta
template <typename T>
__device__ __forceinline__ void adj_dbeta(T a, T b, T c, T* db) {
    const T eps = T(1e-17);
    if (sizeof(T) == 4) {
        const T d1 = (a - T(2) * b) + c, d2 = (a - T(4) * b) + T(3) * c;
        const T g1 = (T(13) / T(6)) * d1, g2 = T(0.5) * d2;
        db[0] = g1 + g2;
        db[1] = T(-2) * g1 - T(4) * g2;
        db[2] = g1 + T(3) * g2;
    } else {
        db[0] = (T(8) / T(3)) * a - (T(19) / T(3)) * b + (T(11) / T(3)) * c;
        db[1] = -(T(19) / T(3)) * a + (T(50) / T(3)) * b - (T(31) / T(3)) * c;
        db[2] = (T(11) / T(3)) * a - (T(31) / T(3)) * b + (T(20) / T(3)) * c;
    }
    db[0] += eps * adj_sgn(a);
    db[1] += eps * adj_sgn(b);
    db[2] += eps * adj_sgn(c);
}


// WENO5 face value of the window y[0..4] on the given side, and optionally
// its gradient d[0..4] (weno5.py:58-96)
template <typename T>
__device__ __forceinline__ T adj_weno(const T* y, bool right, T* d) {
    const T c1 = right ? T(1) / T(16) : T(5) / T(16);
    const T c2 = T(5) / T(8);
    const T c3 = right ? T(5) / T(16) : T(1) / T(16);
    // interpolants u_k = sum_j A[k][j] y_j (weno5.py:86-92)
    T A[3][5];
    for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 5; ++j) A[k][j] = T(0);
    if (right) {
        A[0][0] = T(0.375);  A[0][1] = T(-1.25); A[0][2] = T(1.875);
        A[1][1] = T(-0.125); A[1][2] = T(0.75);  A[1][3] = T(0.375);
        A[2][2] = T(0.375);  A[2][3] = T(0.75);  A[2][4] = T(-0.125);
    } else {
        A[0][0] = T(-0.125); A[0][1] = T(0.75);  A[0][2] = T(0.375);
        A[1][1] = T(0.375);  A[1][2] = T(0.75);  A[1][3] = T(-0.125);
        A[2][2] = T(1.875);  A[2][3] = T(-1.25); A[2][4] = T(0.375);
    }
    T u[3], beta[3], w[3];
    const T cc[3] = {c1, c2, c3};
    for (int k = 0; k < 3; ++k) {
        u[k] = A[k][0] * y[0] + A[k][1] * y[1] + A[k][2] * y[2] + A[k][3] * y[3] + A[k][4] * y[4];
        beta[k] = adj_beta(y[k], y[k + 1], y[k + 2]);
        w[k] = cc[k] / (beta[k] * beta[k]);
    }
    const T W = (w[0] + w[1]) + w[2];
    const T phi = ((w[0] * u[0] + w[1] * u[1]) + w[2] * u[2]) / W;
    if (d) {
        for (int j = 0; j < 5; ++j) d[j] = T(0);
        for (int k = 0; k < 3; ++k) {
            T db[3];
            adj_dbeta(y[k], y[k + 1], y[k + 2], db);
            // (u_k - phi) dw_k/dbeta_k / W with dw_k/dbeta_k = -2 w_k / beta_k, in an
            // order that stays finite for beta near its 1e-17 floor in FP32
            const T s = T(-2) * (u[k] - phi) * (w[k] / W) / beta[k];
            for (int j = 0; j < 5; ++j) d[j] += w[k] * A[k][j] / W;
            for (int t = 0; t < 3; ++t) d[k + t] += s * db[t];
        }
    }
    return phi;
}

// minmod face of the window y[0..4] (the upwind cell is y[2], its neighbours
// y[1], y[3]; y[0], y[4] unused) on the given side, and optionally its
// subgradient d[0..4] (minmod.py:4-71)
template <typename T>
__device__ __forceinline__ T adj_minmod(const T* y, bool right, T* d) {
    const T bwd = y[2] - y[1], fwd = y[3] - y[2];
    const T cen = bwd + fwd;
    const T x[3] = {T(2) * bwd, T(0.5) * cen, T(2) * fwd};
    const T sx = x[0] < T(0) ? T(-1) : T(1);
    const T sy = x[1] < T(0) ? T(-1) : T(1);
    const T sz = x[2] < T(0) ? T(-1) : T(1);
    const T m = fmin(fmin(fabs(x[0]), fabs(x[1])), fabs(x[2]));
    const T slope = T(0.25) * fabs(sx + sy) * (sx + sz) * m;
    const T half = right ? T(0.5) : T(-0.5);
    if (d) {
        for (int j = 0; j < 5; ++j) d[j] = T(0);
        d[2] = T(1);
        if (sx == sy && sx == sz) {
            // d slope / d x_k = 1 for the passed argument k; dx_k / dy
            const int k = fabs(x[0]) == m ? 0 : (fabs(x[1]) == m ? 1 : 2);
            if (k == 0) { d[1] -= half * T(2); d[2] += half * T(2); }
            else if (k == 1) { d[1] -= half * T(0.5); d[3] += half * T(0.5); }
            else { d[2] -= half * T(2); d[3] += half * T(2); }
        }
    }
    return y[2] + half * slope;
}

template <typename T, int RECON>
__device__ __forceinline__ T adj_face(const T* y, bool right, T* d) {
    if (RECON == kAdjMinmod) return adj_minmod<T>(y, right, d);
    return adj_weno<T>(y, right, d);
}

// FP64 block sum over the CTA (kAdjThreads threads)
__device__ __forceinline__ double adj_block_sum(double v, double* red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < kAdjThreads / 32; ++w) s += red[w];
    return s;
}

struct AdjMaxwell {
    double n, u, T, A, N;     // density, bulk velocity, temperature, normalisation, n + eps
};

// collision_operator.py:102-118 with p_dim = 1 and no p2 / p3 motion
__device__ __forceinline__ AdjMaxwell adj_maxwell(const Adj1DArgs& P, double m0, double m1,
                                                  double m2) {
    const double eps = 1e-30, m = P.mass, kB = P.kB;
    AdjMaxwell M;
    M.n = m0 * P.measure;
    M.N = M.n + eps;
    M.u = (m1 * P.measure) / M.N;
    const double E = m2 * P.measure;
    const double nm = M.n * m;
    M.T = (2.0 * (E * m) - nm * (M.u * M.u)) / M.N + eps;
    M.A = sqrt(m / ((2.0 * 3.141592653589793 * kB) * M.T));
    return M;
}

__device__ __forceinline__ double adj_f0(const Adj1DArgs& P, const AdjMaxwell& M, double v) {
    const double dv = v - M.u;
    return M.n * M.A * exp((-P.mass * (dv * dv)) / ((2.0 * P.kB) * M.T));
}

// periodic q-neighbour row
__device__ __forceinline__ int adj_wrap(int i, int n) { return ((i % n) + n) % n; }

// row i of k_out = L(f + c k_in) (k_in may be null), by one CTA
template <typename T, int RECON>
__device__ __forceinline__ void adj_stage_cell(const Adj1DArgs& P, const T* f, const T* k_in,
                                               T c, T* k_out, int i, double* red) {
    const int Np = P.Np1, Nq = P.Nq1;
    auto g = [&](int q, int p) -> T {
        const long long o = (long long)adj_wrap(q, Nq) * Np + p;
        return k_in ? f[o] + c * k_in[o] : f[o];
    };
    double m0 = 0, m1 = 0, m2 = 0;
    for (int p = threadIdx.x; p < Np; p += kAdjThreads) {
        const double v = P.p1_start + (0.5 + p) * P.dp1;
        const double x = g(i, p);
        m0 += x;
        m1 += x * v;
        m2 += 0.5 * x * (v * v);
    }
    m0 = adj_block_sum(m0, red);
    m1 = adj_block_sum(m1, red);
    m2 = adj_block_sum(m2, red);
    const AdjMaxwell M = adj_maxwell(P, m0, m1, m2);
    for (int p = threadIdx.x; p < Np; p += kAdjThreads) {
        const double vd = P.p1_start + (0.5 + p) * P.dp1;
        const T v = T(vd);
        const bool right = v > T(0);
        const int off = right ? 0 : 1;
        T y[5];
        // face i+1/2 (between i and i+1) and face i-1/2
        for (int t = 0; t < 5; ++t) y[t] = g(i - 2 + off + t, p);
        const T phr = adj_face<T, RECON>(y, right, nullptr);
        for (int t = 0; t < 5; ++t) y[t] = g(i - 3 + off + t, p);
        const T phl = adj_face<T, RECON>(y, right, nullptr);
        const T gi = g(i, p);
        T k = -(v * T(P.inv_dq)) * (phr - phl);
        if (P.tau > 0) k += (T(adj_f0(P, M, vd)) - gi) / T(P.tau);
        k_out[(long long)i * Np + p] = k;
    }
}

// k_out = L(f + c k_in), one CTA per q-cell
template <typename T, int RECON>
__global__ void __launch_bounds__(kAdjThreads)
adj_stage_kernel(const Adj1DArgs P, const T* f, const T* k_in, T c, T* k_out) {
    __shared__ double red[kAdjThreads / 32];
    adj_stage_cell<T, RECON>(P, f, k_in, c, k_out, blockIdx.x, red);
}

// f <- f + dt/6 (k1 + 2 k2 + 2 k3 + k4)
template <typename T>
__global__ void adj_combine_kernel(long long n, T* f, const T* k1, const T* k2, const T* k3,
                                   const T* k4, T dt6) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x)
        f[e] = f[e] + dt6 * (((k1[e] + T(2) * k2[e]) + T(2) * k3[e]) + k4[e]);
}

// density n_i = dp sum_p f (FP64), one CTA per q-cell
template <typename T>
__device__ __forceinline__ void adj_density_cell(const Adj1DArgs& P, const T* f, double* dens,
                                                 int i, double* red) {
    double s = 0;
    for (int p = threadIdx.x; p < P.Np1; p += kAdjThreads) s += f[(long long)i * P.Np1 + p];
    s = adj_block_sum(s, red);
    if (threadIdx.x == 0) dens[i] = s * P.measure;
}

template <typename T>
__global__ void __launch_bounds__(kAdjThreads)
adj_density_kernel(const Adj1DArgs P, const T* f, double* dens) {
    __shared__ double red[kAdjThreads / 32];
    adj_density_cell<T>(P, f, dens, blockIdx.x, red);
}

// J += w |nhat_1|^2, nhat_1 = (1/N_q1) sum_i n_i exp(-2 pi i x_i / L) over the
// cell centres; also stores (Re, Im) for the adjoint.  One CTA.
__device__ __forceinline__ void adj_mode_block(const Adj1DArgs& P, const double* dens, double w,
                                               double* J, double* reim, double* red) {
    double re = 0, im = 0;
    for (int i = threadIdx.x; i < P.Nq1; i += kAdjThreads) {
        const double th = 2.0 * 3.141592653589793 * (i + 0.5) / P.Nq1;
        re += dens[i] * cos(th);
        im -= dens[i] * sin(th);
    }
    re = adj_block_sum(re, red) / P.Nq1;
    im = adj_block_sum(im, red) / P.Nq1;
    if (threadIdx.x == 0) {
        *J += w * (re * re + im * im);
        if (reim) { reim[0] = re; reim[1] = im; }
    }
}

__global__ void __launch_bounds__(kAdjThreads)
adj_mode_kernel(const Adj1DArgs P, const double* dens, double w, double* J, double* reim) {
    __shared__ double red[kAdjThreads / 32];
    adj_mode_block(P, dens, w, J, reim, red);
}

// lam += w d|nhat_1|^2 / df (reim from adj_mode_kernel on the same f)
template <typename T>
__device__ __forceinline__ void adj_mode_adjoint_at(const Adj1DArgs& P, const double* reim,
                                                    double w, T* lam, long long e) {
    const int i = int(e / P.Np1);
    const double th = 2.0 * 3.141592653589793 * (i + 0.5) / P.Nq1;
    const double dn = (2.0 / P.Nq1) * (reim[0] * cos(th) - reim[1] * sin(th));
    lam[e] = lam[e] + T(w * dn * P.measure);
}

template <typename T>
__global__ void adj_mode_adjoint_kernel(const Adj1DArgs P, const double* reim, double w, T* lam) {
    const long long n = (long long)P.Nq1 * P.Np1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x)
        adj_mode_adjoint_at<T>(P, reim, w, lam, e);
}

// Row j of L'(g)^T a at g = f + c k_in: epi(o, value) receives every element
// (o its offset); returns sum_p a (-(f0 - g)/tau^2) of the row (thread 0)
template <typename T, int RECON, typename Epi>
__device__ __forceinline__ double adj_vjp_cell(const Adj1DArgs& P, const T* f, const T* k_in, T c,
                                               const T* a, int j, double* red, Epi epi) {
    const int Np = P.Np1, Nq = P.Nq1;
    auto g = [&](int q, int p) -> T {
        const long long o = (long long)adj_wrap(q, Nq) * Np + p;
        return k_in ? f[o] + c * k_in[o] : f[o];
    };
    auto ad = [&](int q, int p) -> T { return a[(long long)adj_wrap(q, Nq) * Np + p]; };

    // BGK part: moments of g in cell j and the sums over p of a df0/d(n, u, T)
    double m0 = 0, m1 = 0, m2 = 0;
    for (int p = threadIdx.x; p < Np; p += kAdjThreads) {
        const double v = P.p1_start + (0.5 + p) * P.dp1;
        const double x = g(j, p);
        m0 += x;
        m1 += x * v;
        m2 += 0.5 * x * (v * v);
    }
    m0 = adj_block_sum(m0, red);
    m1 = adj_block_sum(m1, red);
    m2 = adj_block_sum(m2, red);
    const bool bgk = P.tau > 0;
    const AdjMaxwell M = adj_maxwell(P, m0, m1, m2);
    double Sn = 0, Su = 0, ST = 0, St = 0;
    if (bgk) {
        const double m = P.mass, kB = P.kB;
        for (int p = threadIdx.x; p < Np; p += kAdjThreads) {
            const double v = P.p1_start + (0.5 + p) * P.dp1;
            const double f0 = adj_f0(P, M, v);
            const double av = ad(j, p);
            const double dv = v - M.u;
            Sn += av * (f0 / M.n);                                         // df0/dn
            Su += av * f0 * m * dv / (kB * M.T);                            // df0/du
            ST += av * f0 * (-0.5 / M.T + m * dv * dv / (2.0 * kB * M.T * M.T));  // df0/dT
            St += av * (-(f0 - double(g(j, p))) / (P.tau * P.tau));
        }
        Sn = adj_block_sum(Sn, red);
        Su = adj_block_sum(Su, red);
        ST = adj_block_sum(ST, red);
        St = adj_block_sum(St, red);
    }
    // (n, u, T) as functions of the raw sums (m0, m1, m2)
    const double meas = P.measure, m = P.mass, N = M.N;
    const double dn0 = meas;
    const double du0 = -M.u * meas / N, du1 = meas / N;
    const double E = m2 * meas, nm = M.n * m;
    const double Tnum = 2.0 * (E * m) - nm * (M.u * M.u);
    const double dT0 = ((-m * M.u * M.u * dn0 - 2.0 * nm * M.u * du0) * N - Tnum * dn0) / (N * N);
    const double dT1 = (-2.0 * nm * M.u * du1) / N;
    const double dT2 = (2.0 * m * meas) / N;
    const double G0 = Sn * dn0 + Su * du0 + ST * dT0;
    const double G1 = Su * du1 + ST * dT1;
    const double G2 = ST * dT2;

    for (int p = threadIdx.x; p < Np; p += kAdjThreads) {
        const double vd = P.p1_start + (0.5 + p) * P.dp1;
        const T v = T(vd);
        const bool right = v > T(0);
        const int off = right ? 0 : 1;
        const T k = -(v * T(P.inv_dq));
        T acc = T(0);
        // faces F = j-3 .. j+2: window cells F-2+off .. F+2+off
        for (int F = j - 3; F <= j + 2; ++F) {
            const int s0 = F - 2 + off, pos = j - s0;
            if (pos < 0 || pos > 4) continue;
            T y[5], d[5];
            for (int t = 0; t < 5; ++t) y[t] = g(s0 + t, p);
            adj_face<T, RECON>(y, right, d);
            const T phibar = k * (ad(F, p) - ad(F + 1, p));
            acc += phibar * d[pos];
        }
        double r = double(acc);
        if (bgk)
            r += (-double(ad(j, p)) + (G0 + G1 * vd + G2 * 0.5 * vd * vd)) / P.tau;
        epi((long long)j * Np + p, T(r));
    }
    return St;
}

// out = L'(g)^T a at g = f + c k_in; dtau_part[j] = sum_p a (-(f0 - g)/tau^2)
template <typename T, int RECON>
__global__ void __launch_bounds__(kAdjThreads)
adj_vjp_kernel(const Adj1DArgs P, const T* f, const T* k_in, T c, const T* a, T* out,
               double* dtau_part) {
    __shared__ double red[kAdjThreads / 32];
    const double St = adj_vjp_cell<T, RECON>(P, f, k_in, c, a, blockIdx.x, red,
                                             [&](long long o, T v) { out[o] = v; });
    if (threadIdx.x == 0) dtau_part[blockIdx.x] = St;
}

// ---------------------------------------------------------------------------
// Whole steps as single cooperative launches.  A 1D1V step is a chain of
// small dependent passes (4 stages and the combine forward; 3 stages, 4 VJPs
// and their combines backward), each a few microseconds of work over
// N_q1 x N_p1 cells; one launch per step, with grid-wide barriers between the
// passes, removes the launch gaps between them.  The grid never exceeds the
// co-resident CTAs (cudaLaunchCooperativeKernel refuses otherwise) and CTAs
// take q-rows by a grid-stride loop.  The passes are the per-row functions of
// the separate kernels above, in the same order, so the results are the same.
// ---------------------------------------------------------------------------
template <typename T, int RECON>
__global__ void __launch_bounds__(kAdjThreads)
adj_step_coop_kernel(const Adj1DArgs P, T* f, T* k1, T* k2, T* k3, T* k4, T dt, double* J,
                     double* dens, double Jw) {
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    __shared__ double red[kAdjThreads / 32];
    const int Nq = P.Nq1, Np = P.Np1;
    for (int i = blockIdx.x; i < Nq; i += gridDim.x)
        adj_stage_cell<T, RECON>(P, f, (const T*)nullptr, T(0), k1, i, red);
    grid.sync();
    for (int i = blockIdx.x; i < Nq; i += gridDim.x)
        adj_stage_cell<T, RECON>(P, f, k1, dt / T(2), k2, i, red);
    grid.sync();
    for (int i = blockIdx.x; i < Nq; i += gridDim.x)
        adj_stage_cell<T, RECON>(P, f, k2, dt / T(2), k3, i, red);
    grid.sync();
    for (int i = blockIdx.x; i < Nq; i += gridDim.x)
        adj_stage_cell<T, RECON>(P, f, k3, dt, k4, i, red);
    grid.sync();
    const T dt6 = dt / T(6);
    for (int i = blockIdx.x; i < Nq; i += gridDim.x)
        for (int p = threadIdx.x; p < Np; p += kAdjThreads) {
            const long long e = (long long)i * Np + p;
            f[e] = f[e] + dt6 * (((k1[e] + T(2) * k2[e]) + T(2) * k3[e]) + k4[e]);
        }
    if (J) {
        grid.sync();
        for (int i = blockIdx.x; i < Nq; i += gridDim.x) adj_density_cell<T>(P, f, dens, i, red);
        grid.sync();
        if (blockIdx.x == 0) adj_mode_block(P, dens, Jw, J, nullptr, red);
    }
}

// adjoint of one step (the order of bolt_adj1d_step_adjoint's separate
// launches): A and B alternate as the stage adjoint fields a_s; part holds
// the four stages' per-row dJ/dtau terms, summed in stage order at the end
template <typename T, int RECON>
__global__ void __launch_bounds__(kAdjThreads)
adj_step_adjoint_coop_kernel(const Adj1DArgs P, const T* f, T* lam, T* k1, T* k2, T* k3, T* A,
                             T* B, T* gacc, T dt, double* part, double* dtau, int obj_at_start,
                             double* dens, double* reim, double wobj) {
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    __shared__ double red[kAdjThreads / 32];
    const int Nq = P.Nq1, Np = P.Np1;
    // recompute the stages from f
    for (int i = blockIdx.x; i < Nq; i += gridDim.x)
        adj_stage_cell<T, RECON>(P, f, (const T*)nullptr, T(0), k1, i, red);
    grid.sync();
    for (int i = blockIdx.x; i < Nq; i += gridDim.x)
        adj_stage_cell<T, RECON>(P, f, k1, dt / T(2), k2, i, red);
    grid.sync();
    for (int i = blockIdx.x; i < Nq; i += gridDim.x) {
        adj_stage_cell<T, RECON>(P, f, k2, dt / T(2), k3, i, red);
        for (int p = threadIdx.x; p < Np; p += kAdjThreads) {     // a4 = dt/6 lam
            const long long e = (long long)i * Np + p;
            A[e] = (dt / T(6)) * lam[e];
        }
    }
    grid.sync();
    // stage 4 (state f + dt k3): gacc = lam + g4, a3 = dt/3 lam + dt g4
    for (int j = blockIdx.x; j < Nq; j += gridDim.x) {
        const double St = adj_vjp_cell<T, RECON>(P, f, k3, dt, A, j, red, [&](long long e, T g) {
            gacc[e] = T(1) * lam[e] + T(1) * g;
            B[e] = (dt / T(3)) * lam[e] + dt * g;
        });
        if (threadIdx.x == 0) part[j] = St;
    }
    grid.sync();
    // stage 3 (state f + dt/2 k2): gacc += g3, a2 = dt/3 lam + dt/2 g3
    for (int j = blockIdx.x; j < Nq; j += gridDim.x) {
        const double St = adj_vjp_cell<T, RECON>(P, f, k2, dt / T(2), B, j, red,
                                                 [&](long long e, T g) {
            gacc[e] = T(1) * gacc[e] + T(1) * g;
            A[e] = (dt / T(3)) * lam[e] + (dt / T(2)) * g;
        });
        if (threadIdx.x == 0) part[Nq + j] = St;
    }
    grid.sync();
    // stage 2 (state f + dt/2 k1): gacc += g2, a1 = dt/6 lam + dt/2 g2
    for (int j = blockIdx.x; j < Nq; j += gridDim.x) {
        const double St = adj_vjp_cell<T, RECON>(P, f, k1, dt / T(2), A, j, red,
                                                 [&](long long e, T g) {
            gacc[e] = T(1) * gacc[e] + T(1) * g;
            B[e] = (dt / T(6)) * lam[e] + (dt / T(2)) * g;
        });
        if (threadIdx.x == 0) part[2 * Nq + j] = St;
    }
    grid.sync();
    // stage 1 (state f): lam = gacc + g1
    for (int j = blockIdx.x; j < Nq; j += gridDim.x) {
        const double St = adj_vjp_cell<T, RECON>(P, f, (const T*)nullptr, T(0), B, j, red,
                                                 [&](long long e, T g) {
            lam[e] = T(1) * gacc[e] + T(1) * g;
        });
        if (threadIdx.x == 0) part[3 * Nq + j] = St;
    }
    if (dtau || obj_at_start) grid.sync();
    if (dtau && blockIdx.x == 0) {
        for (int s = 0; s < 4; ++s) {
            double v = 0;
            for (int i = threadIdx.x; i < Nq; i += kAdjThreads) v += part[s * Nq + i];
            v = adj_block_sum(v, red);
            if (threadIdx.x == 0) *dtau += v;
        }
    }
    if (obj_at_start) {
        for (int i = blockIdx.x; i < Nq; i += gridDim.x) adj_density_cell<T>(P, f, dens, i, red);
        grid.sync();
        if (blockIdx.x == 0) adj_mode_block(P, dens, 0.0, reim + 2, reim, red);
        grid.sync();
        const long long n = (long long)Nq * Np;
        for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
             e += (long long)gridDim.x * blockDim.x)
            adj_mode_adjoint_at<T>(P, reim, wobj, lam, e);
    }
}

}  // namespace bolt
