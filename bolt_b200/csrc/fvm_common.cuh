// fvm_common.cuh - device helpers shared by the FVM kernels (sm_100a).
//
// Face reconstruction follows Bolt's reconstruction modules
// (bolt/lib/nonlinear/finite_volume/reconstruction/{weno5,ppm,minmod}.py and
// reconstruct.py:29-44).  Every method is evaluated for ONE cell, y2, from
// the five values y0..y4 = f[i-2..i+2] around it, and returns either its right
// face value (upwind side for C > 0) or its left face value (C <= 0), which is
// what riemann.py:46-49 selects.  The caller passes the per-lane window
// offset so the choice is branch-free inside a warp.
//
// Two arithmetic flavours:
//   * exact (FP64 parity build, compiled with -fmad=false): operation order
//     and constants identical to the reference expressions;
//   * fast (FP32 build): algebraically identical forms with FMA and
//     approximate reciprocals (WENO5 smoothness indicators in the factored
//     13/12 (a-2b+c)^2 + 1/4 (a-4b+3c)^2 form, which expands to the
//     reference's polynomial).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fvm_args.h"

#define BOLT_RECON_PC     0
#define BOLT_RECON_MINMOD 1
#define BOLT_RECON_PPM    2
#define BOLT_RECON_WENO5  3

namespace bolt {

// ---------------------------------------------------------------------------
// small math helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fast_rcp(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ double fast_rcp(double x) { return 1.0 / x; }

template <typename T> struct Consts;
template <> struct Consts<double> {
    static constexpr double c4_3 = 4.0 / 3.0, c19_3 = 19.0 / 3.0, c25_3 = 25.0 / 3.0,
                            c11_3 = 11.0 / 3.0, c31_3 = 31.0 / 3.0, c10_3 = 10.0 / 3.0;
};
template <> struct Consts<float> {
    static constexpr float c4_3 = 4.0f / 3.0f, c19_3 = 19.0f / 3.0f, c25_3 = 25.0f / 3.0f,
                           c11_3 = 11.0f / 3.0f, c31_3 = 31.0f / 3.0f, c10_3 = 10.0f / 3.0f;
};

// Per-lane WENO5 coefficient set: the reference's right-face constants
// (w = {1/16, 5/8, 5/16}/beta^2, u_r interpolants) when the lane's velocity
// is positive, the left-face set otherwise (weno5.py:74-92).
template <typename T>
struct Weno5Side {
    T num1, den1, num2, den2, num3, den3;      // w_k = num_k / ((den_k*beta_k)*beta_k)
    T cw1, cw2, cw3;                           // num_k / den_k (fast path)
    T a10, a11, a12, a20, a21, a22, a30, a31, a32;  // u_k = (a_k0 y + a_k1 y) + a_k2 y
    __device__ __forceinline__ void set(bool right) {
        cw2 = T(0.625);
        cw1 = right ? T(0.0625) : T(0.3125);
        cw3 = right ? T(0.3125) : T(0.0625);
        if (right) {
            num1 = T(1); den1 = T(16); num2 = T(5); den2 = T(8); num3 = T(5); den3 = T(16);
            a10 = T(0.375);  a11 = T(-1.25); a12 = T(1.875);
            a20 = T(-0.125); a21 = T(0.75);  a22 = T(0.375);
            a30 = T(0.375);  a31 = T(0.75);  a32 = T(-0.125);
        } else {
            num1 = T(5); den1 = T(16); num2 = T(5); den2 = T(8); num3 = T(1); den3 = T(16);
            a10 = T(-0.125); a11 = T(0.75);  a12 = T(0.375);
            a20 = T(0.375);  a21 = T(0.75);  a22 = T(-0.125);
            a30 = T(1.875);  a31 = T(-1.25); a32 = T(0.375);
        }
    }
};

// ---------------------------------------------------------------------------
// WENO5, exact reference order (weno5.py:58-96)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double weno_beta_exact(double a, double b, double c) {
    typedef Consts<double> K;
    double poly = ((((K::c4_3 * a * a - K::c19_3 * a * b) + K::c25_3 * b * b)
                    + K::c11_3 * a * c) - K::c31_3 * b * c) + K::c10_3 * c * c;
    return poly + 1e-17 * (((1.0 + fabs(a)) + fabs(b)) + fabs(c));
}

__device__ __forceinline__ double weno5_exact(double y0, double y1, double y2, double y3,
                                              double y4, const Weno5Side<double>& S) {
    double b1 = weno_beta_exact(y0, y1, y2);
    double b2 = weno_beta_exact(y1, y2, y3);
    double b3 = weno_beta_exact(y2, y3, y4);
    double w1 = S.num1 / ((S.den1 * b1) * b1);
    double w2 = S.num2 / ((S.den2 * b2) * b2);
    double w3 = S.num3 / ((S.den3 * b3) * b3);
    double den = (w1 + w2) + w3;
    double u1 = (S.a10 * y0 + S.a11 * y1) + S.a12 * y2;
    double u2 = (S.a20 * y1 + S.a21 * y2) + S.a22 * y3;
    double u3 = (S.a30 * y2 + S.a31 * y3) + S.a32 * y4;
    return ((w1 * u1 + w2 * u2) + w3 * u3) / den;
}

// WENO5, fast FP32 form
__device__ __forceinline__ float weno_beta_fast(float a, float b, float c) {
    float d1 = fmaf(-2.0f, b, a + c);           // a - 2b + c
    float d2 = fmaf(3.0f, c, fmaf(-4.0f, b, a));  // a - 4b + 3c
    float e = fmaf(1e-17f, fabsf(a) + fabsf(b) + fabsf(c), 1e-17f);
    return fmaf(13.0f / 12.0f * d1, d1, fmaf(0.25f * d2, d2, e));
}

__device__ __forceinline__ float weno5_fast(float y0, float y1, float y2, float y3, float y4,
                                            const Weno5Side<float>& S) {
    float r1 = fast_rcp(weno_beta_fast(y0, y1, y2));
    float r2 = fast_rcp(weno_beta_fast(y1, y2, y3));
    float r3 = fast_rcp(weno_beta_fast(y2, y3, y4));
    float w1 = S.cw1 * r1 * r1;
    float w2 = S.cw2 * r2 * r2;
    float w3 = S.cw3 * r3 * r3;
    float u1 = fmaf(S.a12, y2, fmaf(S.a11, y1, S.a10 * y0));
    float u2 = fmaf(S.a22, y3, fmaf(S.a21, y2, S.a20 * y1));
    float u3 = fmaf(S.a32, y4, fmaf(S.a31, y3, S.a30 * y2));
    float num = fmaf(w3, u3, fmaf(w2, u2, w1 * u1));
    return num * fast_rcp(w1 + w2 + w3);
}

// ---------------------------------------------------------------------------
// minmod / MC limiter, theta = 2 (minmod.py:4-71); sign(0) = +1
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T minmod_slope(T ym, T y, T yp) {
    T fwd = yp - y;
    T bwd = y - ym;
    T cen = bwd + fwd;
    T x = T(2) * bwd, yy = T(0.5) * cen, z = T(2) * fwd;
    T m = fmin(fmin(fabs(x), fabs(yy)), fabs(z));
    T sx = x < T(0) ? T(-1) : T(1);
    T sy = yy < T(0) ? T(-1) : T(1);
    T sz = z < T(0) ? T(-1) : T(1);
    return ((T(0.25) * fabs(sx + sy)) * (sx + sz)) * m;
}

// ---------------------------------------------------------------------------
// PPM (ppm.py:58-98): returns right (right=true) or left face of cell y2
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T ppm_dq(T D, T da, T db) {
    T zero = (db * da <= T(0)) ? T(1) : T(0);
    T sgn = (D > T(0)) ? T(1) : T(-1);
    return ((T(1) - zero) * sgn) * fmin(fabs(D), fmin(fabs(da), fabs(db)));
}

template <typename T>
__device__ __forceinline__ T ppm_face(T y0, T y1, T y2, T y3, T y4, bool right) {
    T d0 = T(2) * (y1 - y0), d1 = T(2) * (y2 - y1), d2 = T(2) * (y3 - y2), d3 = T(2) * (y4 - y3);
    T D1 = T(0.5) * (y2 - y0), D2 = T(0.5) * (y3 - y1), D3 = T(0.5) * (y4 - y2);
    T DQ1 = ppm_dq(D1, d0, d1), DQ2 = ppm_dq(D2, d1, d2), DQ3 = ppm_dq(D3, d2, d3);
    T left = T(0.5) * (y2 + y1) - (DQ2 - DQ1) / T(6);
    T rightv = T(0.5) * (y3 + y2) - (DQ3 - DQ2) / T(6);
    T c1 = ((rightv - y2) * (y2 - left) <= T(0)) ? T(1) : T(0);
    T qd = rightv - left;
    T qe = T(6) * (y2 - T(0.5) * (rightv + left));
    T c2 = (qd * (qd - qe) < T(0)) ? T(1) : T(0);
    T c3 = (qd * (qd + qe) < T(0)) ? T(1) : T(0);
    left = left * (T(1) - c1) + c1 * y2;
    rightv = rightv * (T(1) - c1) + c1 * y2;
    left = left * (T(1) - c2) + c2 * (T(3) * y2 - T(2) * rightv);
    rightv = (rightv * c2 + ((T(1) - c2) * rightv) * (T(1) - c3))
             + ((T(1) - c2) * c3) * (T(3) * y2 - T(2) * left);
    return right ? rightv : left;
}

// ---------------------------------------------------------------------------
// Unified face value of cell y2 (right face if `right`, else left face)
// ---------------------------------------------------------------------------
template <int RECON, bool EXACT, typename T>
__device__ __forceinline__ T face_value(T y0, T y1, T y2, T y3, T y4, bool right,
                                        const Weno5Side<T>& S) {
    if (RECON == BOLT_RECON_PC) {
        return y2;
    } else if (RECON == BOLT_RECON_MINMOD) {
        T s = minmod_slope(y1, y2, y3);
        return right ? y2 + T(0.5) * s : y2 - T(0.5) * s;
    } else if (RECON == BOLT_RECON_PPM) {
        return ppm_face(y0, y1, y2, y3, y4, right);
    } else {
        if constexpr (EXACT) {
            return weno5_exact(double(y0), double(y1), double(y2), double(y3), double(y4),
                               reinterpret_cast<const Weno5Side<double>&>(S));
        } else {
            return weno5_fast(y0, y1, y2, y3, y4, S);
        }
    }
}

// ---------------------------------------------------------------------------
// WENO5 along a sliding window.  Consecutive faces share two of their three
// substencils: beta_1 of face f+1 is beta_2 of face f and beta_2 of face f+1
// is beta_3 of face f, so each step computes one new smoothness indicator.
// The exact flavour reuses the identical FP64 values (bit-for-bit the same
// as recomputing them); the fast flavour carries 1/beta^2.
// ---------------------------------------------------------------------------
template <bool EXACT, typename T> struct Weno5Walker;

template <> struct Weno5Walker<true, double> {
    double b2, b3;
    __device__ __forceinline__ double eval(double b1, double y0, double y1, double y2, double y3,
                                           double y4, const Weno5Side<double>& S) {
        double w1 = S.num1 / ((S.den1 * b1) * b1);
        double w2 = S.num2 / ((S.den2 * b2) * b2);
        double w3 = S.num3 / ((S.den3 * b3) * b3);
        double den = (w1 + w2) + w3;
        double u1 = (S.a10 * y0 + S.a11 * y1) + S.a12 * y2;
        double u2 = (S.a20 * y1 + S.a21 * y2) + S.a22 * y3;
        double u3 = (S.a30 * y2 + S.a31 * y3) + S.a32 * y4;
        return ((w1 * u1 + w2 * u2) + w3 * u3) / den;
    }
    __device__ __forceinline__ double first(double y0, double y1, double y2, double y3, double y4,
                                            const Weno5Side<double>& S) {
        double b1 = weno_beta_exact(y0, y1, y2);
        b2 = weno_beta_exact(y1, y2, y3);
        b3 = weno_beta_exact(y2, y3, y4);
        return eval(b1, y0, y1, y2, y3, y4, S);
    }
    // window shifted by one cell: y0..y3 are the previous y1..y4
    __device__ __forceinline__ double next(double y0, double y1, double y2, double y3, double y4,
                                           const Weno5Side<double>& S) {
        double b1 = b2;
        b2 = b3;
        b3 = weno_beta_exact(y2, y3, y4);
        return eval(b1, y0, y1, y2, y3, y4, S);
    }
};

template <> struct Weno5Walker<false, float> {
    float q2, q3;              // 1/beta^2 of substencils 2 and 3
    __device__ __forceinline__ static float inv_sq(float b) {
        float r = fast_rcp(b);
        return r * r;
    }
    __device__ __forceinline__ float eval(float q1, float y0, float y1, float y2, float y3,
                                          float y4, const Weno5Side<float>& S) {
        float w1 = S.cw1 * q1, w2 = S.cw2 * q2, w3 = S.cw3 * q3;
        float u1 = fmaf(S.a12, y2, fmaf(S.a11, y1, S.a10 * y0));
        float u2 = fmaf(S.a22, y3, fmaf(S.a21, y2, S.a20 * y1));
        float u3 = fmaf(S.a32, y4, fmaf(S.a31, y3, S.a30 * y2));
        float num = fmaf(w3, u3, fmaf(w2, u2, w1 * u1));
        return num * fast_rcp(w1 + w2 + w3);
    }
    __device__ __forceinline__ float first(float y0, float y1, float y2, float y3, float y4,
                                           const Weno5Side<float>& S) {
        float q1 = inv_sq(weno_beta_fast(y0, y1, y2));
        q2 = inv_sq(weno_beta_fast(y1, y2, y3));
        q3 = inv_sq(weno_beta_fast(y2, y3, y4));
        return eval(q1, y0, y1, y2, y3, y4, S);
    }
    __device__ __forceinline__ float next(float y0, float y1, float y2, float y3, float y4,
                                          const Weno5Side<float>& S) {
        float q1 = q2;
        q2 = q3;
        q3 = inv_sq(weno_beta_fast(y2, y3, y4));
        return eval(q1, y0, y1, y2, y3, y4, S);
    }
};

// Face walker for any reconstruction: WENO5 carries state, the others are
// evaluated from the window directly.
template <int RECON, bool EXACT, typename T>
struct FaceWalker {
    Weno5Walker<EXACT, T> w;
    __device__ __forceinline__ T first(T y0, T y1, T y2, T y3, T y4, bool right,
                                       const Weno5Side<T>& S) {
        if (RECON == BOLT_RECON_WENO5) return w.first(y0, y1, y2, y3, y4, S);
        return face_value<RECON, EXACT>(y0, y1, y2, y3, y4, right, S);
    }
    __device__ __forceinline__ T next(T y0, T y1, T y2, T y3, T y4, bool right,
                                      const Weno5Side<T>& S) {
        if (RECON == BOLT_RECON_WENO5) return w.next(y0, y1, y2, y3, y4, S);
        return face_value<RECON, EXACT>(y0, y1, y2, y3, y4, right, S);
    }
};

// ---------------------------------------------------------------------------
// Paired WENO5 walker: two q-cells per thread at the same p.  FP32 pairs use
// the sm_100 f32x2 arithmetic; FP64 pairs are two scalar FP64 operations with
// FMA and a Newton-refined reciprocal.  The same walkers also run on a single
// FP64 value per thread (P = double), for the one-row-per-thread form of the
// stage kernel.  Both components share the lane's
// upwind side, so they share the coefficient set.  Smoothness indicators use
// a constant 1e-17 floor (the reference's 1e-17*(1+|a|+|b|+|c|) differs from
// it only where f is flat to 1e-17: there every weight takes the floor and
// the substencil values coincide, so the face value does not depend on it).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f), a); }
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(fast_rcp(a.x), fast_rcp(a.y)); }

// 1/x in FP64 for finite normal x: the hardware approximation refined by two
// Newton-Raphson steps for f(r) = 1/r - x, r <- r + r (1 - x r); each step
// doubles the number of correct bits, the last one lands within an ulp
__device__ __forceinline__ double rcp_nr(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

__device__ __forceinline__ double2 f2(double a) { return make_double2(a, a); }
__device__ __forceinline__ double2 fma2(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}
__device__ __forceinline__ double2 mul2(double2 a, double2 b) {
    return make_double2(a.x * b.x, a.y * b.y);
}
__device__ __forceinline__ double2 add2(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 sub2(double2 a, double2 b) {
    return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 rcp2(double2 a) { return make_double2(rcp_nr(a.x), rcp_nr(a.y)); }

// one FP64 value per thread: the same operations on a scalar
__device__ __forceinline__ double fma2(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ double mul2(double a, double b) { return a * b; }
__device__ __forceinline__ double add2(double a, double b) { return a + b; }
__device__ __forceinline__ double sub2(double a, double b) { return a - b; }
__device__ __forceinline__ double rcp2(double a) { return rcp_nr(a); }

// lane value -> its element type, a constant broadcast to it, and its
// components (n = 2 for a pair, 1 for a scalar)
template <typename P> struct LaneOf;
template <> struct LaneOf<float2> {
    typedef float E;
    static constexpr int n = 2;
    __device__ static float2 splat(float a) { return make_float2(a, a); }
};
template <> struct LaneOf<double2> {
    typedef double E;
    static constexpr int n = 2;
    __device__ static double2 splat(double a) { return make_double2(a, a); }
};
template <> struct LaneOf<double> {
    typedef double E;
    static constexpr int n = 1;
    __device__ static double splat(double a) { return a; }
};
// component c of a lane value
__device__ __forceinline__ float& comp(float2& v, int c) { return c ? v.y : v.x; }
__device__ __forceinline__ double& comp(double2& v, int c) { return c ? v.y : v.x; }
__device__ __forceinline__ double& comp(double& v, int) { return v; }

// element type -> pair type and the walker's constants in that type
template <typename E> struct PairOf;
template <> struct PairOf<float> {
    typedef float2 P;
    __device__ static constexpr float c(float f, double) { return f; }
};
template <> struct PairOf<double> {
    typedef double2 P;
    __device__ static constexpr double c(float, double d) { return d; }
};
// a constant in the element type: the float literal for FP32 (the exact
// value the FP32 path has always used), the double literal for FP64
#define BOLT_K(E, v) (PairOf<E>::c(float(v##f), double(v)))
#define BOLT_KQ(E, n, d) (PairOf<E>::c(float(n##.0f / d##.0f), double(n##.0 / d##.0)))

// Per-lane coefficients of the upwind side.  With D2_k the second difference
// of substencil k and the third differences D3a = y0 - 3y1 + 3y2 - y3 =
// D2_1 - D2_2, D3b = y1 - 3y2 + 3y3 - y4 = D2_2 - D2_3, the reference's weighted
// value sum w_k u_k / sum w_k equals u2 + (w1 (u1 - u2) + w3 (u3 - u2)) / sum w_k
// with u1 - u2 = k1 D3a, u3 - u2 = k3 D3b (right face: k = 0.375, 0.125;
// left face: -0.125, -0.375) and u2 = (y2 + ys)/2 - D2_2/8, ys = y3 (right) or
// y1 (left).  With q_k = 1/beta_k^2 and the weights (1, 10, 5)/16 (right) or
// (5, 10, 1)/16 (left), the walker returns TWICE the face value as
//   (y2 + ys - D2_2/4) + (q3 D3b + r q1 D3a) / (a1 q1 + a2 q2 + a3 q3),
// r = (w1 k1)/(w3 k3) and a_k = w_k / (2 w3 k3); callers halve the flux factor.
template <typename E, typename P = typename PairOf<E>::P>
struct Weno5PairT {
    P r, a1, a2, a3;
    bool right;
    __device__ __forceinline__ void set(bool rt) {
        right = rt;
        r = LaneOf<P>::splat(rt ? BOLT_K(E, 0.6) : BOLT_KQ(E, 5, 3));
        a1 = LaneOf<P>::splat(rt ? BOLT_K(E, 0.8) : BOLT_KQ(E, -20, 3));
        a2 = LaneOf<P>::splat(rt ? BOLT_K(E, 8.0) : BOLT_KQ(E, -40, 3));
        a3 = LaneOf<P>::splat(rt ? BOLT_K(E, 4.0) : BOLT_KQ(E, -4, 3));
    }
};

// smoothness indicator of substencil (a, b, c) given its second difference
// D2 = a - 2b + c: 13/12 D2^2 + 1/4 (a - 4b + 3c)^2 + 1e-17, where
// (a - 4b + 3c)/2 = D2/2 + (c - b)
template <typename P>
__device__ __forceinline__ P beta_pair(P D2, P b, P c) {
    typedef typename LaneOf<P>::E E;
    const P e = fma2(LaneOf<P>::splat(BOLT_K(E, 0.5)), D2, sub2(c, b));
    return fma2(mul2(LaneOf<P>::splat(BOLT_KQ(E, 13, 12)), D2), D2,
                fma2(e, e, LaneOf<P>::splat(BOLT_K(E, 1e-17))));
}

template <typename P>
__device__ __forceinline__ P second_diff(P a, P b, P c) {
    typedef typename LaneOf<P>::E E;
    return fma2(LaneOf<P>::splat(BOLT_K(E, -2.0)), b, add2(a, c));
}

// Sliding walker: carries 1/beta^2 of substencils 2 and 3, the second
// difference of substencil 3 and the third difference D3b of the last face.
template <typename E, typename P = typename PairOf<E>::P>
struct Weno5PairWalkerT {
    typedef Weno5PairT<E, P> Side;
    P q2, q3, d23, d3b;
    __device__ __forceinline__ static P inv_sq(P b) {
        const P r = rcp2(b);
        return mul2(r, r);
    }
    __device__ __forceinline__ P eval(P q1, P d3a, P d22, P y1, P y2, P y3,
                                      const Side& S) const {
        const P ys = S.right ? y3 : y1;
        const P base = fma2(LaneOf<P>::splat(BOLT_K(E, -0.25)), d22, add2(y2, ys));
        const P num = fma2(q3, d3b, mul2(mul2(S.r, q1), d3a));
        const P den = fma2(S.a3, q3, fma2(S.a2, q2, mul2(S.a1, q1)));
        return fma2(num, rcp2(den), base);
    }
    __device__ __forceinline__ P first(P y0, P y1, P y2, P y3, P y4, const Side& S) {
        const P d21 = second_diff(y0, y1, y2);
        const P d22 = second_diff(y1, y2, y3);
        d23 = second_diff(y2, y3, y4);
        const P q1 = inv_sq(beta_pair(d21, y1, y2));
        q2 = inv_sq(beta_pair(d22, y2, y3));
        q3 = inv_sq(beta_pair(d23, y3, y4));
        const P d3a = sub2(d21, d22);
        d3b = sub2(d22, d23);
        return eval(q1, d3a, d22, y1, y2, y3, S);
    }
    // window advanced by one cell: y0..y4 are the new window's values
    __device__ __forceinline__ P next(P y0, P y1, P y2, P y3, P y4, const Side& S) {
        const P q1 = q2;
        const P d3a = d3b;
        const P d22 = d23;
        q2 = q3;
        d23 = second_diff(y2, y3, y4);
        q3 = inv_sq(beta_pair(d23, y3, y4));
        d3b = sub2(d22, d23);
        return eval(q1, d3a, d22, y1, y2, y3, S);
    }
};

// Minmod faces for the paired kernel, same interface as Weno5PairWalkerT:
// twice the face value of the window's centre cell y2 (its right face for
// right-moving lanes, its left face otherwise), 2 y2 +- the limited slope of
// (y1, y2, y3) (minmod.py:4-71).  No state is carried between faces.
template <typename E, typename P = typename PairOf<E>::P>
struct MinmodPairWalkerT {
    typedef Weno5PairT<E, P> Side;
    __device__ __forceinline__ static P face(P y1, P y2, P y3, bool right) {
        P sl;
#pragma unroll
        for (int c = 0; c < LaneOf<P>::n; ++c) {
            const E m = minmod_slope(comp(y1, c), comp(y2, c), comp(y3, c));
            comp(sl, c) = right ? m : -m;
        }
        return fma2(LaneOf<P>::splat(BOLT_K(E, 2.0)), y2, sl);
    }
    __device__ __forceinline__ P first(P, P y1, P y2, P y3, P, const Side& S) {
        return face(y1, y2, y3, S.right);
    }
    __device__ __forceinline__ P next(P, P y1, P y2, P y3, P, const Side& S) {
        return face(y1, y2, y3, S.right);
    }
};

// PPM (ppm.py:4-100) and piecewise-constant faces for the paired kernel:
// twice the face value of the window's centre cell y2, per element
template <typename E, typename P = typename PairOf<E>::P>
struct PpmPairWalkerT {
    typedef Weno5PairT<E, P> Side;
    __device__ __forceinline__ P first(P y0, P y1, P y2, P y3, P y4, const Side& S) {
        return next(y0, y1, y2, y3, y4, S);
    }
    __device__ __forceinline__ P next(P y0, P y1, P y2, P y3, P y4, const Side& S) {
        P o;
#pragma unroll
        for (int c = 0; c < LaneOf<P>::n; ++c)
            comp(o, c) = E(2) * ppm_face(comp(y0, c), comp(y1, c), comp(y2, c), comp(y3, c),
                                         comp(y4, c), S.right);
        return o;
    }
};

template <typename E, typename P = typename PairOf<E>::P>
struct ConstPairWalkerT {
    typedef Weno5PairT<E, P> Side;
    __device__ __forceinline__ P first(P, P, P y2, P, P, const Side&) {
        return add2(y2, y2);
    }
    __device__ __forceinline__ P next(P, P, P y2, P, P, const Side&) {
        return add2(y2, y2);
    }
};

// ---------------------------------------------------------------------------
// Per-thread asynchronous global -> shared copies (cp.async, 4 bytes, cached
// in L1), committed in groups; wait_group<N> returns once at most N of this
// thread's groups are still in flight (always completes: no timeout needed).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;"
                 ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst))),
                   "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------------------
// mbarrier + TMA (cp.async.bulk.tensor) wrappers.  Waits are bounded: after
// a budget of clock cycles (the launch's wait_cycles for the tile waits,
// kDefaultWaitCycles for the clean-up of a failed CTA) the wait reports
// failure and the caller records BOLT_ERR_TIMEOUT instead of hanging.
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// returns false if the barrier did not complete within `budget` clock cycles
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity,
                                                  long long budget = kDefaultWaitCycles) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    for (;;) {
        for (int it = 0; it < 256; ++it)
            if (mbar_try_wait(bar, parity)) return true;
        if (clock64() - t0 > budget) return false;
    }
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)),
          "r"(x), "r"(y), "r"(z)
        : "memory");
}

// shared -> global box store; completion tracked by bulk groups of the issuing thread
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int x,
                                             int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];"
        ::"l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// shared -> global box reduction: global += shared, element type of the map
__device__ __forceinline__ void tma_reduce_add_3d(const CUtensorMap* map, const void* src, int x,
                                                  int y, int z) {
    asm volatile(
        "cp.reduce.async.bulk.tensor.3d.global.shared::cta.add.tile.bulk_group"
        " [%0, {%2, %3, %4}], [%1];"
        ::"l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ void bulk_commit() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// the committed stores no longer read shared memory
__device__ __forceinline__ void bulk_wait_read_all() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Named CTA barrier `id` (1..15) over `n` threads: producers arrive without
// waiting, consumers wait until all n have arrived; shared-memory writes made
// by the producers before arriving are visible to the consumers after it.
__device__ __forceinline__ void named_bar_arrive(int id, int n) {
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ void named_bar_sync(int id, int n) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// the committed stores are complete
__device__ __forceinline__ void bulk_wait_all() {
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ---------------------------------------------------------------------------
// warp reductions (FP64)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace bolt
