/*
 * bolt_oracle_c.c - FP64 C/OpenMP restatement of Bolt's FVM kinetic update
 * for the fields-off path (q1/q2 advection + BGK relaxation), used as the
 * timed CPU baseline.  TEST/BENCH INFRASTRUCTURE ONLY: never linked into the
 * product library.
 *
 * Follows (paths within the Bolt project):
 *   df_dt_fvm.py:56-97            q-fluxes, flux difference, BGK source
 *   reconstruction/weno5.py:4-98  point-value WENO5 (and minmod.py, ppm.py)
 *   riemann.py:46-49              upwind select by the sign of C_q
 *   collision_operator.py:16-128  Maxwellian from the moments, -(f - f0)/tau
 *   compute_moments.py:7-59       sum over p times dp1*dp2*dp3
 *   fvm_operator.py:6-35          RK2 midpoint with halo refresh per stage
 *   integrators.py:15-28          classic RK4 stages
 * Layout: f[q2g][q1g][s][p] (p1 fastest), ghost zones Ng, periodic in q.
 * Expressions keep the reference's operation order (compile without
 * -ffast-math and with -ffp-contract=off).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct OracleGrid {
    int Nq1, Nq2, Ng, Np1, Np2, Np3, Ns, p_dim;
    double dq1, dq2;
    double p1_start[8], p2_start[8], p3_start[8], dp1[8], dp2[8], dp3[8], mass[8];
    double kB, tau;
    int recon;       /* 0 pc, 1 minmod, 2 ppm, 3 weno5 */
    int bgk;
} OracleGrid;

static double beta(double a, double b, double c) {
    double poly = ((((4.0 / 3.0) * a * a - (19.0 / 3.0) * a * b) + (25.0 / 3.0) * b * b)
                   + (11.0 / 3.0) * a * c - (31.0 / 3.0) * b * c) + (10.0 / 3.0) * c * c;
    return poly + 1e-17 * (((1.0 + fabs(a)) + fabs(b)) + fabs(c));
}

/* right (upwind for C > 0) or left face value of cell y2 */
static double face(int recon, const double y[5], int right) {
    if (recon == 0) return y[2];
    if (recon == 1) {
        double fwd = y[3] - y[2], bwd = y[2] - y[1], cen = bwd + fwd;
        double x = 2 * bwd, yy = 0.5 * cen, z = 2 * fwd;
        double m = fmin(fmin(fabs(x), fabs(yy)), fabs(z));
        double sx = x < 0 ? -1 : 1, sy = yy < 0 ? -1 : 1, sz = z < 0 ? -1 : 1;
        double s = ((0.25 * fabs(sx + sy)) * (sx + sz)) * m;
        return right ? y[2] + 0.5 * s : y[2] - 0.5 * s;
    }
    if (recon == 2) {
        double y0 = y[0], y1 = y[1], y2 = y[2], y3 = y[3], y4 = y[4];
        double d0 = 2 * (y1 - y0), d1 = 2 * (y2 - y1), d2 = 2 * (y3 - y2), d3 = 2 * (y4 - y3);
        double D1 = 0.5 * (y2 - y0), D2 = 0.5 * (y3 - y1), D3 = 0.5 * (y4 - y2);
#define DQ(D, da, db) (((1.0 - ((db) * (da) <= 0)) * ((D) > 0 ? 1.0 : -1.0)) * \
                       fmin(fabs(D), fmin(fabs(da), fabs(db))))
        double Q1 = DQ(D1, d0, d1), Q2 = DQ(D2, d1, d2), Q3 = DQ(D3, d2, d3);
#undef DQ
        double l = 0.5 * (y2 + y1) - (Q2 - Q1) / 6, r = 0.5 * (y3 + y2) - (Q3 - Q2) / 6;
        double c1 = ((r - y2) * (y2 - l) <= 0), qd = r - l, qe = 6 * (y2 - 0.5 * (r + l));
        double c2 = (qd * (qd - qe) < 0), c3 = (qd * (qd + qe) < 0);
        l = l * (1 - c1) + c1 * y2;
        r = r * (1 - c1) + c1 * y2;
        l = l * (1 - c2) + c2 * (3 * y2 - 2 * r);
        r = (r * c2 + ((1 - c2) * r) * (1 - c3)) + ((1 - c2) * c3) * (3 * y2 - 2 * l);
        return right ? r : l;
    }
    {
        double b1 = beta(y[0], y[1], y[2]), b2 = beta(y[1], y[2], y[3]), b3 = beta(y[2], y[3], y[4]);
        if (right) {
            double w1 = 1 / ((16 * b1) * b1), w2 = 5 / ((8 * b2) * b2), w3 = 5 / ((16 * b3) * b3);
            double u1 = (0.375 * y[0] - 1.25 * y[1]) + 1.875 * y[2];
            double u2 = (-0.125 * y[1] + 0.75 * y[2]) + 0.375 * y[3];
            double u3 = (0.375 * y[2] + 0.75 * y[3]) - 0.125 * y[4];
            return ((w1 * u1 + w2 * u2) + w3 * u3) / ((w1 + w2) + w3);
        } else {
            double w1 = 5 / ((16 * b1) * b1), w2 = 5 / ((8 * b2) * b2), w3 = 1 / ((16 * b3) * b3);
            double u1 = (-0.125 * y[0] + 0.75 * y[1]) + 0.375 * y[2];
            double u2 = (0.375 * y[1] + 0.75 * y[2]) - 0.125 * y[3];
            double u3 = (1.875 * y[2] - 1.25 * y[3]) + 0.375 * y[4];
            return ((w1 * u1 + w2 * u2) + w3 * u3) / ((w1 + w2) + w3);
        }
    }
}

static void fill_ghosts(double* f, const OracleGrid* g) {
    const int Nq1g = g->Nq1 + 2 * g->Ng, Nq2g = g->Nq2 + 2 * g->Ng;
    const long row = (long)g->Ns * g->Np1 * g->Np2 * g->Np3;
#pragma omp parallel for schedule(static)
    for (int jj = 0; jj < Nq2g; ++jj) {
        for (int ii = 0; ii < Nq1g; ++ii) {
            int i = ii - g->Ng, j = jj - g->Ng;
            if (i >= 0 && i < g->Nq1 && j >= 0 && j < g->Nq2) continue;
            int si = ((i % g->Nq1) + g->Nq1) % g->Nq1 + g->Ng;
            int sj = ((j % g->Nq2) + g->Nq2) % g->Nq2 + g->Ng;
            memcpy(f + ((long)jj * Nq1g + ii) * row, f + ((long)sj * Nq1g + si) * row,
                   row * sizeof(double));
        }
    }
}

/* df/dt for interior cells; k has the layout of f (ghost entries untouched) */
static void dfdt(const double* f, double* k, const OracleGrid* g) {
    const int Ng = g->Ng, Nq1g = g->Nq1 + 2 * Ng;
    const int Np = g->Np1 * g->Np2 * g->Np3;
    const long row = (long)g->Ns * Np, col = row * Nq1g;
#pragma omp parallel for schedule(static) collapse(2)
    for (int j = 0; j < g->Nq2; ++j) {
        for (int i = 0; i < g->Nq1; ++i) {
            for (int s = 0; s < g->Ns; ++s) {
                const double* fc = f + (long)(j + Ng) * col + (long)(i + Ng) * row + (long)s * Np;
                double* kc = k + (long)(j + Ng) * col + (long)(i + Ng) * row + (long)s * Np;
                double mm[5] = {0, 0, 0, 0, 0};
                double A = 0, u1 = 0, u2 = 0, u3 = 0, twokT = 1, m = g->mass[s];
                if (g->bgk) {
                    for (int p = 0; p < Np; ++p) {
                        int i1 = p % g->Np1, i2 = (p / g->Np1) % g->Np2, i3 = p / (g->Np1 * g->Np2);
                        double v1 = g->p1_start[s] + (0.5 + i1) * g->dp1[s];
                        double v2 = g->p2_start[s] + (0.5 + i2) * g->dp2[s];
                        double v3 = g->p3_start[s] + (0.5 + i3) * g->dp3[s];
                        double fv = fc[p];
                        mm[0] += fv; mm[1] += fv * v1; mm[2] += fv * v2; mm[3] += fv * v3;
                        mm[4] += (0.5 * fv) * ((v1 * v1 + v2 * v2) + v3 * v3);
                    }
                    double meas = (g->dp3[s] * g->dp2[s]) * g->dp1[s], eps = 1e-30;
                    double n = mm[0] * meas;
                    u1 = (mm[1] * meas) / (n + eps);
                    u2 = (mm[2] * meas) / (n + eps);
                    u3 = (mm[3] * meas) / (n + eps);
                    double E = mm[4] * meas, nm = n * m;
                    double T = (1.0 / g->p_dim) * ((((2.0 * (E * m) - nm * (u1 * u1)) - nm * (u2 * u2))
                                                    - nm * (u3 * u3))) / (n + eps) + eps;
                    twokT = (2.0 * g->kB) * T;
                    double base = m / ((2.0 * 3.141592653589793 * g->kB) * T);
                    A = n * (g->p_dim == 3 ? pow(base, 1.5) : (g->p_dim == 2 ? base : sqrt(base)));
                }
                for (int p = 0; p < Np; ++p) {
                    int i1 = p % g->Np1, i2 = (p / g->Np1) % g->Np2, i3 = p / (g->Np1 * g->Np2);
                    double v1 = g->p1_start[s] + (0.5 + i1) * g->dp1[s];
                    double v2 = g->p2_start[s] + (0.5 + i2) * g->dp2[s];
                    double v3 = g->p3_start[s] + (0.5 + i3) * g->dp3[s];
                    /* q1 faces i (left) and i+1 (right) */
                    double y[5], Fl, Fr, Gb = 0, Gt = 0;
                    int r1 = v1 > 0, o1 = r1 ? -3 : -2;
                    for (int t = 0; t < 5; ++t) y[t] = fc[(long)(o1 + t) * row + p];
                    Fl = v1 * face(g->recon, y, r1);
                    for (int t = 0; t < 5; ++t) y[t] = fc[(long)(o1 + 1 + t) * row + p];
                    Fr = v1 * face(g->recon, y, r1);
                    double kk = (-(Fr - Fl)) / g->dq1;
                    if (g->Nq2 > 1) {
                        int r2 = v2 > 0, o2 = r2 ? -3 : -2;
                        for (int t = 0; t < 5; ++t) y[t] = fc[(long)(o2 + t) * col + p];
                        Gb = v2 * face(g->recon, y, r2);
                        for (int t = 0; t < 5; ++t) y[t] = fc[(long)(o2 + 1 + t) * col + p];
                        Gt = v2 * face(g->recon, y, r2);
                        kk = kk - (Gt - Gb) / g->dq2;
                    }
                    if (g->bgk) {
                        double d1 = v1 - u1, fmb = A * exp((-m * (d1 * d1)) / twokT);
                        if (g->p_dim >= 2) { double d2 = v2 - u2; fmb = fmb * exp((-m * (d2 * d2)) / twokT); }
                        if (g->p_dim == 3) { double d3 = v3 - u3; fmb = fmb * exp((-m * (d3 * d3)) / twokT); }
                        kk = kk + (-(fc[p] - fmb) / g->tau);
                    }
                    kc[p] = kk;
                }
            }
        }
    }
}

static void axpy_interior(double* out, const double* base, const double* k, double c,
                          const OracleGrid* g) {
    const int Ng = g->Ng, Nq1g = g->Nq1 + 2 * Ng;
    const long row = (long)g->Ns * g->Np1 * g->Np2 * g->Np3, col = row * Nq1g;
#pragma omp parallel for schedule(static) collapse(2)
    for (int j = 0; j < g->Nq2; ++j)
        for (int i = 0; i < g->Nq1; ++i) {
            long o = (long)(j + Ng) * col + (long)(i + Ng) * row;
            for (long p = 0; p < row; ++p) out[o + p] = base[o + p] + k[o + p] * c;
        }
}

/* One RK step of f (ghosted, periodic) in place.  integrator: 2 or 4.
 * Returns 0, or -1 if scratch allocation failed. */
int oracle_rk_step(double* f, const OracleGrid* g, double dt, int integrator, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    const long n = (long)(g->Nq1 + 2 * g->Ng) * (g->Nq2 + 2 * g->Ng) * g->Ns * g->Np1 * g->Np2 * g->Np3;
    double* x = (double*)malloc(n * sizeof(double));
    double* k = (double*)calloc(n, sizeof(double));
    if (!x || !k) { free(x); free(k); return -1; }
    fill_ghosts(f, g);
    if (integrator == 2) {
        dfdt(f, k, g);
        memcpy(x, f, n * sizeof(double));
        axpy_interior(x, f, k, dt / 2, g);
        fill_ghosts(x, g);
        dfdt(x, k, g);
        axpy_interior(f, f, k, dt, g);
    } else {
        double* acc = (double*)malloc(n * sizeof(double));
        if (!acc) { free(x); free(k); return -1; }
        memcpy(x, f, n * sizeof(double));
        memcpy(acc, f, n * sizeof(double));
        const double c[4] = {0.5 * dt, 0.5 * dt, dt, 0};
        const double w[4] = {dt / 6, dt / 3, dt / 3, dt / 6};
        const double* src = f;
        for (int st = 0; st < 4; ++st) {
            dfdt(src, k, g);
            axpy_interior(acc, acc, k, w[st], g);
            if (st < 3) {
                axpy_interior(x, f, k, c[st], g);
                fill_ghosts(x, g);
                src = x;
            }
        }
        const int Ng = g->Ng, Nq1g = g->Nq1 + 2 * Ng;
        const long row = (long)g->Ns * g->Np1 * g->Np2 * g->Np3, col = row * Nq1g;
        for (int j = 0; j < g->Nq2; ++j)
            for (int i = 0; i < g->Nq1; ++i) {
                long o = (long)(j + Ng) * col + (long)(i + Ng) * row;
                memcpy(f + o, acc + o, row * sizeof(double));
            }
        free(acc);
    }
    fill_ghosts(f, g);
    free(x);
    free(k);
    return 0;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
