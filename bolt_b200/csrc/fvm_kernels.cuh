// fvm_kernels.cuh - the FVM kernels of the kinetic update (sm_100a).
//
// Kernel inventory (templated on the storage type T = double | float and on
// EXACT = reference operation order, used by the FP64 parity build):
//
//   qstage_kernel   q1/q2 advection + BGK relaxation + RK stage combine +
//                   FP64 partial moments of the stage output.  This is
//                   df_dt_fvm.py:56-97 (q-part and source) fused with the
//                   stage update of fvm_operator.py:26,33 / integrators.py:15-28.
//   pstage_kernel   p1/p2/p3 advection with C_p from the cell-centred fields
//                   (df_dt_fvm.py:245-323), added to the q-part, then the RK
//                   combine (used only when fields are enabled).
//   moments_kernel  compute_moments.py:7-59 for any moment of moments.py.
//   ghost_kernel    communicate_f + apply_bcs_f (periodic wrap, mirror,
//                   Dirichlet inflow, zero for ghosted outflow cells).
//   fdtd kernels    fields.py:568-647 / fdtd_explicit.py:9-177 on the Yee grid.
//
// Layout: f[q2g][q1g][s][p] with p = (p3, p2, p1) flattened, p1 fastest.
// The q-stage kernel works on tiles of TQ1 x TQ2 q-cells x 32 consecutive p
// (one warp lane per p).  A tile plus its 3-cell q-halo is brought into shared
// memory by one TMA box copy (double-buffered, mbarrier completion), or by
// coalesced loads with wrap-around indexing when TMA's alignment rules do not
// hold.  Each CTA owns one q-tile and a contiguous range of p-chunks of one
// species; its partial velocity moments of the stage output are written per
// (p-split, q-cell) and summed by the next stage's prologue (deterministic,
// no atomics).
#pragma once

#include "fvm_common.cuh"
#include "fvm_args.h"

namespace bolt {

// ---------------------------------------------------------------------------
// moment contributions of one value (FP64), reference moments.py:6-24
// ---------------------------------------------------------------------------
struct PVel {
    double v1, v2, v3, vsq;
};

__device__ __forceinline__ PVel lane_velocity(const SpeciesGrid& sg, int s, int ip1, int ip2,
                                              int ip3) {
    PVel v;
    v.v1 = sg.p1_start[s] + (0.5 + ip1) * sg.dp1[s];
    v.v2 = sg.p2_start[s] + (0.5 + ip2) * sg.dp2[s];
    v.v3 = sg.p3_start[s] + (0.5 + ip3) * sg.dp3[s];
    v.vsq = (v.v1 * v.v1 + v.v2 * v.v2) + v.v3 * v.v3;
    return v;
}

// Periodic images of interior cell (ii, jj) in the ghost zones (any Ng/Nq).
template <typename T>
__device__ __forceinline__ void write_ghost_images(T* out, T v, int ii, int jj, int s, int p,
                                                   int Ng, int Nq1, int Nq2, int Nq1g, int Nq2g,
                                                   int per1, int per2, long long rowstride,
                                                   long long colstride, int Np) {
    const int n1 = per1 ? (Ng + Nq1 - 1) / Nq1 : 0;
    const int n2 = per2 ? (Ng + Nq2 - 1) / Nq2 : 0;
    for (int t1 = -n1; t1 <= n1; ++t1) {
        const int g1 = ii + Ng + t1 * Nq1;
        if (g1 < 0 || g1 >= Nq1g) continue;
        for (int t2 = -n2; t2 <= n2; ++t2) {
            const int g2 = jj + Ng + t2 * Nq2;
            if (g2 < 0 || g2 >= Nq2g || (t1 == 0 && t2 == 0)) continue;
            out[(long long)g2 * colstride + (long long)g1 * rowstride + (long long)s * Np + p] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// Maxwellian parameters of q-cell (ii, jj) from the stage input's partial
// moments (collision_operator.py:102-118, f0 :49-65), FP64:
// qq = {n*A, u1, u2, u3, 2 kB T} with A the normalisation of the p_dim-D
// Maxwellian.  Cells outside the grid get the parameters of zero moments.
// ---------------------------------------------------------------------------
// the parameters from the moment sums mm (sum over the partial slots);
// SQRT_POW: the 3-D normalisation base^1.5 as base*sqrt(base) (within an ulp
// or two of pow, which the reference-order path keeps)
template <bool SQRT_POW = false>
__device__ __forceinline__ void bgk_params_from_sums(const QStageArgs& a, int s, const double* mm,
                                                     double* qq) {
    const double m = a.sg.mass[s];
    const double kB = a.kB;
    const double measure = (a.sg.dp3[s] * a.sg.dp2[s]) * a.sg.dp1[s];
    const double eps = 1e-30;
    // moments as compute_moments returns them: sum * measure, times initial_mu
    // on the polar2D grid
    const bool polar = a.sg.polar2d != 0;
    const double sc = a.sg.mom_scale;
    double mv[kNumMom];
#pragma unroll
    for (int q = 0; q < kNumMom; ++q) mv[q] = polar ? sc * (mm[q] * measure) : mm[q] * measure;
    double n = mv[0];
    double u1 = mv[1] / (n + eps);
    double u2 = mv[2] / (n + eps);
    double u3 = mv[3] / (n + eps);
    double E = mv[4];
    double nm = n * m;
    double Tt = (1.0 / a.p_dim) * ((((2.0 * (E * m) - nm * (u1 * u1)) - nm * (u2 * u2))
                                    - nm * (u3 * u3))) / (n + eps) + eps;
    double twokT = (2.0 * kB) * Tt;
    double base = m / ((2.0 * 3.141592653589793 * kB) * Tt);
    const double rb = sqrt(base);
    double A = a.p_dim == 3 ? (SQRT_POW ? base * rb : pow(base, 1.5)) : (a.p_dim == 2 ? base : rb);
    qq[0] = n * A;
    qq[1] = u1;
    qq[2] = u2;
    qq[3] = u3;
    qq[4] = twokT;
}

// moment q of q-cell (ii, jj): the partial slots summed in slot order
__device__ __forceinline__ double bgk_moment_sum(const QStageArgs& a, int s, int ii, int jj,
                                                 int q) {
    const long long plane = (long long)a.Nq2 * a.Nq1;
    double v = 0.0;
    if (ii < a.Nq1 && jj < a.Nq2) {
        const double* src = a.mom_in + ((long long)q * a.Ns + s) * plane +
                            (long long)jj * a.Nq1 + ii;
        const long long step = (long long)kNumMom * a.Ns * plane;
#pragma unroll 4
        for (int sp = 0; sp < a.nsplit_in; ++sp) v += src[sp * step];
    }
    return v;
}

__device__ __forceinline__ void bgk_cell_params(const QStageArgs& a, int s, int ii, int jj,
                                                double* qq) {
    double mm[kNumMom];
#pragma unroll
    for (int q = 0; q < kNumMom; ++q) mm[q] = bgk_moment_sum(a, s, ii, jj, q);
    bgk_params_from_sums(a, s, mm, qq);
}

// exp table entry q of a q-cell: p1 entries carry n*A, inactive axes are 1
__device__ __forceinline__ double bgk_table_entry(const QStageArgs& a, const double* qq,
                                                  const double* vgrid, int q, double m) {
    const int Np1 = a.Np1, Np2 = a.Np2;
    const double u = q < Np1 ? qq[1] : (q < Np1 + Np2 ? qq[2] : qq[3]);
    const bool act = q < Np1 || (q < Np1 + Np2 ? a.p_dim >= 2 : a.p_dim == 3);
    const double dv = vgrid[q] - u;
    const double ev = act ? exp((-m * (dv * dv)) / qq[4]) : 1.0;
    return q < Np1 ? qq[0] * ev : ev;
}

// ---------------------------------------------------------------------------
// q-stage prologue shared by the scalar and paired kernels: zero the current
// accumulators, the species' p-cell centres, the TMA barriers, and for BGK the
// Maxwellian of the stage input per q-cell (collision_operator.py:102-118,
// f0 :49-65) with its per-q-cell exp tables (the p1 table carries n*A).
// ---------------------------------------------------------------------------
template <int NQ, int TQ1, bool BGK>
__device__ __forceinline__ void qstage_prologue(const QStageArgs& a, int s, int i0, int j0,
                                                double* j_acc, double* vgrid, double* qc,
                                                double* tabs, uint64_t* bars) {
    const int tid = threadIdx.x;
    const int Np1 = a.Np1, Np2 = a.Np2, Np3 = a.Np3;
    const int ntab = Np1 + Np2 + Np3;
    for (int c = tid; c < NQ * 3; c += NTHREADS) j_acc[c] = 0.0;
    for (int q = tid; q < ntab; q += NTHREADS) {
        if (q < Np1) vgrid[q] = a.sg.p1_start[s] + (0.5 + q) * a.sg.dp1[s];
        else if (q < Np1 + Np2) vgrid[q] = a.sg.p2_start[s] + (0.5 + (q - Np1)) * a.sg.dp2[s];
        else vgrid[q] = a.sg.p3_start[s] + (0.5 + (q - Np1 - Np2)) * a.sg.dp3[s];
    }
    if (tid == 0 && a.use_tma) {
        prefetch_tmap(&a.tmap);
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_barrier_init();
    }
    __syncthreads();

    // ---- BGK prologue: Maxwellian of the stage input per q-cell (FP64) ----
    // collision_operator.py:102-118 and f0 :49-65
    if (BGK) {
        for (int c = tid; c < NQ; c += NTHREADS)
            bgk_cell_params(a, s, i0 + c % TQ1, j0 + c / TQ1, qc + c * 5);
        __syncthreads();
        if (!a.bgk_direct) {
            // exp tables over (q-cell, p1 | p2 | p3); the p1 entry carries n*A
            const double m = a.sg.mass[s];
            for (int e = tid; e < NQ * ntab; e += NTHREADS) {
                const int c = e / ntab, q = e % ntab;
                tabs[e] = bgk_table_entry(a, qc + c * 5, vgrid, q, m);
            }
        }
    }
    __syncthreads();

}

// ---------------------------------------------------------------------------
// q-stage kernel
//
// Per p-chunk (32 consecutive p of one species) and q-tile:
//   phase A  q1 faces: one upwind face value per face, walking each tile row
//            with a sliding window; D1 = (-(F_R - F_L)) / dq1 -> stage buffer
//   phase B  q2 faces likewise, BGK, RK combine; writes out1/out2 to global
//            and out1 back into the stage buffer
//   phase C  FP64 moments of out1 from the stage buffer: each thread owns one
//            q-cell and a quarter of the chunk's p values, accumulating in
//            registers across all chunks of the CTA (reduced once at the end)
// ---------------------------------------------------------------------------
template <typename T, bool EXACT, int RECON, int TQ1, int TQ2, bool Q2, bool BGK>
__global__ void __launch_bounds__(NTHREADS, 2)
qstage_kernel(const __grid_constant__ QStageArgs a) {
    constexpr int HX = TQ1 + 2 * HALO;
    constexpr int HY = Q2 ? TQ2 + 2 * HALO : 1;
    constexpr int NQ = TQ1 * TQ2;
    constexpr int NWARP = NTHREADS / 32;
    constexpr int NQUART = NTHREADS / NQ;       // threads per q-cell in phase C
    constexpr int PQ = PW / NQUART;             // p values per phase-C thread
    static_assert(NTHREADS % NQ == 0 && PW % NQUART == 0, "phase C mapping");
    constexpr int TILE = HY * HX * PW;
    // phase A: rows split into NSEG segments; phase B: ITEMS (column, segment)
    // items per warp of SEGB rows each -> NSLOT cells per thread
    constexpr int NSEG = (TQ2 >= NWARP) ? 1 : (NWARP / TQ2);
    constexpr int SEG = (TQ1 + NSEG - 1) / NSEG;
    constexpr int NSEGB = (TQ1 >= NWARP) ? 1 : (NWARP / TQ1);
    constexpr int SEGB = (TQ2 + NSEGB - 1) / NSEGB;
    constexpr int ITEMS = TQ1 * NSEGB / NWARP;
    static_assert(TQ1 * NSEGB % NWARP == 0, "phase B items per warp");
    constexpr int NSLOT = ITEMS * SEGB;

    const int Np1 = a.Np1, Np2 = a.Np2, Np3 = a.Np3, Np = a.Np, Ng = a.Ng;
    const int Nq1 = a.Nq1, Nq2 = a.Nq2;
    const int ntab = Np1 + Np2 + Np3;
    const QLayout Lo = qstage_layout(TQ1, TQ2, Q2, sizeof(T), BGK, a.bgk_direct, ntab);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* tile = reinterpret_cast<T*>(smem_raw + Lo.tile);              // [NB][HY][HX][PW]
    T* stage = reinterpret_cast<T*>(smem_raw + Lo.stage);            // [NQ][PWP]
    double* vtab = reinterpret_cast<double*>(smem_raw + Lo.vtab);    // [4][PW]
    double* j_acc = reinterpret_cast<double*>(smem_raw + Lo.jacc);   // [NQ][3]
    double* qc = reinterpret_cast<double*>(smem_raw + Lo.qc);        // [NQ][5]
    double* tabs = reinterpret_cast<double*>(smem_raw + Lo.tabs);    // [NQ][ntab]
    double* vgrid = reinterpret_cast<double*>(smem_raw + Lo.vgrid);  // [ntab]
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + Lo.bars);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tile1 = blockIdx.x % a.ntiles1, tile2 = blockIdx.x / a.ntiles1;
    const int s = blockIdx.y / a.nsplit, split = blockIdx.y % a.nsplit;
    const int i0 = tile1 * TQ1, j0 = tile2 * TQ2;                     // interior origin
    const int nchunks = (Np + PW - 1) / PW;
    const int k_begin = split * a.chunks_per_split;
    const int k_end = min(nchunks, k_begin + a.chunks_per_split);
    const long long rowstride = (long long)a.Ns * Np;                 // per q1 step
    const long long colstride = rowstride * a.Nq1g;                   // per q2 step
    const T* fs = static_cast<const T*>(a.fs);
    // CTA-uniform predicates: whole tile inside the domain and every chunk
    // complete (no per-cell masks), tile within reach of a periodic border
    const bool tile_full = (i0 + TQ1 <= Nq1) && (j0 + TQ2 <= Nq2);
    const bool fast = tile_full && a.full_chunks;
    const bool border = (a.periodic1 && (i0 < Ng || i0 + TQ1 > Nq1 - Ng)) ||
                        (a.periodic2 && (j0 < Ng || j0 + TQ2 > Nq2 - Ng));

    qstage_prologue<NQ, TQ1, BGK>(a, s, i0, j0, j_acc, vgrid, qc, tabs, bars);

    // ---- tile loader -------------------------------------------------------
    bool failed = false;       // a bounded wait gave up
    const unsigned tile_bytes = TILE * sizeof(T);
    auto issue = [&](int k, int buf) {
        if (k >= k_end) return;
        if (a.use_tma) {
            if (a.stall_test) return;           // test hook: the wait below runs out
            if (tid == 0) {
                mbar_arrive_expect_tx(&bars[buf], tile_bytes);
                tma_load_3d(tile + buf * TILE, &a.tmap, &bars[buf], s * Np + k * PW,
                            i0 + Ng - HALO, Q2 ? j0 + Ng - HALO : j0 + Ng);
            }
        } else {
            // coalesced loads with wrap-around (af.shift semantics) indexing
            T* dst = tile + buf * TILE;
            for (int r = warp; r < HY * HX; r += NWARP) {
                int hy = r / HX, hx = r % HX;
                int g1 = i0 + Ng - HALO + hx;
                int g2 = Q2 ? j0 + Ng - HALO + hy : j0 + Ng;
                g1 = ((g1 % a.Nq1g) + a.Nq1g) % a.Nq1g;
                g2 = ((g2 % a.Nq2g) + a.Nq2g) % a.Nq2g;
                int p = k * PW + lane;
                T v = T(0);
                if (p < Np) v = fs[(long long)g2 * colstride + (long long)g1 * rowstride
                                   + (long long)s * Np + p];
                dst[r * PW + lane] = v;
            }
        }
    };

    unsigned phase0 = 0u, phase1 = 0u;
    const int NB = Lo.nbuf;                     // 1 or 2 halo tiles
    issue(k_begin, 0);
    if (NB == 2) issue(k_begin + 1, 1);

    T* out1 = static_cast<T*>(a.out1);
    T* out2 = static_cast<T*>(a.out2);
    const T* base1 = static_cast<const T*>(a.base1);
    const T* base2 = static_cast<const T*>(a.base2);
    const T* tau_arr = static_cast<const T*>(a.tau_arr);
    const T c1 = T(a.c1), c2 = T(a.c2);
    const T inv_tau = T(1.0 / a.tau);
    const T inv_dq1 = T(1.0 / a.dq1), inv_dq2 = T(1.0 / a.dq2);
    const double mneg = -a.sg.mass[s];
    const bool want_mom = a.mom_out != nullptr;
    const bool want_j = a.want_j != 0;
    // phase C ownership: q-cell pc_c, p values [pc_q*PQ, pc_q*PQ + PQ) of each chunk
    const int pc_c = tid % NQ, pc_q = tid / NQ;
    double macc[kNumMom] = {0, 0, 0, 0, 0};

    // this lane's p index within the species, kept as (ip1, ip2, ip3) and
    // advanced by PW per chunk without divisions
    int p = k_begin * PW + lane;
    int ip1 = p % Np1, ip2 = (p / Np1) % Np2, ip3 = p / (Np1 * Np2);
    // element offset of this thread's first phase-B cell (q-cell (i0+ic0, j0+rb0))
    // for item 0; other slots add compile-time multiples of the strides
    const int ic0 = warp / NSEGB, rb0 = (warp % NSEGB) * SEGB;
    const long long tbase = (long long)(j0 + rb0 + Ng) * colstride
                          + (long long)(i0 + ic0 + Ng) * rowstride + (long long)s * Np;
    const long long item_step = (long long)(NWARP / NSEGB) * rowstride;   // next item: columns

    int buf = 0;
    for (int k = k_begin; k < k_end; ++k, buf ^= (NB - 1)) {
        if (a.use_tma) {
            const unsigned ph = buf ? phase1 : phase0;
            if (!mbar_wait_bounded(&bars[buf], ph, a.wait_cycles)) failed = true;
            if (buf) phase1 ^= 1u; else phase0 ^= 1u;
        }
        // tile visible; previous chunk's phase C done with `stage`.  A wait
        // that ran out ends the CTA: record it and let the copies still in
        // flight (chunks k .. k+NB-1) land, bounded, before returning.
        if (__syncthreads_or(failed)) {
            if (tid == 0) {
                atomicExch(a.err, 4);
                // chunk k's parity was already flipped above; chunk k+1's not
                // (under the stall hook no copy was issued)
                for (int j = 0; j < NB && k + j < k_end && !a.stall_test; ++j) {
                    const int b = (buf + j) % NB;
                    const unsigned ph = (b ? phase1 : phase0) ^ (j == 0 ? 1u : 0u);
                    mbar_wait_bounded(&bars[b], ph);
                }
            }
            return;
        }
        const T* X = tile + buf * TILE;
        const bool pvalid = p < Np;
        const int jp1 = pvalid ? ip1 : 0, jp2 = pvalid ? ip2 : 0, jp3 = pvalid ? ip3 : 0;
        const double V1 = vgrid[jp1], V2 = vgrid[Np1 + jp2], V3 = vgrid[Np1 + Np2 + jp3];
        const T v1 = T(V1), v2 = T(V2);

        // ---- prefetch the combine operands of this thread's phase-B cells -----
        // (issued now so the HBM latency overlaps phase A)
        T pre1[NSLOT], pre2[NSLOT];
#pragma unroll
        for (int it = 0; it < ITEMS; ++it) {
#pragma unroll
            for (int r = 0; r < SEGB; ++r) {
                const int ic = (warp + it * NWARP) / NSEGB;
                const int rr = rb0 + r;
                const bool cvalid = fast || (pvalid && i0 + ic < Nq1 && j0 + rr < Nq2 && rr < TQ2);
                const long long g = tbase + it * item_step + r * colstride + p;
                pre1[it * SEGB + r] = (base1 && cvalid) ? base1[g] : T(0);
                pre2[it * SEGB + r] = (base2 && cvalid) ? base2[g] : T(0);
            }
        }

        // ---- phase A: q1 faces -> D1 = (-(F_R - F_L)) / dq1 ------------------
        {
            const bool right = v1 > T(0);
            const int off = right ? 0 : 1;
            Weno5Side<T> S; S.set(right);
            for (int item = warp; item < TQ2 * NSEG; item += NWARP) {
                const int jr = item / NSEG, sg = item % NSEG;
                const int cb = sg * SEG, ce = min(TQ1, cb + SEG);
                if (cb >= ce) continue;
                const T* row = X + ((Q2 ? jr + HALO : 0) * HX) * PW + lane + off * PW;
                // window for face f (between cells f-1 and f): cols f+off .. f+off+4
                T y0 = row[(cb + 0) * PW], y1 = row[(cb + 1) * PW];
                T y2 = row[(cb + 2) * PW], y3 = row[(cb + 3) * PW];
                T y4 = row[(cb + 4) * PW];
                FaceWalker<RECON, EXACT, T> W;
                T fv = W.first(y0, y1, y2, y3, y4, right, S);
                T Fprev = v1 * fv;
                double jsum_prev = double(fv);
#pragma unroll 2
                for (int cc = cb; cc < ce; ++cc) {
                    y0 = y1; y1 = y2; y2 = y3; y3 = y4;
                    y4 = row[(cc + 5) * PW];
                    T fn = W.next(y0, y1, y2, y3, y4, right, S);
                    T Fn = v1 * fn;
                    T d;
                    if (EXACT) d = (-(Fn - Fprev)) / T(a.dq1);
                    else d = (Fprev - Fn) * inv_dq1;
                    stage[(jr * TQ1 + cc) * PWP + lane] = d;
                    if (want_j) {
                        // J1 uses the state at each cell's left face (df_dt_fvm.py:214-216)
                        double c = pvalid ? jsum_prev * V1 : 0.0;
                        c = warp_sum(c);
                        if (lane == 0) j_acc[(jr * TQ1 + cc) * 3 + 0] += c;
                    }
                    Fprev = Fn;
                    jsum_prev = double(fn);
                }
            }
        }
        __syncthreads();

        // ---- phase B: q2 faces, BGK, RK combine, outputs ---------------------
        if (warp == 0) {
            vtab[0 * PW + lane] = pvalid ? V1 : 0.0;
            vtab[1 * PW + lane] = pvalid ? V2 : 0.0;
            vtab[2 * PW + lane] = pvalid ? V3 : 0.0;
            vtab[3 * PW + lane] = pvalid ? (V1 * V1 + V2 * V2) + V3 * V3 : 0.0;
        }
        {
            const bool right = v2 > T(0);
            const int off = right ? 0 : 1;
            Weno5Side<T> S; S.set(right);
            const int toff1 = jp1, toff2 = Np1 + jp2, toff3 = Np1 + Np2 + jp3;
#pragma unroll
            for (int it = 0; it < ITEMS; ++it) {
                const int item = warp + it * NWARP;
                const int ic = item / NSEGB;
                const T* col = X + (ic + HALO) * PW + lane;
                const T* colw = col + (rb0 + off) * HX * PW;
                T y0, y1, y2, y3, y4, Fprev = T(0), fprev = T(0);
                FaceWalker<RECON, EXACT, T> W;
                if (Q2) {
                    y0 = colw[0 * HX * PW]; y1 = colw[1 * HX * PW]; y2 = colw[2 * HX * PW];
                    y3 = colw[3 * HX * PW]; y4 = colw[4 * HX * PW];
                    fprev = W.first(y0, y1, y2, y3, y4, right, S);
                    Fprev = v2 * fprev;
                }
                // the FP64 reference-order body is long (divisions in the WENO
                // weights): rolled, it stays in the instruction cache
#pragma unroll (EXACT ? 1 : SEGB)
                for (int r = 0; r < SEGB; ++r) {
                    const int rr = rb0 + r;
                    if (rr >= TQ2) break;
                    const int ii = i0 + ic, jj = j0 + rr;
                    const bool cvalid = fast || (pvalid && ii < Nq1 && jj < Nq2);
                    const int cq = rr * TQ1 + ic;
                    T kq = stage[cq * PWP + lane];
                    T fcell = col[((Q2 ? rr + HALO : 0) * HX) * PW];
                    T fbot = fprev;
                    if (Q2) {
                        y0 = y1; y1 = y2; y2 = y3; y3 = y4;
                        y4 = colw[(r + 5) * HX * PW];
                        T fn = W.next(y0, y1, y2, y3, y4, right, S);
                        T Fn = v2 * fn;
                        if (EXACT) kq = kq - (Fn - Fprev) / T(a.dq2);
                        else kq = kq - (Fn - Fprev) * inv_dq2;
                        Fprev = Fn;
                        fprev = fn;
                    }
                    T kk = kq;
                    const long long gidx = tbase + it * item_step + r * colstride + p;
                    if (BGK) {
                        double fmb;
                        const double* qq = qc + cq * 5;
                        if (a.bgk_direct) {
                            // f0 of collision_operator.py:52-65 evaluated per cell
                            double d1v = V1 - qq[1];
                            fmb = qq[0] * exp((mneg * (d1v * d1v)) / qq[4]);
                            if (a.p_dim >= 2) {
                                double d2v = V2 - qq[2];
                                fmb = fmb * exp((mneg * (d2v * d2v)) / qq[4]);
                            }
                            if (a.p_dim == 3) {
                                double d3v = V3 - qq[3];
                                fmb = fmb * exp((mneg * (d3v * d3v)) / qq[4]);
                            }
                        } else {
                            const double* tb = tabs + cq * ntab;
                            fmb = (tb[toff1] * tb[toff2]) * tb[toff3];
                        }
                        if (EXACT) {
                            double tauv = tau_arr ? double(tau_arr[cvalid ? gidx : 0]) : a.tau;
                            kk = T(double(kk) + (-(double(fcell) - fmb) / tauv));
                        } else {
                            T itau = tau_arr ? T(1) / tau_arr[cvalid ? gidx : 0] : inv_tau;
                            kk = kk + (T(fmb) - fcell) * itau;
                        }
                    }
                    if (want_j) {
                        double jc2 = cvalid ? double(fbot) * V2 : 0.0;
                        double jc3 = cvalid ? double(fcell) * V3 : 0.0;
                        jc2 = warp_sum(jc2);
                        jc3 = warp_sum(jc3);
                        if (lane == 0) { j_acc[cq * 3 + 1] += jc2; j_acc[cq * 3 + 2] += jc3; }
                    }
                    // RK stage combine (fvm_operator.py:26,33; integrators.py:18-25)
                    const T o1 = base1 ? pre1[it * SEGB + r] + kk * c1 : kk;
                    if (cvalid) {
                        out1[gidx] = o1;
                        if (out2) out2[gidx] = pre2[it * SEGB + r] + kk * c2;
                        // wrap-around ghost copies (what the next halo refresh would do)
                        if (border && ((a.periodic1 && (ii < Ng || ii >= Nq1 - Ng)) ||
                                       (a.periodic2 && (jj < Ng || jj >= Nq2 - Ng))))
                            write_ghost_images(out1, o1, ii, jj, s, p, Ng, Nq1, Nq2,
                                               a.Nq1g, a.Nq2g, a.periodic1, a.periodic2,
                                               rowstride, colstride, Np);
                        // a q2 slab: the neighbours' ghost rows of the same buffer
                        if (a.peer_lo && jj < Ng)
                            static_cast<T*>(a.peer_lo)[gidx + (long long)Nq2 * colstride] = o1;
                        if (a.peer_hi && jj >= Nq2 - Ng)
                            static_cast<T*>(a.peer_hi)[gidx - (long long)Nq2 * colstride] = o1;
                        // a q1 block: the neighbours' ghost columns
                        if (a.peer_left && ii < Ng)
                            static_cast<T*>(a.peer_left)[gidx + (long long)Nq1 * rowstride] = o1;
                        if (a.peer_right && ii >= Nq1 - Ng)
                            static_cast<T*>(a.peer_right)[gidx - (long long)Nq1 * rowstride] = o1;
                        if (a.flag && !isfinite(o1)) atomicOr(a.flag, 1);
                    }
                    stage[cq * PWP + lane] = cvalid ? o1 : T(0);
                }
            }
        }
        __syncthreads();   // tile `buf` consumed, stage holds out1 of the chunk
        if (a.use_tma) fence_proxy_async();
        issue(k + NB, buf);

        // ---- phase C: FP64 moments of out1 (moments.py:6-24) ------------------
        if (want_mom) {
            const T* sp = stage + pc_c * PWP + pc_q * PQ;
            const double* vt = vtab + pc_q * PQ;
#pragma unroll
            for (int t = 0; t < PQ; ++t) {
                const double ov = double(sp[t]);
                macc[0] += ov;
                macc[1] += ov * vt[t];
                macc[2] += ov * vt[PW + t];
                macc[3] += ov * vt[2 * PW + t];
                macc[4] += (0.5 * ov) * vt[3 * PW + t];
            }
        }
        // advance this lane's p by one chunk
        p += PW;
        ip1 += PW;
        while (ip1 >= Np1) {
            ip1 -= Np1;
            if (++ip2 == Np2) { ip2 = 0; ++ip3; }
        }
    }
    __syncthreads();

    // ---- epilogue: partial moments / currents of this split ------------------
    const long long plane = (long long)Nq2 * Nq1;
    if (want_mom) {
        double* red = reinterpret_cast<double*>(smem_raw + Lo.tile);   // tile no longer used
#pragma unroll
        for (int q = 0; q < kNumMom; ++q) red[(pc_q * NQ + pc_c) * kNumMom + q] = macc[q];
        __syncthreads();
        for (int c = tid; c < NQ * kNumMom; c += NTHREADS) {
            int cq = c / kNumMom, q = c % kNumMom;
            double v = 0.0;
#pragma unroll
            for (int h = 0; h < NQUART; ++h) v += red[(h * NQ + cq) * kNumMom + q];
            int ii = i0 + cq % TQ1, jj = j0 + cq / TQ1;
            if (ii < Nq1 && jj < Nq2)
                a.mom_out[(((long long)split * kNumMom + q) * a.Ns + s) * plane
                          + (long long)jj * Nq1 + ii] = v;
        }
    }
    if (want_j && a.j_out) {
        for (int c = tid; c < NQ * 3; c += NTHREADS) {
            int cq = c / 3, q = c % 3;
            int ii = i0 + cq % TQ1, jj = j0 + cq / TQ1;
            if (ii < Nq1 && jj < Nq2)
                a.j_out[(((long long)split * 3 + q) * a.Ns + s) * plane
                        + (long long)jj * Nq1 + ii] = j_acc[c];
        }
    }
}

// ---------------------------------------------------------------------------
// p-stage kernel (fields enabled): one CTA per (interior q-cell, species)
// holds the whole p-block in shared memory.
//   k = k_q + (-(d1 + d2 + d3)),  d_a = (F_a(right) - F_a(left)) * (1/dp_a)
// (df_dt_fvm.py:245-323), with circular neighbours along each p axis, C_p
// from the cell-centred fields (advection_terms.py:147-188), then the RK
// combine and the FP64 moments of out1 (full sums: nsplit = 1).
// ---------------------------------------------------------------------------

// q / n and q % n for 0 <= q < 2^24 with n >= 1, from a float reciprocal
// and one correction step
struct PDiv {
    int n;
    float inv;
    __device__ __forceinline__ void set(int nn) { n = nn; inv = 1.0f / float(nn); }
    __device__ __forceinline__ int div(int q, int* rem) const {
        int d = __float2int_rz(float(q) * inv);
        int r = q - d * n;
        if (r < 0) { --d; r += n; }
        else if (r >= n) { ++d; r -= n; }
        *rem = r;
        return d;
    }
};

// flux at the left face of element c along an axis with n cells (n >= 3: a
// window position pos-3 .. pos+2 wraps at most once), pos its index along
// the axis, neighbours circular within the axis
template <int RECON, bool EXACT, typename T>
__device__ __forceinline__ T p_face_flux(const T* fb, int c, int stride, int n, int pos,
                                         T C, const Weno5Side<T>& Sr, const Weno5Side<T>& Sl) {
    const bool right = C > T(0);
    const int off = right ? -3 : -2;          // window start relative to the cell
    T y[5];
#pragma unroll
    for (int t = 0; t < 5; ++t) {
        int q = pos + off + t;
        if (n >= 3) {
            q = q < 0 ? q + n : (q >= n ? q - n : q);
        } else {
            q = ((q % n) + n) % n;
        }
        y[t] = fb[c + (q - pos) * stride];
    }
    T fv = face_value<RECON, EXACT>(y[0], y[1], y[2], y[3], y[4], right, right ? Sr : Sl);
    return C * fv;
}

template <typename T, bool EXACT, int RECON>
__global__ void __launch_bounds__(PTHREADS)
pstage_kernel(const __grid_constant__ PStageArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* fb = reinterpret_cast<T*>(smem_raw);      // [Np]
    T* Fx[3] = {fb + a.Np, fb + 2 * a.Np, fb + 3 * a.Np};   // left-face fluxes per p axis
    // p-cell centres of the species along p1, p2, p3 (after the four arrays,
    // 8-byte aligned)
    double* vg = reinterpret_cast<double*>(smem_raw + ((4 * (size_t)a.Np * sizeof(T) + 7) & ~(size_t)7));
    __shared__ double red[PTHREADS / 32][kNumMom];

    const int tid = threadIdx.x;
    const int ii = blockIdx.x % a.Nq1, jj = blockIdx.x / a.Nq1, s = blockIdx.y;
    const long long rowstride = (long long)a.Ns * a.Np;
    const long long colstride = rowstride * a.Nq1g;
    const long long cbase = (long long)(jj + a.Ng) * colstride + (long long)(ii + a.Ng) * rowstride
                          + (long long)s * a.Np;
    const T* fs = static_cast<const T*>(a.fs);
    const int n1 = a.Np1, n2 = a.Np2, n3 = a.Np3;
    for (int c = tid; c < a.Np; c += PTHREADS) fb[c] = fs[cbase + c];
    for (int q = tid; q < n1 + n2 + n3; q += PTHREADS) {
        if (q < n1) vg[q] = a.sg.p1_start[s] + (0.5 + q) * a.sg.dp1[s];
        else if (q < n1 + n2) vg[q] = a.sg.p2_start[s] + (0.5 + (q - n1)) * a.sg.dp2[s];
        else vg[q] = a.sg.p3_start[s] + (0.5 + (q - n1 - n2)) * a.sg.dp3[s];
    }
    const long long plane_g = (long long)a.Nq2g * a.Nq1g;
    const long long qg = (long long)(jj + a.Ng) * a.Nq1g + (ii + a.Ng);
    const double E1 = a.cell[0 * plane_g + qg], E2 = a.cell[1 * plane_g + qg];
    const double E3 = a.cell[2 * plane_g + qg], B1 = a.cell[3 * plane_g + qg];
    const double B2 = a.cell[4 * plane_g + qg], B3 = a.cell[5 * plane_g + qg];
    const double em = a.sg.charge[s] / a.sg.mass[s];
    Weno5Side<T> Sr, Sl;
    Sr.set(true);
    Sl.set(false);
    PDiv D1, D2;
    D1.set(n1);
    D2.set(n2);
    __syncthreads();

    // element c -> (i1, i2, i3)
    auto split = [&](int c, int& i1, int& i2, int& i3) {
        const int r12 = D1.div(c, &i1);
        i3 = D2.div(r12, &i2);
    };
    // left-face fluxes of every element along each p axis with more than one
    // cell (a single-cell axis contributes exactly zero), one pass
    for (int c = tid; c < a.Np; c += PTHREADS) {
        int i1, i2, i3;
        split(c, i1, i2, i3);
        const double v1 = vg[i1], v2 = vg[n1 + i2], v3 = vg[n1 + n2 + i3];
        if (n1 > 1)
            Fx[0][c] = p_face_flux<RECON, EXACT>(fb, c, 1, n1, i1,
                                                 T(em * ((E1 + v2 * B3) - v3 * B2)), Sr, Sl);
        if (n2 > 1)
            Fx[1][c] = p_face_flux<RECON, EXACT>(fb, c, n1, n2, i2,
                                                 T(em * ((E2 + v3 * B1) - v1 * B3)), Sr, Sl);
        if (n3 > 1)
            Fx[2][c] = p_face_flux<RECON, EXACT>(fb, c, n1 * n2, n3, i3,
                                                 T(em * ((E3 + v1 * B2) - v2 * B1)), Sr, Sl);
    }
    __syncthreads();
    // final combine
    T* out1 = static_cast<T*>(a.out1);
    T* out2 = static_cast<T*>(a.out2);
    const T* base1 = static_cast<const T*>(a.base1);
    const T* base2 = static_cast<const T*>(a.base2);
    const T* kq = static_cast<const T*>(a.kq);
    double macc[kNumMom] = {0, 0, 0, 0, 0};
    const T c1 = T(a.c1), c2 = T(a.c2);
    const bool ghost_cell = (a.periodic1 && (ii < a.Ng || ii >= a.Nq1 - a.Ng)) ||
                            (a.periodic2 && (jj < a.Ng || jj >= a.Nq2 - a.Ng));
    const T inv1 = T(1.0 / a.sg.dp1[s]), inv2 = T(1.0 / a.sg.dp2[s]);
    const T inv3 = T(1.0 / a.sg.dp3[s]);
    for (int c = tid; c < a.Np; c += PTHREADS) {
        int i1, i2, i3;
        split(c, i1, i2, i3);
        // d_a = (F_a(right face) - F_a(left face)) / dp_a, circular along the axis
        T t1 = T(0), t2 = T(0), t3 = T(0);
        if (n1 > 1) {
            const int cn = i1 + 1 < n1 ? c + 1 : c - (n1 - 1);
            t1 = (Fx[0][cn] - Fx[0][c]) * inv1;
        }
        if (n2 > 1) {
            const int cn = i2 + 1 < n2 ? c + n1 : c - (n2 - 1) * n1;
            t2 = (Fx[1][cn] - Fx[1][c]) * inv2;
        }
        if (n3 > 1) {
            const int cn = i3 + 1 < n3 ? c + n1 * n2 : c - (n3 - 1) * n1 * n2;
            t3 = (Fx[2][cn] - Fx[2][c]) * inv3;
        }
        const long long g = cbase + c;
        if (a.term) {
            // one p-flux divergence (df_dt_fvm.py:325-335 term_to_return)
            out1[g] = a.term == 1 ? t1 : (a.term == 2 ? t2 : t3);
            continue;
        }
        T kk = kq[g] + (-((t1 + t2) + t3));
        T o1 = base1 ? base1[g] + kk * c1 : kk;
        out1[g] = o1;
        if (out2) out2[g] = base2[g] + kk * c2;
        if (ghost_cell)
            write_ghost_images(out1, o1, ii, jj, s, c, a.Ng, a.Nq1, a.Nq2, a.Nq1g, a.Nq2g,
                               a.periodic1, a.periodic2, rowstride, colstride, a.Np);
        if (a.flag && !isfinite(double(o1))) atomicOr(a.flag, 1);
        if (a.mom_out) {
            const double w1 = vg[i1], w2 = vg[n1 + i2], w3 = vg[n1 + n2 + i3];
            const double vsq = (w1 * w1 + w2 * w2) + w3 * w3;
            const double ov = double(o1);
            macc[0] += ov; macc[1] += ov * w1; macc[2] += ov * w2; macc[3] += ov * w3;
            macc[4] += (0.5 * ov) * vsq;
        }
    }
    if (a.mom_out) {
        const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
        for (int q = 0; q < kNumMom; ++q) {
            double v = warp_sum(macc[q]);
            if (lane == 0) red[warp][q] = v;
        }
        __syncthreads();
        if (tid < kNumMom) {
            double v = 0.0;
            for (int w = 0; w < PTHREADS / 32; ++w) v += red[w][tid];
            const long long plane = (long long)a.Nq2 * a.Nq1;
            a.mom_out[((long long)tid * a.Ns + s) * plane + (long long)jj * a.Nq1 + ii] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// moments (compute_moments.py:7-59 with moments.py:6-58), FP64 output.
// One CTA per (ghosted q-cell, species).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256)
moment_kernel(const T* f, int mid, double* out, int Ns, int Np1, int Np2, int Np3, int Nq1g,
              int Nq2g, SpeciesGrid sg) {
    __shared__ double red[8];
    const int q = blockIdx.x, s = blockIdx.y, tid = threadIdx.x;
    const int Np = Np1 * Np2 * Np3;
    const T* fp = f + ((long long)q * Ns + s) * Np;
    double acc = 0.0;
    for (int c = tid; c < Np; c += 256) {
        const int i1 = c % Np1, i2 = (c / Np1) % Np2, i3 = c / (Np1 * Np2);
        const PVel V = lane_velocity(sg, s, i1, i2, i3);
        const double fv = double(fp[c]);
        double g;
        switch (mid) {
            case 0: g = fv; break;
            case 1: g = fv * V.v1; break;
            case 2: g = fv * V.v2; break;
            case 3: g = fv * V.v3; break;
            case 4: g = (0.5 * fv) * V.vsq; break;
            case 5: g = (0.5 * fv) * (V.v1 * V.v1); break;
            case 6: g = (0.5 * fv) * (V.v2 * V.v2); break;
            case 7: g = (0.5 * fv) * (V.v3 * V.v3); break;
            case 8: g = (fv * V.v1) * V.vsq; break;
            case 9: g = (fv * V.v2) * V.vsq; break;
            default: g = (fv * V.v3) * V.vsq; break;
        }
        acc += g;
    }
    acc = warp_sum(acc);
    if ((tid & 31) == 0) red[tid >> 5] = acc;
    __syncthreads();
    if (tid == 0) {
        double v = 0.0;
        for (int w = 0; w < 8; ++w) v += red[w];
        const double measure = (sg.dp3[s] * sg.dp2[s]) * sg.dp1[s];
        out[(long long)q * Ns + s] = sg.polar2d ? sg.mom_scale * (v * measure) : v * measure;
    }
}

// 16-byte vectors of f: 4 FP32 or 2 FP64 values
template <typename T> struct Vec16;
template <> struct Vec16<float> {
    typedef float4 V;
    static constexpr int n = 4;
    __device__ static void get(const V& v, double (&o)[4]) { o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; }
};
template <> struct Vec16<double> {
    typedef double2 V;
    static constexpr int n = 2;
    __device__ static void get(const V& v, double (&o)[2]) { o[0] = v.x; o[1] = v.y; }
};

// Moment sums of n consecutive p of one p1 row, values o_t at v1 = V1 + t dp1
// (t = 0..n-1), v2, v3 fixed: from S0 = sum o_t, S1 = sum t o_t, S2 = sum t^2 o_t
// (moments.py:6-24 with the p1 velocities of the row)
template <int n>
__device__ __forceinline__ void add_moment_run(const double (&o)[n], double V1, double dp1,
                                               double v2, double v3, double (&acc)[kNumMom]) {
    double S0 = 0.0, S1 = 0.0, S2 = 0.0;
#pragma unroll
    for (int t = 0; t < n; ++t) {
        S0 += o[t];
        S1 = fma(double(t), o[t], S1);
        S2 = fma(double(t * t), o[t], S2);
    }
    acc[0] += S0;
    acc[1] = fma(V1, S0, fma(dp1, S1, acc[1]));
    acc[2] = fma(v2, S0, acc[2]);
    acc[3] = fma(v3, S0, acc[3]);
    const double e0 = fma(V1, V1, fma(v2, v2, v3 * v3));
    acc[4] = fma(0.5, fma(e0, S0, fma(2.0 * V1 * dp1, S1, (dp1 * dp1) * S2)), acc[4]);
}

// (i1, i2, i3) of a p-cell index that a thread advances by a fixed stride,
// kept without divisions: the stride is split once into its p1 remainder and
// its p2 / p3 row steps, and each advance carries from p1 into p2 and from p2
// into p3 (each part stays below twice its range, so one subtraction does)
struct PCellWalk {
    int i1, i2, i3;        // current p-cell
    int d1, d2, d3;        // the stride as (p1, p2, p3) steps
    int Np1, Np2;
    __device__ __forceinline__ PCellWalk(int p, int stride, int np1, int np2)
        : Np1(np1), Np2(np2) {
        i1 = p % np1;
        const int r = p / np1;
        i2 = r % np2;
        i3 = r / np2;
        d1 = stride % np1;
        const int rs = stride / np1;
        d2 = rs % np2;
        d3 = rs / np2;
    }
    __device__ __forceinline__ void advance() {
        i1 += d1;
        int c = 0;
        if (i1 >= Np1) { i1 -= Np1; c = 1; }
        i2 += d2 + c;
        c = 0;
        if (i2 >= Np2) { i2 -= Np2; c = 1; }
        i3 += d3 + c;
    }
};

// The five BGK moments of the interior cells as one "split" of partial sums
// ([1][5][Ns][Nq2][Nq1], sums without the measure factor).  One CTA per q-cell
// streams its p-block in 16-byte vectors, four in flight per thread (N_p1 a
// multiple of the vector width; otherwise one value at a time).
template <typename T>
__global__ void __launch_bounds__(256)
moments5_kernel(const T* f, double* part, int Ns, int Np1, int Np2, int Np3, int Nq1, int Nq2,
                int Ng, SpeciesGrid sg) {
    __shared__ double red[8][kNumMom];
    const int q = blockIdx.x, s = blockIdx.y, tid = threadIdx.x;
    const int ii = q % Nq1, jj = q / Nq1;
    const int Np = Np1 * Np2 * Np3;
    const int Nq1g = Nq1 + 2 * Ng;
    const T* fp = f + (((long long)(jj + Ng) * Nq1g + (ii + Ng)) * Ns + s) * Np;
    double acc[kNumMom] = {0, 0, 0, 0, 0};
    typedef Vec16<T> VT;
    constexpr int VN = VT::n;
    if (Np1 % VN == 0 && (reinterpret_cast<uintptr_t>(f) & 15) == 0) {
        const typename VT::V* fv = reinterpret_cast<const typename VT::V*>(fp);
        const int nv = Np / VN;
        const double p1s = sg.p1_start[s], p2s = sg.p2_start[s], p3s = sg.p3_start[s];
        const double dp1 = sg.dp1[s], dp2 = sg.dp2[s], dp3 = sg.dp3[s];
        // the vectors c = tid, tid + 256, ... in that order: p-cell c * VN
        PCellWalk w(tid * VN, 256 * VN, Np1, Np2);
        for (int c0 = tid; c0 < nv; c0 += 4 * 256) {
            typename VT::V v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (c0 + u * 256 < nv) v[u] = __ldg(fv + c0 + u * 256);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int c = c0 + u * 256;
                if (c >= nv) break;
                double o[VN];
                VT::get(v[u], o);
                add_moment_run<VN>(o, p1s + (0.5 + w.i1) * dp1, dp1, p2s + (0.5 + w.i2) * dp2,
                                   p3s + (0.5 + w.i3) * dp3, acc);
                w.advance();
            }
        }
    } else {
        for (int c = tid; c < Np; c += 256) {
            const int i1 = c % Np1, i2 = (c / Np1) % Np2, i3 = c / (Np1 * Np2);
            const PVel V = lane_velocity(sg, s, i1, i2, i3);
            const double fv = double(fp[c]);
            acc[0] += fv; acc[1] += fv * V.v1; acc[2] += fv * V.v2; acc[3] += fv * V.v3;
            acc[4] += (0.5 * fv) * V.vsq;
        }
    }
#pragma unroll
    for (int m = 0; m < kNumMom; ++m) {
        double v = warp_sum(acc[m]);
        if ((tid & 31) == 0) red[tid >> 5][m] = v;
    }
    __syncthreads();
    if (tid < kNumMom) {
        double v = 0.0;
        for (int w = 0; w < 8; ++w) v += red[w][tid];
        part[((long long)tid * Ns + s) * Nq2 * Nq1 + (long long)jj * Nq1 + ii] = v;
    }
}

// ---------------------------------------------------------------------------
// halo refresh: communicate_f (periodic wrap; ghosted halos are zero), then
// apply_bcs_f per axis (boundaries.py:415-577): the mirror image
// (boundaries.py:226-413, cartesian or polar2D p-grid) and/or the Dirichlet inflow
// select (:147-225).  Every value is read from an interior cell, so one pass
// gives the reference's sequential left, right, bottom, top result everywhere
// except in the corner cells (ghost in both q1 and q2) of mixed mirror /
// Dirichlet axes, which no interior update reads (the q1 and q2 stencils are
// separate).
// One CTA per ghost cell (grid-stride over the cells): the cell, its source
// cell and its kind are worked out once; the cell's (species, p) block is
// contiguous, so a plain image (periodic, or zero) is a copy of the source
// cell's block in 16-byte vectors, and only cells whose values depend on p
// (a mirror's velocity reflection, a Dirichlet inflow select, a shearing-box
// resample) go element by element.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256)
ghost_kernel(T* f, const T* dl, const T* dr, const T* db, const T* dt,
             int Nq1, int Nq2, int Ng, int Ns, int Np, int Np1, int Np2,
             int per1, int per2, int dir1, int dir2, int mir1, int mir2,
             int ext1, int ext2, SpeciesGrid sg, GhostShear sh,
             long long nghost_cells) {
    const int Nq1g = Nq1 + 2 * Ng;
    const int rowlen = Ns * Np;                            // one q-cell's values
    const long long rowstride = rowlen;
    const long long colstride = rowstride * Nq1g;
    const long long nrow = (long long)Ng * Nq1g;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (long long gc = blockIdx.x; gc < nghost_cells; gc += gridDim.x) {
        // enumerate ghost cells: rows [0,Ng) and [Nq2+Ng, Nq2g) full width, then
        // the left/right ghost columns of the interior rows
        int g1, g2;
        if (gc < 2 * nrow) {
            const int r = int(gc / Nq1g), c = int(gc % Nq1g);
            g2 = r < Ng ? r : Nq2 + r;          // r in [Ng, 2Ng) -> Nq2+Ng .. Nq2+2Ng-1
            g1 = c;
        } else {
            const long long rem = gc - 2 * nrow;
            const int r = int(rem / (2 * Ng)), c = int(rem % (2 * Ng));
            g2 = Ng + r;
            g1 = c < Ng ? c : Nq1 + c;
        }
        const int i = g1 - Ng, j = g2 - Ng;
        const bool in1 = i >= 0 && i < Nq1, in2 = j >= 0 && j < Nq2;
        // ghost rows / columns of an external axis belong to the caller
        if ((ext1 && !in1) || (ext2 && !in2)) continue;
        const long long g = (long long)g2 * colstride + (long long)g1 * rowstride;
        T* dst = f + g;
        // a shearing-box strip (every cell of the N_g ghost columns or rows,
        // corners included): the periodic image resampled along the other axis
        if ((sh.axis == 1 && !in1) || (sh.axis == 2 && !in2)) {
            const bool lo = sh.axis == 1 ? i < 0 : j < 0;
            const int N = sh.axis == 1 ? Nq2 : Nq1;           // resampled axis
            const int own = sh.axis == 1 ? g2 : g1;           // position along it
            double pos = (sh.start + (own - Ng) * sh.dq) + 0.5 * sh.dq;     // ghosted centre
            pos = lo ? pos - sh.shift : pos + sh.shift;
            const double L = sh.end - sh.start;
            for (int it = 0; it < 4 && pos > sh.end; ++it) pos -= L;
            for (int it = 0; it < 4 && pos < sh.start; ++it) pos += L;
            // continuous index among the ghosted centres, then interior indices
            const double x = (pos - ((sh.start + (-Ng) * sh.dq) + 0.5 * sh.dq)) / sh.dq;
            const int jb = (int)floor(x);
            const double t = x - jb;
            const int fixed = sh.axis == 1 ? ((i % Nq1) + Nq1) % Nq1 : ((j % Nq2) + Nq2) % Nq2;
            const T* src[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int m = (((jb - 1 + k - Ng) % N) + N) % N;   // periodic extension
                const int ci = sh.axis == 1 ? fixed : m, cj = sh.axis == 1 ? m : fixed;
                src[k] = f + (long long)(cj + Ng) * colstride + (long long)(ci + Ng) * rowstride;
            }
            for (int sp = tid; sp < rowlen; sp += nt) {
                double pv[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) pv[k] = double(src[k][sp]);
                // Catmull-Rom cubic between pv[1] and pv[2] (tangents (pv[k+1]-pv[k-1])/2)
                const double v = pv[1] + 0.5 * t * ((pv[2] - pv[0]) +
                                 t * ((2.0 * pv[0] - 5.0 * pv[1] + 4.0 * pv[2] - pv[3]) +
                                      t * (3.0 * (pv[1] - pv[2]) + pv[3] - pv[0])));
                dst[sp] = T(v);
            }
            continue;
        }
        // source cell: periodic wrap, or the mirror image across the edge
        // (ghost i < 0 <- interior -1-i, i >= N <- 2N-1-i); none (zero) for a
        // non-periodic, non-mirror axis
        int si = i, sj = j;
        bool have = true;
        const bool m1 = !in1 && !per1 && mir1, m2 = !in2 && !per2 && mir2;
        if (!in2) {
            if (per2) sj = ((j % Nq2) + Nq2) % Nq2;
            else if (mir2) sj = j < 0 ? -1 - j : 2 * Nq2 - 1 - j;
            else have = false;
        }
        if (!in1) {
            if (per1) si = ((i % Nq1) + Nq1) % Nq1;
            else if (mir1) si = i < 0 ? -1 - i : 2 * Nq1 - 1 - i;
            else have = false;
        }
        const bool d1 = dir1 && !in1, d2 = dir2 && !in2;
        const T* src = f + (long long)(sj + Ng) * colstride + (long long)(si + Ng) * rowstride;
        if (!m1 && !m2 && !d1 && !d2) {
            // the same (species, p) block as the source cell, or zeros
            constexpr int VW = 16 / (int)sizeof(T);
            if ((rowlen % VW) == 0 && (reinterpret_cast<uintptr_t>(f) & 15) == 0) {
                typedef typename Vec16<T>::V V;
                const V* s4 = reinterpret_cast<const V*>(src);
                V* d4 = reinterpret_cast<V*>(dst);
                const int nv = rowlen / VW;
                if (have) {
                    for (int k = tid; k < nv; k += nt) d4[k] = s4[k];
                } else {
                    V z;
                    memset(&z, 0, sizeof(z));
                    for (int k = tid; k < nv; k += nt) d4[k] = z;
                }
            } else {
                for (int sp = tid; sp < rowlen; sp += nt) dst[sp] = have ? src[sp] : T(0);
            }
            continue;
        }
        // element by element: the velocity reflected across a mirror edge.
        // Cartesian grid (boundaries.py:226-301): the normal velocity index
        // reversed, p1 at q1 edges, p2 at q2 edges.  Polar2D grid
        // (boundaries.py:313-413, p2 the angle theta): at q2 edges
        // theta -> -theta, the p2 index reversed; at q1 edges
        // theta -> pi - theta, each half of the p2 index range reversed on its
        // own.  The reference applies the q1 edges before the q2 edges, so a
        // corner ghost takes the q1 map of the q2 map of its own p2 index.
        // Then the Dirichlet inflow values where the velocity normal to the
        // edge points into the domain.
        for (int sp = tid; sp < rowlen; sp += nt) {
            const int p = sp % Np;
            const int i1 = p % Np1, i2 = (p / Np1) % Np2;
            int ps = sp, k2 = i2;                          // source p2 index
            if (m2) k2 = Np2 - 1 - k2;
            if (m1) {
                if (sg.polar2d) {
                    const int H = Np2 / 2;
                    k2 = k2 < H ? H - 1 - k2 : Np2 - 1 + H - k2;
                } else {
                    ps += Np1 - 1 - 2 * i1;
                }
            }
            ps += Np1 * (k2 - i2);
            T v = have ? src[ps] : T(0);
            const int s = sp / Np;
            const double v1 = sg.p1_start[s] + (0.5 + i1) * sg.dp1[s];
            const double v2 = sg.p2_start[s] + (0.5 + i2) * sg.dp2[s];
            if (d1 && i < 0 && v1 > 0) v = dl[g + sp];
            if (d1 && i >= Nq1 && v1 < 0) v = dr[g + sp];
            if (d2 && j < 0 && v2 > 0) v = db[g + sp];
            if (d2 && j >= Nq2 && v2 < 0) v = dt[g + sp];
            dst[sp] = v;
        }
    }
}

}  // namespace bolt
