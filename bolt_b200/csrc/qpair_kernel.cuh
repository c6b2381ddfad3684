// qpair_kernel.cuh - paired WENO5 q-stage kernel (sm_100a), FP32 or FP64.
//
// The fused RK stage of the 2D3V FVM update with fields off
// (df_dt_fvm.py:56-97 q-part + BGK source, combined with the stage update of
// integrators.py:15-28 / fvm_operator.py:26,33) for an 8x8 q-tile and 32
// consecutive p-cells of one species per chunk.  Every thread walks two
// adjacent q-rows or q-columns of the same p at once, as a pair: f32x2
// arithmetic in FP32, two FMA-contracted FP64 operations with Newton-refined
// reciprocals in FP64.  The two directions run side by side in different
// warps, each walker covering a whole 8-cell line (9 faces):
//
//   q1 walkers  warps 0-3, warp w: rows 2w, 2w+1; q1 part of df/dt + BGK
//               source -> D1 tile, then a named-barrier arrival
//   q2 walkers  warps 4-7, warp w: cols 2(w-4), 2(w-4)+1; q2 flux differences
//               held in registers, then (after the named barrier) k = D1 +
//               q2 part, out1 = base1 + c1 k, out2 = base2 + c2 k into shared
//               staging tiles
//   phase C     all warps, after the CTA barrier that closes the chunk: FP64
//               velocity moments of out1 and the divergence check
//
// All global traffic of the FP32 form is TMA: the halo tile of the stage input (14x14x32,
// double-buffered), the base1 tile (8x8x32, double-buffered; taken from the
// halo tile when it is the stage input itself) and the out1/out2 tiles; an
// out2 that is its own base (the RK4 accumulator) gets c2 k by TMA reduce-add
// (stores from shared memory, bulk-group completion).  out1 is staged with
// the 128-byte swizzle so that phase C reads 8 consecutive p of one q-cell as
// two conflict-free 16-byte loads.  Barrier waits are time-bounded and a
// failure is made CTA-uniform, recorded in the error word, and ends the work.
//
// FP64 differences: the out1 staging tile is two 128-byte-swizzled halves of
// 16 p each (the swizzle covers 128-byte rows), stored by two TMA stores; the
// RK4 accumulator's increment goes from the q2 walkers' registers into global
// memory by red.global.add.f64 (coalesced 256-byte rows; the TMA unit has no
// FP64 tensor reduction, and 64 row-wise bulk reductions issued by one warp
// held that warp back by a third of each chunk); one CTA per SM (221 KB of
// shared memory).  With one CTA per SM the FP64 form walks ONE row (column)
// per thread (ROWS = 1): 16 warps, q1 walkers warps 0-7 (row w, + BGK, then
// the periodic ghost images), q2 walkers warps 8-15 (column w-8, then phase
// C), at most 128 registers, so that twice the warps hide the FP64 latencies
// that a single 8-warp CTA left exposed.
//
// Launch conditions (checked by the host): FP32 or FP64, any reconstruction in q, 8x8 tiling,
// N_q1, N_q2 multiples of 8 and at least 2 N_g, N_p multiple of 32, N_p1
// multiple of 8, BGK by exp tables, all five buffers 16-byte aligned, f with
// fewer than 2^31 elements (32-bit offsets).
#pragma once

#include <type_traits>

#include "fvm_kernels.cuh"

namespace bolt {

// Geometry of the out1 staging tile: CS elements of one q-cell per 128-byte
// row (32 FP32, or 16 FP64 with the 32 p split into two halves of 64 rows),
// VE elements per 16-byte chunk; the 128-byte swizzle XORs the chunk index
// with (q-cell mod 8).
template <typename E> struct PairStage;
template <> struct PairStage<float> {
    static constexpr int CS = 32, VE = 4;
};
template <> struct PairStage<double> {
    static constexpr int CS = 16, VE = 2;
};

// staging-tile index of element p (0..31) of q-cell c
template <typename E>
__device__ __forceinline__ int stg(int c, int p) {
    constexpr int CS = PairStage<E>::CS, VE = PairStage<E>::VE;
    const int h = p / CS, pp = p % CS;
    return h * 64 * CS + c * CS + ((((pp / VE) ^ (c & 7)) * VE) | (pp % VE));
}

// the 8 consecutive elements of a q-cell row starting at 16-byte chunk ch0
// (key = q-cell mod 8), as FP64
__device__ __forceinline__ void load8(const float* row, int ch0, int key, double (&o)[8]) {
    const float4 u = reinterpret_cast<const float4*>(row)[ch0 ^ key];
    const float4 w = reinterpret_cast<const float4*>(row)[(ch0 + 1) ^ key];
    o[0] = u.x; o[1] = u.y; o[2] = u.z; o[3] = u.w;
    o[4] = w.x; o[5] = w.y; o[6] = w.z; o[7] = w.w;
}
__device__ __forceinline__ void load8(const double* row, int ch0, int key, double (&o)[8]) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double2 v = reinterpret_cast<const double2*>(row)[(ch0 + j) ^ key];
        o[2 * j] = v.x;
        o[2 * j + 1] = v.y;
    }
}

__device__ __forceinline__ float2 mk2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk2(double a, double b) { return make_double2(a, b); }

// Prologue (the tile loads already in flight): p-cell centres of the species,
// and for BGK the Maxwellian of the stage input per q-cell with exp tables
// over the p1 and p2 cells and the CTA's p3 rows [p3lo, p3lo + n3) stored as element
// pairs over q-cell pairs P = m*8 + col (cells of rows 2m and 2m+1 in one tile
// column, the pair a q1 walker holds): tab[q*kTabPitch + P], the pitch of 33
// pairs keeping a warp's reads of different q (one per lane) on distinct banks.
template <typename E, bool BGK, int NT>
__device__ __forceinline__ void qpair_prologue(const QStageArgs& a, int s, int i0, int j0,
                                               double* vgrid, double* qc,
                                               typename PairOf<E>::P* tabs, int p3lo, int n3) {
    static_assert(NT >= 256, "moment-sum mapping needs 256 threads");
    const int tid = threadIdx.x;
    const int Np1 = a.Np1, Np2 = a.Np2;
    const int ntab = Np1 + Np2 + a.Np3;
    for (int q = tid; q < ntab; q += NT) {
        if (q < Np1) vgrid[q] = a.sg.p1_start[s] + (0.5 + q) * a.sg.dp1[s];
        else if (q < Np1 + Np2) vgrid[q] = a.sg.p2_start[s] + (0.5 + (q - Np1)) * a.sg.dp2[s];
        else vgrid[q] = a.sg.p3_start[s] + (0.5 + (q - Np1 - Np2)) * a.sg.dp3[s];
    }
    if (BGK) {
        // the 64 cells' moment sums: thread t sums moment t/64 of cell t%64
        // (threads 0-63 also moment 4), all its partial-slot loads issued
        // before the first add, so the CTA waits for one round of loads; then
        // each cell's parameters from its sums
        static_assert(kNumMom == 5, "moment-sum mapping");
        double* mm = qc + 64 * kNumMom;
        if (NT == 256 || tid < 256) {
            const int c = tid & 63, q = tid >> 6;
            const int ii = i0 + (c & 7), jj = j0 + (c >> 3);
            const long long plane = (long long)a.Nq2 * a.Nq1;
            const long long step = (long long)kNumMom * a.Ns * plane;
            const double* src = a.mom_in + ((long long)q * a.Ns + s) * plane +
                                (long long)jj * a.Nq1 + ii;
            const double* src4 = src + 4 * (long long)a.Ns * plane;
            double v = 0.0, v4 = 0.0;
            const int n = a.nsplit_in;
            int sp = 0;
            if (q == 0) {
                for (; sp + 4 <= n; sp += 4) {
                    double l[4], l4[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        l[i] = src[(sp + i) * step];
                        l4[i] = src4[(sp + i) * step];
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        v += l[i];
                        v4 += l4[i];
                    }
                }
                for (; sp < n; ++sp) { v += src[sp * step]; v4 += src4[sp * step]; }
                mm[c * kNumMom + 4] = v4;
            } else {
                for (; sp + 8 <= n; sp += 8) {
                    double l[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) l[i] = src[(sp + i) * step];
#pragma unroll
                    for (int i = 0; i < 8; ++i) v += l[i];
                }
                for (; sp < n; ++sp) v += src[sp * step];
            }
            mm[c * kNumMom + q] = v;
        }
        __syncthreads();
        for (int c = tid; c < 64; c += NT)
            bgk_params_from_sums<true>(a, s, mm + c * kNumMom, qc + c * 5);
    }
    __syncthreads();
    if (BGK) {
        // One (q-cell, axis) per thread: the axis's exp factors
        // e_j = exp(-beta x_j^2), x_j = v_j - u, beta = m / (2 kB T), from the
        // row nearest u outwards by e_{j+1} = e_j g_j, g_{j+1} = g_j exp(-2 beta dv^2)
        // (and mirrored below it), so each factor shrinks away from the maximum
        // and nothing overflows; three exps per axis instead of one per row.  The
        // products carry about j^2/2 roundings (under 1e-13 relative at 24 rows).
        const double m = a.sg.mass[s];
        const int n12 = Np1 + Np2;
        E* tel = reinterpret_cast<E*>(tabs);
        for (int t = tid; t < 64 * 3; t += NT) {
            const int c = t & 63, ax = t >> 6;
            const double* qq = qc + c * 5;
            // the table column of cell c: pair P, component hi (row 2m+1 of the pair)
            E* col = tel + 2 * ((c >> 4) * 8 + (c & 7)) + ((c >> 3) & 1);
            const int r0 = ax == 0 ? 0 : (ax == 1 ? Np1 : n12);
            const int nr = ax == 0 ? Np1 : (ax == 1 ? Np2 : n3);
            const int q0 = ax == 2 ? n12 + p3lo : r0;           // p-cell of row r0
            const double dv = ax == 0 ? a.sg.dp1[s] : (ax == 1 ? a.sg.dp2[s] : a.sg.dp3[s]);
            const double scale = ax == 0 ? qq[0] : 1.0;         // p1 rows carry n*A
            const bool act = ax == 0 || (ax == 1 ? a.p_dim >= 2 : a.p_dim == 3);
            E* out = col + 2 * kTabPitch * r0;
            if (!act) {
                for (int j = 0; j < nr; ++j) out[2 * kTabPitch * j] = E(scale);
                continue;
            }
            const double u = qq[1 + ax], beta = m / qq[4];
            int jc = (int)floor((u - vgrid[q0]) / dv + 0.5);
            jc = min(max(jc, 0), nr - 1);
            const double x = vgrid[q0 + jc] - u;
            const double e = exp(-beta * (x * x));
            const double cc = exp(-2.0 * beta * (dv * dv));
            out[2 * kTabPitch * jc] = E(scale * e);
            double ej = e, g = exp(-beta * fma(2.0 * x, dv, dv * dv));
            for (int j = jc + 1; j < nr; ++j) {
                ej *= g;
                g *= cc;
                out[2 * kTabPitch * j] = E(scale * ej);
            }
            ej = e;
            g = exp(-beta * fma(-2.0 * x, dv, dv * dv));
            for (int j = jc - 1; j >= 0; --j) {
                ej *= g;
                g *= cc;
                out[2 * kTabPitch * j] = E(scale * ej);
            }
        }
    }
    __syncthreads();
}

// Tiles of an n1 x n2 tile grid split by a ring e1 tiles wide along q1 and e2
// along q2: the inner rectangle, row-major ...
__device__ __forceinline__ void tile_inner(int n1, int e1, int e2, int bx, int& t1, int& t2) {
    const int w = n1 - 2 * e1;
    t1 = e1 + bx % w;
    t2 = e2 + bx / w;
}

// ... and the ring: its bottom rows, the outer columns of the middle rows,
// its top rows
__device__ __forceinline__ void tile_ring(int n1, int n2, int e1, int e2, int bx, int& t1,
                                          int& t2) {
    if (bx < e2 * n1) {
        t1 = bx % n1;
        t2 = bx / n1;
        return;
    }
    bx -= e2 * n1;
    const int mid = max(0, n2 - 2 * e2);
    const int m = n1 > 2 * e1 ? 2 * e1 : n1;    // ring tiles of a middle row
    if (bx < mid * m) {
        t2 = e2 + bx / m;
        const int c = bx % m;
        t1 = m == n1 ? c : (c < e1 ? c : n1 - 2 * e1 + c);
        return;
    }
    bx -= mid * m;
    t1 = bx % n1;
    t2 = n2 - e2 + bx / n1;
}

// The q-tile of grid column bx.  tile_sel 0: every tile, those that write
// periodic images (the ring along periodic axes) first, so that the last CTAs
// of a launch are the shorter inner ones; 1: the tiles whose halo stays inside
// the block's interior along its external axes (ext1 / ext2); 2: the other
// tiles.  An 8x8 tile's halo reaches 3 cells past it, so only the outermost
// tiles read ghost cells.
__device__ __forceinline__ void qpair_tile(const QStageArgs& a, int bx, int& t1, int& t2) {
    const int n1 = a.ntiles1, n2 = a.ntiles2;
    if (a.tile_sel == 0) {
        const int e1 = a.periodic1 ? 1 : 0, e2 = a.periodic2 ? 1 : 0;
        const int ring = n1 * n2 - max(0, n1 - 2 * e1) * max(0, n2 - 2 * e2);
        if (bx < ring) tile_ring(n1, n2, e1, e2, bx, t1, t2);
        else tile_inner(n1, e1, e2, bx - ring, t1, t2);
        return;
    }
    const int e1 = a.ext1 ? 1 : 0, e2 = a.ext2 ? 1 : 0;
    if (a.tile_sel == 1) tile_inner(n1, e1, e2, bx, t1, t2);
    else tile_ring(n1, n2, e1, e2, bx, t1, t2);
}

// Stage modes (which of out1 = base1 + c1 k, out2 = base2 + c2 k exist and
// where their bases come from):
//   QP_X1   base1 = stage input (from the halo tile), out1 only
//   QP_X2   base1 = base2 = stage input, out1 and out2 stored
//   QP_B1   base1 tiles loaded (double-buffered), out1 only
//   QP_B1R2 base1 tiles loaded, out2 = base2 in place: c2 k is added to it by
//           a TMA reduce-add (no base2 load)
//   QP_K    out1 = k itself (the q-part of df/dt when a p-stage follows: fields
//           enabled), no base, no moments
enum QPairMode { QP_X1 = 0, QP_X2 = 1, QP_B1 = 2, QP_B1R2 = 3, QP_K = 4 };

template <typename E, bool BGK, int MODE, int RECON, int ROWS>
__global__ void __launch_bounds__(ROWS == 2 ? NTHREADS : 2 * NTHREADS,
                                  (sizeof(E) == 4 && ROWS == 2) ? 2 : 1)
qpair_kernel(const __grid_constant__ QStageArgs a) {
    static_assert((ROWS == 1) == (sizeof(E) == 8), "FP64 walks single rows, FP32 row pairs");
    // a lane value: two rows (columns) as a pair, or one
    typedef typename std::conditional<ROWS == 2, typename PairOf<E>::P, E>::type P;
    // WENO5 faces with the sliding walker, or minmod / PPM / piecewise-constant faces
    using Walker = typename std::conditional<
        RECON == BOLT_RECON_MINMOD, MinmodPairWalkerT<E, P>,
        typename std::conditional<
            RECON == BOLT_RECON_PPM, PpmPairWalkerT<E, P>,
            typename std::conditional<RECON == BOLT_RECON_PC, ConstPairWalkerT<E, P>,
                                      Weno5PairWalkerT<E, P>>::type>::type>::type;
    typedef Weno5PairT<E, P> Side;
    typedef typename PairOf<E>::P TabP;               // table entries: row pairs
    constexpr int NT = ROWS == 2 ? NTHREADS : 2 * NTHREADS;
    constexpr int CS = PairStage<E>::CS, VE = PairStage<E>::VE;
    constexpr bool F64 = sizeof(E) == 8;
    constexpr bool BX = MODE == QP_X1 || MODE == QP_X2 || MODE == QP_K;   // no base tiles
    constexpr bool KOUT = MODE == QP_K;
    constexpr bool HAS2 = MODE == QP_X2 || MODE == QP_B1R2;
    constexpr bool RED2 = MODE == QP_B1R2;
    constexpr int TQ = 8, HX = TQ + 2 * HALO, NQ = TQ * TQ, NWARP = NT / 32;
    constexpr int XT = HX * HX * PW;                 // elements of one halo tile
    constexpr int TE = TQ * TQ * PW;                 // elements of one 8x8 tile
    constexpr int NQUART = NTHREADS / NQ;            // phase C: threads per q-cell
    static_assert(NWARP == 8 * (3 - ROWS) && NQUART == 4, "8 walkers per direction");

    const int Np1 = a.Np1, Np2 = a.Np2, Np = a.Np, Ng = a.Ng;
    const int Nq1 = a.Nq1, Nq2 = a.Nq2;
    const int ntab = Np1 + Np2 + a.Np3;
    const PLayout Lo = qpair_layout(ntab, BGK, sizeof(E));
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* sm = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    E* X = reinterpret_cast<E*>(sm + Lo.x);
    E* o1s = reinterpret_cast<E*>(sm + Lo.o1);
    E* o2s = reinterpret_cast<E*>(sm + Lo.o2);
    E* b1s = reinterpret_cast<E*>(sm + Lo.b1);
    E* d1s = reinterpret_cast<E*>(sm + Lo.d1);
    TabP* tabs = reinterpret_cast<TabP*>(sm + Lo.tabs);
    double* vgrid = reinterpret_cast<double*>(sm + Lo.vgrid);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + Lo.bars);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int tile1, tile2;
    qpair_tile(a, (int)blockIdx.x, tile1, tile2);
    const int s = blockIdx.y / a.nsplit, split = blockIdx.y % a.nsplit;
    const int i0 = tile1 * TQ, j0 = tile2 * TQ;
    const int k_begin = split * a.chunks_per_split;
    const int k_end = min(Np / PW, k_begin + a.chunks_per_split);
    const int xs = s * Np;                           // TMA x coordinate of the species
    const bool peer2 = a.peer_lo != nullptr;          // q2 images go to the neighbours
    const bool peer1 = a.peer_left != nullptr;        // q1 images go to the neighbours
    const bool border = ((a.periodic1 || peer1) && (i0 < Ng || i0 + TQ > Nq1 - Ng)) ||
                        ((a.periodic2 || peer2) && (j0 < Ng || j0 + TQ > Nq2 - Ng));

    if (tid == 0) {
        prefetch_tmap(&a.tmap);
        prefetch_tmap(&a.tm_b1);
        prefetch_tmap(&a.tm_o1);
        prefetch_tmap(&a.tm_o2);
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], 1);
        mbar_init(&bars[3], 1);
        fence_barrier_init();
    }

    bool failed = false;
    unsigned pend = 0u;        // thread 0: barriers with a load in flight
    auto load_x = [&](int k, int b) {
        if (k < k_end && !a.stall_test) {       // test hook: no copy, the wait runs out
            pend |= 1u << b;
            mbar_arrive_expect_tx(&bars[b], XT * sizeof(E));
            tma_load_3d(X + b * XT, &a.tmap, &bars[b], xs + k * PW, i0 + Ng - HALO,
                        j0 + Ng - HALO);
        }
    };
    auto load_b = [&](int k, int b) {          // base1 tile of chunk k -> buffer b
        if (!BX && k < k_end && !a.stall_test) {
            pend |= 4u << b;
            mbar_arrive_expect_tx(&bars[2 + b], TE * sizeof(E));
            tma_load_3d(b1s + b * TE, &a.tm_b1, &bars[2 + b], xs + k * PW, i0 + Ng, j0 + Ng);
        }
    };
    // the first tiles load while the tables are built: thread 0 initialised
    // the barriers itself, the other threads reach them after the prologue
    if (tid == 0) {
        load_x(k_begin, 0);
        load_x(k_begin + 1, 1);
        load_b(k_begin, 0);
        load_b(k_begin + 1, 1);
    }
    // p3 rows of this CTA's p-range (the tables hold only those)
    const int p3lo = (k_begin * PW) / (Np1 * Np2);
    const int n3 = k_begin < k_end ? (k_end * PW - 1) / (Np1 * Np2) - p3lo + 1 : 0;
    qpair_prologue<E, BGK, NT>(a, s, i0, j0, vgrid, reinterpret_cast<double*>(d1s), tabs, p3lo,
                               n3);

    E* __restrict__ out1 = static_cast<E*>(a.out1);
    const P c1 = LaneOf<P>::splat(E(a.c1)), c2 = LaneOf<P>::splat(E(a.c2));
    const E inv_dq1 = E(1.0 / a.dq1), inv_dq2 = E(1.0 / a.dq2);
    const P inv_tau = LaneOf<P>::splat(E(1.0 / a.tau));
    const bool want_mom = a.mom_out != nullptr;
    const bool check = a.flag != nullptr;
    const unsigned rowstride = (unsigned)(a.Ns * Np);
    const unsigned colstride = rowstride * (unsigned)a.Nq1g;
    bool nonfinite = false;

    // phase A / B lane: p = k*32 + lane
    int ip1, ip2, ip3;
    {
        const int p = k_begin * PW + lane;
        ip1 = p % Np1; ip2 = (p / Np1) % Np2; ip3 = p / (Np1 * Np2);
    }
    // phase C (all warps of the pair form, the q2 walkers of the single-row
    // form): q-cell pc_c = (row warp%8, col lane%8), p = k*32 + 8*pc_q .. +7
    // with pc_q = lane/8: the group holds the lane's own p and lies in one p1
    // row (N_p1 % 8 == 0), so its velocities follow from the lane's
    const int pc_w = ROWS == 2 ? warp : (warp & 7);
    const int pc_c = pc_w * TQ + (lane & 7), pc_q = lane >> 3;
    const double dp1 = a.sg.dp1[s];
    const double t_own = double(lane & 7);
    double macc[kNumMom] = {0, 0, 0, 0, 0};

    // pairs: q1 walkers (warps 0-3) rows 2w, 2w+1, q2 walkers (warps 4-7)
    // columns 2(w-4), 2(w-4)+1; single rows: q1 walkers (warps 0-7) row w, q2
    // walkers (warps 8-15) column w-8; each walks the 8 cells of its line
    const bool q1w = warp < NWARP / 2;
    const bool pc_on = ROWS == 2 || !q1w;             // this warp runs phase C
    const int lp = ROWS == 2 ? 2 * (warp & 3) : (warp & 7);   // first row / column
    const int sw0 = stg<E>(lp, lane) - lp * CS;       // swizzled lane slot, column lp
    const int sw1 = stg<E>(lp + 1, lane) - (lp + 1) * CS;
    // a lane value from element p (and p + off, the pair's second line), and back
    auto ld = [](const E* p, int off) -> P {
        if constexpr (ROWS == 2) return mk2(p[0], p[off]);
        else return p[0];
    };
    auto st = [](E* p, int off, P v) {
        if constexpr (ROWS == 2) { p[0] = v.x; p[off] = v.y; }
        else p[0] = v;
    };
    // phase C source: 8 p from 16-byte chunk c_ch0 of q-cell pc_c's staging row
    const E* c_row = o1s + (8 * pc_q / CS) * 64 * CS + pc_c * CS;
    const int c_ch0 = (8 * pc_q % CS) / VE, c_key = pc_c & 7;
    // table entries of row lp (its pair, or its component of the pair), TW
    // lane values per table pair
    constexpr int TW = 3 - ROWS;
    const P* tb_row = reinterpret_cast<const P*>(reinterpret_cast<const E*>(tabs) +
                                                 2 * (lp >> 1) * TQ + (ROWS == 2 ? 0 : (lp & 1)));

    // periodic ghost images (border CTAs): offsets of column `warp` of the
    // tile, the q1 image shift g_d1, and the rows [0, g_bot) with a q2 image
    // at +N_q2 and [g_top, TQ) with one at -N_q2 (element offsets)
    // (pairs: every warp; single rows: the q1 walkers)
    int g_src = 0, g_dst = 0, g_d1 = 0, g_d2 = 0, g_bot = 0, g_top = TQ;
    const bool g_on = border && (ROWS == 2 || q1w);
    if (g_on) {
        const int ii = i0 + pc_w;
        g_src = stg<E>(pc_w, lane);                        // row r adds r*TQ*CS
        g_dst = (j0 + Ng) * (int)colstride + (ii + Ng) * (int)rowstride + xs + lane;
        if (a.periodic1 || peer1)
            g_d1 = ii < Ng ? Nq1 * (int)rowstride : (ii >= Nq1 - Ng ? -Nq1 * (int)rowstride : 0);
        if (a.periodic2 || peer2) {
            g_d2 = Nq2 * (int)colstride;
            g_bot = max(0, min(TQ, Ng - j0));
            g_top = min(TQ, max(0, Nq2 - Ng - j0));
        }
    }

    unsigned phx0 = 0u, phx1 = 0u, phb0 = 0u, phb1 = 0u;
    int buf = 0;
    for (int k = k_begin; k < k_end; ++k, buf ^= 1) {
        // every thread waits for the halo tile itself; a failed wait (here or
        // for the base tile) leaves the chunk's shared-memory results unused
        // and reaches every thread at the CTA barrier that ends the chunk
        if (!failed && !mbar_wait_bounded(&bars[buf], buf ? phx1 : phx0, a.wait_cycles))
            failed = true;
        const E* Xb = X + buf * XT;
        const double V1 = vgrid[ip1], V2 = vgrid[Np1 + ip2];

        if (q1w) {
            // ---- q1 faces of rows lp, lp+1, BGK -> D1 --------------------------
            // D1 of the previous chunk was last read before its closing barrier
            const E v1 = E(V1);
            const bool right = v1 > E(0);
            Side S; S.set(right);
            const E* ra = Xb + ((lp + HALO) * HX + (right ? 0 : 1)) * PW + lane;
            constexpr int rb = HX * PW;                // the pair's second row
            P y0 = ld(ra + 0 * PW, rb);
            P y1 = ld(ra + 1 * PW, rb);
            P y2 = ld(ra + 2 * PW, rb);
            P y3 = ld(ra + 3 * PW, rb);
            P y4 = ld(ra + 4 * PW, rb);
            Walker W;
            const P vq = LaneOf<P>::splat(E(0.5) * v1 * inv_dq1);   // walker: 2x face value
            P Fprev = W.first(y0, y1, y2, y3, y4, S);
            E* da = d1s + lp * TQ * PW + lane;
            const P* t1 = tb_row + ip1 * kTabPitch * TW;
            const P* t2 = tb_row + (Np1 + ip2) * kTabPitch * TW;
            const P* t3 = tb_row + (Np1 + Np2 + ip3 - p3lo) * kTabPitch * TW;
#pragma unroll
            for (int c = 0; c < TQ; ++c) {
                y0 = y1; y1 = y2; y2 = y3; y3 = y4;
                y4 = ld(ra + (c + 5) * PW, rb);
                const P Fn = W.next(y0, y1, y2, y3, y4, S);
                P d = mul2(sub2(Fprev, Fn), vq);
                Fprev = Fn;
                if (BGK) {
                    // the cell itself is the window's y2 (right-moving) or y1
                    const P fcell = right ? y2 : y1;
                    const P f0 = mul2(mul2(t1[c * TW], t2[c * TW]), t3[c * TW]);
                    d = fma2(sub2(f0, fcell), inv_tau, d);
                }
                st(da + c * PW, TQ * PW, d);
            }
            // the store of chunk k-1 must be done reading the staging tiles
            // before the q2 walkers write them
            if (warp == 0) bulk_wait_read_all();
            named_bar_arrive(1, NT);
        } else {
            // ---- q2 faces of columns lp, lp+1, then combine with D1 ---------------
            const E v2 = E(V2);
            const bool right = v2 > E(0);
            Side S; S.set(right);
            const E* ca = Xb + ((right ? 0 : 1) * HX + lp + HALO) * PW + lane;
            constexpr int cb = PW;                     // the pair's second column
            P y0 = ld(ca + 0 * HX * PW, cb);
            P y1 = ld(ca + 1 * HX * PW, cb);
            P y2 = ld(ca + 2 * HX * PW, cb);
            P y3 = ld(ca + 3 * HX * PW, cb);
            P y4 = ld(ca + 4 * HX * PW, cb);
            Walker W;
            P Fprev = W.first(y0, y1, y2, y3, y4, S);
            P dq[TQ];                                  // flux differences of rows 0..7
#pragma unroll
            for (int r = 0; r < TQ; ++r) {
                y0 = y1; y1 = y2; y2 = y3; y3 = y4;
                y4 = ld(ca + (r + 5) * HX * PW, cb);
                const P Fn = W.next(y0, y1, y2, y3, y4, S);
                dq[r] = sub2(Fprev, Fn);
                Fprev = Fn;
            }
            if (!BX && !failed &&
                !mbar_wait_bounded(&bars[2 + buf], buf ? phb1 : phb0, a.wait_cycles))
                failed = true;
            named_bar_sync(1, NT);                    // D1 written, staging tiles free
            const P vq = LaneOf<P>::splat(E(0.5) * v2 * inv_dq2);
            const E* dk = d1s + lp * PW + lane;
            const E* bb1 = b1s + buf * TE + lp * PW + lane;
            const E* cella = Xb + (HALO * HX + lp + HALO) * PW + lane;
            E* ob1 = o1s + lp * CS;
            E* ob2 = o2s + lp * PW + lane;
            // FP64 accumulator: element (row r, column lp, p) of chunk k
            E* accp = static_cast<E*>(a.out2) + ((j0 + Ng) * colstride +
                                                 (i0 + lp + Ng) * rowstride + xs + k * PW + lane);
#pragma unroll
            for (int r = 0; r < TQ; ++r) {
                const P kq = ld(dk + r * TQ * PW, PW);
                const P kk = fma2(dq[r], vq, kq);
                const P fcell = BX ? ld(cella + r * HX * PW, PW) : kk;
                const P o1 = KOUT ? kk : fma2(kk, c1, BX ? fcell : ld(bb1 + r * TQ * PW, PW));
                if constexpr (ROWS == 2) {
                    ob1[r * TQ * CS + sw0] = o1.x;
                    ob1[r * TQ * CS + CS + sw1] = o1.y;
                } else {
                    ob1[r * TQ * CS + sw0] = o1;
                }
                if constexpr (RED2 && F64) {
                    // the increment c2 k straight into the accumulator: one
                    // add per element and stage, so acc + inc exactly
                    atomicAdd(accp + r * colstride, mul2(kk, c2));
                } else if (HAS2) {
                    // QP_X2: the full out2; QP_B1R2: the increment c2 k
                    const P o2 = RED2 ? mul2(kk, c2) : fma2(kk, c2, fcell);
                    st(ob2 + r * TQ * PW, PW, o2);
                }
            }
        }
        fence_proxy_async();       // staging writes -> visible to the bulk-copy proxy
        failed = __syncthreads_or(failed);                        // closes the chunk
        if (failed) break;
        if (buf) { phx1 ^= 1u; phb1 ^= 1u; } else { phx0 ^= 1u; phb0 ^= 1u; }
        pend &= ~(5u << buf);
        if (tid == 0) {
            tma_store_3d(&a.tm_o1, o1s, xs + k * PW, i0 + Ng, j0 + Ng);
            if (F64)        // second half of the 32 p (the swizzled rows hold 16)
                tma_store_3d(&a.tm_o1, o1s + 64 * CS, xs + k * PW + CS, i0 + Ng, j0 + Ng);
            if (MODE == QP_X2) tma_store_3d(&a.tm_o2, o2s, xs + k * PW, i0 + Ng, j0 + Ng);
            if (RED2 && !F64) tma_reduce_add_3d(&a.tm_o2, o2s, xs + k * PW, i0 + Ng, j0 + Ng);
            bulk_commit();
            load_x(k + 2, buf);
            load_b(k + 2, buf);
        }

        // ---- periodic ghost images of border cells, from the staged out1 -------
        // warp w owns tile column w%8; images along q1 (whole column), along q2
        // (rows below g_bot and from g_top) and at the corners (2 N_g <= N_q)
        if (g_on) {
            const E* src = o1s + g_src;
            E* dst = out1 + (g_dst + k * PW);
            // q1 / q2 images: this buffer (periodic axis) or the neighbours'
            // copies (a cut axis; then no corner cell is needed)
            E* dlo = peer2 ? static_cast<E*>(a.peer_lo) + (g_dst + k * PW) : dst;
            E* dhi = peer2 ? static_cast<E*>(a.peer_hi) + (g_dst + k * PW) : dst;
            const int gc1 = (peer1 || peer2) ? 0 : g_d1;
            if (g_d1) {
                E* d1 = peer1 ? static_cast<E*>(g_d1 > 0 ? a.peer_left : a.peer_right) +
                                    (g_dst + k * PW)
                              : dst;
#pragma unroll
                for (int r = 0; r < TQ; ++r)
                    d1[r * (int)colstride + g_d1] = src[r * TQ * CS];
            }
            for (int r = 0; r < g_bot; ++r) {
                const E v = src[r * TQ * CS];
                dlo[r * (int)colstride + g_d2] = v;
                if (gc1) dst[r * (int)colstride + gc1 + g_d2] = v;
            }
            for (int r = g_top; r < TQ; ++r) {
                const E v = src[r * TQ * CS];
                dhi[r * (int)colstride - g_d2] = v;
                if (gc1) dst[r * (int)colstride + gc1 - g_d2] = v;
            }
        }

        // ---- phase C: FP64 moments of out1, divergence check ------------------
        // 8 consecutive p of one p1 row: v1 = V1_0 + t dp1 (t = 0..7), v2, v3
        // fixed, so every moment follows from S0 = sum o_t, S1 = sum t o_t and
        // S2 = sum t^2 o_t (moments.py:6-24 / compute_moments.py:7-59)
        if ((want_mom || check) && pc_on) {
            double ov[8];
            load8(c_row, c_ch0, c_key, ov);
            const double o0 = ov[0], o1 = ov[1], o2 = ov[2], o3 = ov[3];
            const double o4 = ov[4], o5 = ov[5], o6 = ov[6], o7 = ov[7];
            const double S0 = ((o0 + o1) + (o2 + o3)) + ((o4 + o5) + (o6 + o7));
            const double S1 = fma(7.0, o7, fma(6.0, o6, fma(5.0, o5, fma(4.0, o4,
                              fma(3.0, o3, fma(2.0, o2, o1))))));
            const double S2 = fma(49.0, o7, fma(36.0, o6, fma(25.0, o5, fma(16.0, o4,
                              fma(9.0, o3, fma(4.0, o2, o1))))));
            nonfinite |= !isfinite(S0);
            const double W1 = fma(-t_own, dp1, V1), W2 = V2, W3 = vgrid[Np1 + Np2 + ip3];
            macc[0] += S0;
            macc[1] = fma(W1, S0, fma(dp1, S1, macc[1]));
            macc[2] = fma(W2, S0, macc[2]);
            macc[3] = fma(W3, S0, macc[3]);
            // 0.5 sum o_t (v1_t^2 + v2^2 + v3^2)
            const double e0 = fma(W1, W1, fma(W2, W2, W3 * W3));
            const double q = fma(e0, S0, fma(2.0 * W1 * dp1, S1, (dp1 * dp1) * S2));
            macc[4] = fma(0.5, q, macc[4]);
        }
        ip1 += PW;
        while (ip1 >= Np1) {
            ip1 -= Np1;
            if (++ip2 == Np2) { ip2 = 0; ++ip3; }
        }
    }
    if (failed) {
        // a barrier wait ran out: record it, then let the copies still in
        // flight land (bounded) before the CTA releases its shared memory
        if (warp == 0) bulk_wait_all();
        if (tid == 0) {
            atomicExch(a.err, 4);
            if (pend & 1u) mbar_wait_bounded(&bars[0], phx0);
            if (pend & 2u) mbar_wait_bounded(&bars[1], phx1);
            if (pend & 4u) mbar_wait_bounded(&bars[2], phb0);
            if (pend & 8u) mbar_wait_bounded(&bars[3], phb1);
        }
        return;
    }
    if (warp == 0) bulk_wait_all();
    // one flag write per CTA (the flag may live in host memory)
    if (__syncthreads_or(check && nonfinite) && tid == 0) atomicOr(a.flag, 1);

    const long long plane = (long long)Nq2 * Nq1;
    if (want_mom) {
        double* red = reinterpret_cast<double*>(sm + Lo.x);
        if (pc_on) {
#pragma unroll
            for (int q = 0; q < kNumMom; ++q) red[(pc_q * NQ + pc_c) * kNumMom + q] = macc[q];
        }
        __syncthreads();
        for (int c = tid; c < NQ * kNumMom; c += NT) {
            const int cq = c / kNumMom, q = c % kNumMom;
            double v = 0.0;
#pragma unroll
            for (int h = 0; h < NQUART; ++h) v += red[(h * NQ + cq) * kNumMom + q];
            const int ii = i0 + (cq & 7), jj = j0 + (cq >> 3);
            a.mom_out[(((long long)split * kNumMom + q) * a.Ns + s) * plane
                      + (long long)jj * Nq1 + ii] = v;
        }
    }
}

template <typename E, int R, int W>
static void (*pick_qpair(int bgk, int mode))(QStageArgs) {
    switch (mode) {
        case QP_X1:
            return bgk ? qpair_kernel<E, true, QP_X1, R, W> : qpair_kernel<E, false, QP_X1, R, W>;
        case QP_X2:
            return bgk ? qpair_kernel<E, true, QP_X2, R, W> : qpair_kernel<E, false, QP_X2, R, W>;
        case QP_B1:
            return bgk ? qpair_kernel<E, true, QP_B1, R, W> : qpair_kernel<E, false, QP_B1, R, W>;
        case QP_K:
            return bgk ? qpair_kernel<E, true, QP_K, R, W> : qpair_kernel<E, false, QP_K, R, W>;
        default:
            return bgk ? qpair_kernel<E, true, QP_B1R2, R, W>
                       : qpair_kernel<E, false, QP_B1R2, R, W>;
    }
}

// the stage mode from which buffers the stage reads and writes, then the
// reconstruction's instantiation
template <typename E>
static cudaError_t launch_qpair(const QStageArgs& a, int bgk, int recon, dim3 grid, size_t smem,
                                cudaStream_t st) {
    const bool has2 = a.out2 != nullptr;
    // first RK4 / RK2 stage: the bases are the stage input
    const bool bx = a.base1 == a.fs && (!has2 || a.base2 == a.fs);
    int mode;
    if (a.base1 == nullptr && !has2) mode = QP_K;
    else if (bx) mode = has2 ? QP_X2 : QP_X1;
    else if (!has2) mode = QP_B1;
    else if (a.base2 == a.out2) mode = QP_B1R2;
    else return cudaErrorInvalidValue;        // excluded by the host's dispatch
    // FP32: row pairs, 8 warps, 2 CTAs per SM; FP64: one row per thread, 16
    // warps, 1 CTA per SM (the shared memory of the double-buffered tiles)
    constexpr int W = sizeof(E) == 4 ? 2 : 1;
    void (*k)(QStageArgs);
    switch (recon) {
        case BOLT_RECON_MINMOD: k = pick_qpair<E, BOLT_RECON_MINMOD, W>(bgk, mode); break;
        case BOLT_RECON_PPM: k = pick_qpair<E, BOLT_RECON_PPM, W>(bgk, mode); break;
        case BOLT_RECON_PC: k = pick_qpair<E, BOLT_RECON_PC, W>(bgk, mode); break;
        default: k = pick_qpair<E, BOLT_RECON_WENO5, W>(bgk, mode); break;
    }
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, W == 2 ? NTHREADS : 2 * NTHREADS, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace bolt
