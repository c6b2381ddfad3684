// fvm_args.h - constants and kernel argument blocks shared by host and device.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace bolt {

constexpr int kMaxSpecies = 8;
constexpr int PW = 32;          // p-cells per chunk (one per lane)
constexpr int HALO = 3;         // q-stencil half width incl. face shift
constexpr int NTHREADS = 256;   // q-stage CTA size (8 warps)
constexpr int kNumMom = 5;      // n, mom_v1, mom_v2, mom_v3, energy
constexpr int PWP = PW + 1;     // padded stage-buffer row (conflict-free column reads)
// default budget of a bounded mbarrier wait, in SM clock cycles (~2 s at the
// boost clock); after it the wait reports failure and the kernel records
// BOLT_ERR_TIMEOUT in its error word instead of hanging
constexpr long long kDefaultWaitCycles = 4000000000LL;

// Shared-memory carve-up of the q-stage kernel (byte offsets), used by the
// kernel and by the host to size the launch.
struct QLayout {
    unsigned tile, stage, vtab, jacc, qc, tabs, vgrid, bars, total;
    int nbuf;               // halo tiles in flight (2: double-buffered)
};

// dynamic shared memory per CTA that still lets two CTAs share an SM
// (228 KB per SM, 1 KB reserved per CTA)
constexpr unsigned kTwoCtaSmem = 113u * 1024u;

__host__ __device__ inline unsigned qalign(unsigned x, unsigned a) { return (x + a - 1) / a * a; }

__host__ __device__ inline QLayout qstage_layout_n(int tq1, int tq2, int q2, int elem, int bgk,
                                                   int bgk_direct, int ntab, int nbuf) {
    QLayout L;
    L.nbuf = nbuf;
    const unsigned hx = tq1 + 2 * HALO, hy = q2 ? tq2 + 2 * HALO : 1;
    const unsigned nq = tq1 * tq2;
    unsigned o = 0;
    L.tile = o;  o += qalign((unsigned)nbuf * hy * hx * PW * elem, 128);
    // the epilogue reuses the tile region for the cross-thread moment reduction
    const unsigned red = (unsigned)(NTHREADS * kNumMom * sizeof(double));
    if (o < red) o = qalign(red, 128);
    L.stage = o; o += qalign(nq * PWP * elem, 16);
    L.vtab = o;  o += 4 * PW * sizeof(double);
    L.jacc = o;  o += nq * 3 * sizeof(double);
    L.qc = o;    o += nq * 5 * sizeof(double);
    L.tabs = o;  o += (bgk && !bgk_direct) ? nq * ntab * sizeof(double) : 0;
    L.vgrid = o; o += ntab * sizeof(double);      // p1, p2, p3 cell centres of the species
    L.bars = o;  o += 2 * sizeof(unsigned long long);
    L.total = o;
    return L;
}

// Double-buffered halo tiles when two CTAs per SM still fit, else one (the
// FP64 8x8 tile with exp tables: 160 KB double-buffered, 110 KB single) --
// the co-resident CTA then hides the load that double-buffering would.
__host__ __device__ inline QLayout qstage_layout(int tq1, int tq2, int q2, int elem, int bgk,
                                                 int bgk_direct, int ntab) {
    const QLayout L2 = qstage_layout_n(tq1, tq2, q2, elem, bgk, bgk_direct, ntab, 2);
    if (L2.total <= kTwoCtaSmem) return L2;
    return qstage_layout_n(tq1, tq2, q2, elem, bgk, bgk_direct, ntab, 1);
}

// Shared-memory carve-up of the paired kernel (8x8 q-tile, FP32 or FP64
// elements of `elem` bytes), offsets from a 1024-byte aligned base (the
// 128-byte swizzled output tile needs it; the kernel aligns the dynamic base
// itself, hence the 1 KB of slack in total).  FP32: 111.8 KB (two CTAs per
// SM); FP64: 216.7 KB (one).
struct PLayout {
    unsigned x, o1, o2, b1, d1, tabs, vgrid, bars, total;
};

constexpr unsigned kPairTileElems = 8 * 8 * PW;                        // one 8x8 tile
constexpr unsigned kPairHaloElems = (8 + 2 * HALO) * (8 + 2 * HALO) * PW;  // 14x14 halo tile
constexpr unsigned kTabPitch = 33;       // exp-table row: 32 q-cell pairs + 1 pad

__host__ __device__ inline PLayout qpair_layout(int ntab, int bgk, unsigned elem) {
    PLayout L;
    unsigned o = 0;
    const unsigned tile = kPairTileElems * elem;
    L.x = o;  o += 2 * kPairHaloElems * elem;     // double-buffered halo tile
    o = qalign(o, 1024);
    L.o1 = o; o += tile;                          // out1 staging (128B swizzle)
    L.o2 = o; o += tile;                          // out2 staging
    L.b1 = o; o += 2 * tile;                      // base1 tile, double-buffered
    L.d1 = o; o += tile;                          // q1 part of df/dt (prologue: Maxwellian
                                                  // parameters of the 64 q-cells)
    L.tabs = o; o += bgk ? kTabPitch * ntab * 2 * elem : 0u;  // exp tables, a pair per q-cell pair
    L.vgrid = o; o += ntab * sizeof(double);
    L.bars = qalign(o, 8); o = L.bars + 4 * sizeof(unsigned long long);
    L.total = o + 1024;
    return L;
}

// Shearing-box ghost strips (boundaries.py:6-145): axis 1 (q1 strips,
// resampled along q2) or axis 2 (q2 strips, resampled along q1), with the
// shift already reduced modulo the resampled axis's length
struct GhostShear {
    int axis;                   // 0: none, 1: q1 strips, 2: q2 strips
    double shift;               // q omega L t mod L_other (>= 0 or < 0)
    double start, end, dq;      // the resampled axis: domain and spacing
};

struct SpeciesGrid {
    double p1_start[kMaxSpecies], p2_start[kMaxSpecies], p3_start[kMaxSpecies];
    double dp1[kMaxSpecies], dp2[kMaxSpecies], dp3[kMaxSpecies];
    double mass[kMaxSpecies], charge[kMaxSpecies];
    // p-space grid (params.p_space_grid): 0 cartesian; 1 polar2D, whose
    // moments carry the factor mom_scale = params.initial_mu
    // (compute_moments.py:48-53) and whose mirror edges map the angle p2
    // (boundaries.py:313-413)
    int polar2d;
    double mom_scale;
};

struct QStageArgs {
    CUtensorMap tmap;           // 3-D map over fs: (Ns*Np, Nq1g, Nq2g), box (32, TQ1+6, HY)
    const void* fs;             // stage input (stencil source), ghosted
    const void* base1;          // out1 = base1 + c1*k   (null: out1 = k)
    const void* base2;          // out2 = base2 + c2*k   (null: no out2)
    void* out1;
    void* out2;
    const void* tau_arr;        // f-shaped tau or null
    const double* mom_in;       // partial moments of fs [nsplit_in][5][Ns][Nq2][Nq1]
    double* mom_out;            // partial moments of out1 [nsplit][5][Ns][Nq2][Nq1] or null
    double* j_out;              // partial currents [nsplit][3][Ns][Nq2][Nq1] or null
    int* flag;                  // divergence flag (host-mapped) or null
    int* err;                   // sticky device error word
    double c1, c2, tau;
    double dq1, dq2, kB;
    int Nq1, Nq2, Ng, Ns, Np1, Np2, Np3, Np, Nq1g, Nq2g;
    int periodic1, periodic2;   // write wrap-around ghost copies of out1
    int nsplit_in, nsplit, chunks_per_split, ntiles1;
    int use_tma, p_dim, want_j;
    int bgk_direct;             // 1: exp per cell (no per-q-cell exp tables)
    int full_chunks;            // Np % 32 == 0: every p-chunk is complete
    // budget of the tile waits (cycles); stall_test != 0 (a test hook) issues
    // no tile copies, so the first wait runs out with nothing in flight
    long long wait_cycles;
    int stall_test;
    SpeciesGrid sg;
    // paired kernel only: 8x8x32 boxes over base1, out1 (128B swizzle), out2
    CUtensorMap tm_b1, tm_o1, tm_o2;
    // paired kernel only: which q-tiles the grid's columns cover -- all (0),
    // the tiles whose halo stays inside the block along its external axes
    // ext1 (q1) / ext2 (q2) (1), or the remaining ones (2); ntiles2 tile rows
    int tile_sel, ext1, ext2, ntiles2;
    // q2 slab neighbours' copies of out1 (or null): the bottom N_g interior
    // rows are also stored N_q2 rows higher in peer_lo (the lower neighbour's
    // top ghost rows), the top N_g rows N_q2 rows lower in peer_hi
    void* peer_lo;
    void* peer_hi;
    // q1 block neighbours' copies of out1 (or null): the left N_g interior
    // columns are also stored N_q1 columns further right in peer_left (the
    // left neighbour's right ghost columns), the right N_g columns N_q1
    // columns further left in peer_right
    void* peer_left;
    void* peer_right;
};

// semi-Lagrangian q-step (asl_kernels.cuh): interpolation of the interior
struct AslArgs {
    const void* f;       // ghosted input (Nq2g, Nq1g, Ns, Np)
    void* out;           // interior cells written, same layout
    double dt;
    double q1_start, q2_start, dq1, dq2;
    int Nq1, Nq2, Ng, Ns, Np1, Np2, Np3, Np;
    SpeciesGrid sg;
};

struct PStageArgs {
    const void* fs;        // stage input (ghosted)
    const void* kq;        // q-part of df/dt (ghosted layout, interior valid)
    const void* base1;
    const void* base2;
    void* out1;
    void* out2;
    const double* cell;    // cell-centred fields [6][Nq2g][Nq1g]
    double* mom_out;       // [1][5][Ns][Nq2][Nq1] or null
    int* flag;
    double c1, c2;
    int Nq1, Nq2, Ng, Ns, Np1, Np2, Np3, Np, Nq1g, Nq2g;
    int periodic1, periodic2;
    int term;              // 0: the stage combine; 1..3: out1 <- d_flux_pk_dpk alone
    SpeciesGrid sg;
};

constexpr int PTHREADS = 256;

struct FieldArgs {
    double* yee;            // [6][Nq2g][Nq1g]
    double* cell;           // [6][Nq2g][Nq1g]
    double* ebefore;        // [3][Nq2g][Nq1g]
    double* J;              // [3][Nq2g][Nq1g]
    const double* jpart;    // [nsplit][3][Ns][Nq2][Nq1]
    const double* j_given;  // [3][Nq2g][Nq1g] species-summed currents from the caller, or null
    int nsplit, Ns, Nq1, Nq2, Ng, Nq1g, Nq2g;
    int ext1, ext2;         // external axes: their ghosts come from the neighbouring blocks
    double dq1, dq2, dt, eps, mu;
    double charge[kMaxSpecies], measure[kMaxSpecies];
    double mom_scale;           // the moments' factor: initial_mu on polar2D, else 1
};

}  // namespace bolt
