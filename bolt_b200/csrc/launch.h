// launch.h - host-side launchers of the FVM kernels, one set per dtype.
// Implemented in kernels_f64.cu (FP64, reference operation order, no FMA
// contraction) and kernels_f32.cu (FP32 fast path).
#pragma once

#include <cuda_runtime.h>

#include "fvm_args.h"

namespace bolt {

enum Tiling { TILING_2D = 0, TILING_1D = 1, TILING_1D_Q2 = 2 };

struct TileShape {
    int tq1, tq2, q2;
};

inline TileShape tile_shape(int tiling) {
    switch (tiling) {
        case TILING_2D: return {8, 8, 1};
        case TILING_1D: return {64, 1, 0};
        default: return {64, 1, 1};
    }
}

// bytes of dynamic shared memory of the q-stage kernel
inline size_t qstage_smem(int tiling, size_t elem, int bgk, int bgk_direct, int ntab) {
    TileShape t = tile_shape(tiling);
    return qstage_layout(t.tq1, t.tq2, t.q2, (int)elem, bgk, bgk_direct, ntab).total;
}

// bytes of dynamic shared memory of the paired kernel (elem: 4 FP32, 8 FP64)
inline size_t qpair_smem(int ntab, int bgk, size_t elem) {
    return qpair_layout(ntab, bgk, (unsigned)elem).total;
}

// p-split of the q-stage grid (q-tiles x species x splits): the split that
// minimises (waves, rounded up) x (chunks per CTA + ~2 chunks of prologue), a
// wave being the GPU's SMs x the stage kernel's resident CTAs per SM (from its
// shared memory, at most 2).  Shared by the context and the allocation-free
// entry point.
struct PSplit {
    int nsplit, chunks_per_split;
};

inline PSplit choose_psplit(int nchunks, long long base_ctas, int sms, size_t smem_per_cta) {
    long long per_sm = 233472LL / (long long)(smem_per_cta + 1024);
    per_sm = per_sm < 1 ? 1 : (per_sm > 2 ? 2 : per_sm);
    const long long wave = (long long)(sms > 0 ? sms : 1) * per_sm;
    double best = 1e300;
    int best_cps = nchunks;
    for (int n = 1; n <= nchunks && n <= 64; ++n) {
        const int cps = (nchunks + n - 1) / n;
        const int ne = (nchunks + cps - 1) / cps;
        const long long waves = (base_ctas * ne + wave - 1) / wave;
        const double cost = (double)waves * (cps + 2.0);
        if (cost < best - 1e-9) {
            best = cost;
            best_cps = cps;
        }
    }
    return PSplit{(nchunks + best_cps - 1) / best_cps, best_cps};
}

// SM count of the current device (148 on B200 if the query fails)
inline int current_sm_count() {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// the f, flux and two divergence arrays, then the p-cell centres (doubles)
inline size_t pstage_smem(int Np, size_t elem, int ntab) {
    return ((4 * (size_t)Np * elem + 7) & ~(size_t)7) + (size_t)ntab * sizeof(double);
}

#define BOLT_DECLARE_LAUNCHERS(SUFFIX, T)                                                   \
    cudaError_t launch_qstage_##SUFFIX(const QStageArgs& a, int recon, int tiling, int bgk, \
                                       dim3 grid, size_t smem, cudaStream_t st);            \
    cudaError_t launch_pstage_##SUFFIX(const PStageArgs& a, int recon, dim3 grid,           \
                                       size_t smem, cudaStream_t st);                       \
    cudaError_t launch_moment_##SUFFIX(const void* f, int mid, double* out, int Ns,          \
                                       int Np1, int Np2, int Np3, int Nq1g, int Nq2g,        \
                                       const SpeciesGrid& sg, cudaStream_t st);             \
    cudaError_t launch_moments5_##SUFFIX(const void* f, double* part, int Ns, int Np1,       \
                                         int Np2, int Np3, int Nq1, int Nq2, int Ng,         \
                                         const SpeciesGrid& sg, cudaStream_t st);           \
    cudaError_t launch_ghost_##SUFFIX(void* f, const void* dl, const void* dr,               \
                                      const void* db, const void* dt, int Nq1, int Nq2,      \
                                      int Ng, int Ns, int Np, int Np1, int Np2, int per1,    \
                                      int per2, int dir1, int dir2, int mir1, int mir2,      \
                                      int ext1, int ext2, const SpeciesGrid& sg,             \
                                      const GhostShear& sh, cudaStream_t st);

// electrostatic field solve of one df/dt argument (poisson.cu)
struct PoissonArgs {
    const double* part;       // density partial sums [Ns][Nq2][Nq1] (moments5 split 0)
    double2* rho_hat;         // Nq2 x Nq1 complex work
    double2* e_hat;           // 2 x Nq2 x Nq1 complex work (E1, E2)
    double* cell;             // (6, Nq2g, Nq1g) cell-centred fields; E1, E2 written
    int Nq1, Nq2, Ng, Ns;
    double dq1, dq2, eps;
    double charge[kMaxSpecies], measure[kMaxSpecies];
    double mom_scale;         // the moments' factor: initial_mu on polar2D, else 1
};
int poisson_plans_create(int Nq1, int Nq2, int* fwd, int* inv);
void poisson_plans_destroy(int fwd, int inv);
cudaError_t launch_poisson(const PoissonArgs& a, int fwd, int inv, cudaStream_t st,
                           long long* launches);

BOLT_DECLARE_LAUNCHERS(f64, double)
BOLT_DECLARE_LAUNCHERS(f32, float)

// advective semi-Lagrangian step in q (asl_kernels.cuh): the interpolation of
// the interior at the feet of the characteristics, and the BGK source
cudaError_t launch_asl_q_f64(const AslArgs& a, int* flag, cudaStream_t st);
cudaError_t launch_asl_q_f32(const AslArgs& a, int* flag, cudaStream_t st);
cudaError_t launch_asl_src_f64(const QStageArgs& a, const void* in, const void* base, void* out,
                               double c, int mode, int* flag, double* mom_out, cudaStream_t st);
cudaError_t launch_asl_src_f32(const QStageArgs& a, const void* in, const void* base, void* out,
                               double c, int mode, int* flag, double* mom_out, cudaStream_t st);

// paired q-stage (8x8 tiling, fused combine, TMA in and out): FP32, and FP64
// with FMA contraction and Newton-refined reciprocals (BOLT_F64_FAST)
cudaError_t launch_qpair_f32(const QStageArgs& a, int bgk, int recon, dim3 grid, size_t smem,
                             cudaStream_t st);
cudaError_t launch_qpair_f64(const QStageArgs& a, int bgk, int recon, dim3 grid, size_t smem,
                             cudaStream_t st);

// FDTD sequence (FP64): prepare -> halo -> E -> halo -> B -> to_cell
cudaError_t launch_fdtd(const FieldArgs& a, cudaStream_t st, long long* launches);
cudaError_t launch_fdtd_part(const FieldArgs& a, int part, cudaStream_t st, long long* launches);
cudaError_t launch_field_halo(const FieldArgs& a, cudaStream_t st);

}  // namespace bolt
