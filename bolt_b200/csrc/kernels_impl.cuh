// kernels_impl.cuh - instantiation switchboard shared by kernels_f64.cu and
// kernels_f32.cu.  Define BOLT_T, BOLT_EXACT and BOLT_SUFFIX before including.
#pragma once

#include "launch.h"
#include "fvm_kernels.cuh"
#include "asl_kernels.cuh"

namespace bolt {

#define BOLT_CAT2(a, b) a##b
#define BOLT_CAT(a, b) BOLT_CAT2(a, b)

template <int RECON, int TQ1, int TQ2, bool Q2, bool BGK>
static cudaError_t qlaunch(const QStageArgs& a, dim3 grid, size_t smem, cudaStream_t st) {
    auto k = qstage_kernel<BOLT_T, BOLT_EXACT, RECON, TQ1, TQ2, Q2, BGK>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, NTHREADS, smem, st>>>(a);
    return cudaGetLastError();
}

template <int RECON>
static cudaError_t qdispatch(const QStageArgs& a, int tiling, int bgk, dim3 grid, size_t smem,
                             cudaStream_t st) {
    if (tiling == TILING_2D)
        return bgk ? qlaunch<RECON, 8, 8, true, true>(a, grid, smem, st)
                   : qlaunch<RECON, 8, 8, true, false>(a, grid, smem, st);
    if (tiling == TILING_1D)
        return bgk ? qlaunch<RECON, 64, 1, false, true>(a, grid, smem, st)
                   : qlaunch<RECON, 64, 1, false, false>(a, grid, smem, st);
    return bgk ? qlaunch<RECON, 64, 1, true, true>(a, grid, smem, st)
               : qlaunch<RECON, 64, 1, true, false>(a, grid, smem, st);
}

cudaError_t BOLT_CAT(launch_qstage_, BOLT_SUFFIX)(const QStageArgs& a, int recon, int tiling,
                                                  int bgk, dim3 grid, size_t smem,
                                                  cudaStream_t st) {
    switch (recon) {
        case BOLT_RECON_PC: return qdispatch<BOLT_RECON_PC>(a, tiling, bgk, grid, smem, st);
        case BOLT_RECON_MINMOD: return qdispatch<BOLT_RECON_MINMOD>(a, tiling, bgk, grid, smem, st);
        case BOLT_RECON_PPM: return qdispatch<BOLT_RECON_PPM>(a, tiling, bgk, grid, smem, st);
        default: return qdispatch<BOLT_RECON_WENO5>(a, tiling, bgk, grid, smem, st);
    }
}

template <int RECON>
static cudaError_t plaunch(const PStageArgs& a, dim3 grid, size_t smem, cudaStream_t st) {
    auto k = pstage_kernel<BOLT_T, BOLT_EXACT, RECON>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, PTHREADS, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t BOLT_CAT(launch_pstage_, BOLT_SUFFIX)(const PStageArgs& a, int recon, dim3 grid,
                                                  size_t smem, cudaStream_t st) {
    switch (recon) {
        case BOLT_RECON_PC: return plaunch<BOLT_RECON_PC>(a, grid, smem, st);
        case BOLT_RECON_MINMOD: return plaunch<BOLT_RECON_MINMOD>(a, grid, smem, st);
        case BOLT_RECON_PPM: return plaunch<BOLT_RECON_PPM>(a, grid, smem, st);
        default: return plaunch<BOLT_RECON_WENO5>(a, grid, smem, st);
    }
}

cudaError_t BOLT_CAT(launch_moment_, BOLT_SUFFIX)(const void* f, int mid, double* out, int Ns,
                                                  int Np1, int Np2, int Np3, int Nq1g, int Nq2g,
                                                  const SpeciesGrid& sg, cudaStream_t st) {
    dim3 grid(Nq1g * Nq2g, Ns);
    moment_kernel<BOLT_T><<<grid, 256, 0, st>>>(static_cast<const BOLT_T*>(f), mid, out, Ns, Np1,
                                                Np2, Np3, Nq1g, Nq2g, sg);
    return cudaGetLastError();
}

cudaError_t BOLT_CAT(launch_moments5_, BOLT_SUFFIX)(const void* f, double* part, int Ns, int Np1,
                                                    int Np2, int Np3, int Nq1, int Nq2, int Ng,
                                                    const SpeciesGrid& sg, cudaStream_t st) {
    dim3 grid(Nq1 * Nq2, Ns);
    moments5_kernel<BOLT_T><<<grid, 256, 0, st>>>(static_cast<const BOLT_T*>(f), part, Ns, Np1,
                                                  Np2, Np3, Nq1, Nq2, Ng, sg);
    return cudaGetLastError();
}

cudaError_t BOLT_CAT(launch_ghost_, BOLT_SUFFIX)(void* f, const void* dl, const void* dr,
                                                 const void* db, const void* dt, int Nq1, int Nq2,
                                                 int Ng, int Ns, int Np, int Np1, int Np2,
                                                 int per1, int per2, int dir1, int dir2,
                                                 int mir1, int mir2, int ext1, int ext2,
                                                 const SpeciesGrid& sg, const GhostShear& sh,
                                                 cudaStream_t st) {
    const long long Nq1g = Nq1 + 2 * Ng;
    const long long ncells = 2LL * Ng * Nq1g + 2LL * Ng * Nq2;
    if (ncells == 0) return cudaSuccess;
    // one CTA per ghost cell (grid-stride beyond 16 CTAs per SM), its threads
    // over the cell's (species, p) block
    const long long rowlen = (long long)Ns * Np;
    const long long blocks = ncells < 148 * 16 ? ncells : 148 * 16;
    const int threads = rowlen >= 2048 ? 256 : (rowlen >= 512 ? 128 : 64);
    ghost_kernel<BOLT_T><<<(unsigned)blocks, threads, 0, st>>>(
        static_cast<BOLT_T*>(f), static_cast<const BOLT_T*>(dl), static_cast<const BOLT_T*>(dr),
        static_cast<const BOLT_T*>(db), static_cast<const BOLT_T*>(dt), Nq1, Nq2, Ng, Ns, Np, Np1,
        Np2, per1, per2, dir1, dir2, mir1, mir2, ext1, ext2, sg, sh, ncells);
    return cudaGetLastError();
}

cudaError_t BOLT_CAT(launch_asl_q_, BOLT_SUFFIX)(const AslArgs& a, int* flag, cudaStream_t st) {
    constexpr int R = AslRows<BOLT_T>::R;
    const long long total = (long long)((a.Nq2 + R - 1) / R) * a.Ns * a.Np;   // threads
    if (total == 0) return cudaSuccess;
    // 32-bit element offsets when the ghosted array has fewer than 2^31 elements
    const long long elems = (long long)(a.Nq2 + 2 * a.Ng) * (a.Nq1 + 2 * a.Ng) * a.Ns * a.Np;
    if (elems < (1LL << 31))
        asl_q_kernel<BOLT_T, int><<<(unsigned)((total + 255) / 256), 256, 0, st>>>(a, flag);
    else
        asl_q_kernel<BOLT_T, long long><<<(unsigned)((total + 255) / 256), 256, 0, st>>>(a, flag);
    return cudaGetLastError();
}

cudaError_t BOLT_CAT(launch_asl_src_, BOLT_SUFFIX)(const QStageArgs& a, const void* in,
                                                   const void* base, void* out, double c,
                                                   int mode, int* flag, double* mom_out,
                                                   cudaStream_t st) {
    dim3 grid(a.Nq1 * a.Nq2, a.Ns);
    asl_src_kernel<BOLT_T><<<grid, 256, 0, st>>>(a, in, base, out, c, mode, flag, mom_out);
    return cudaGetLastError();
}

}  // namespace bolt
