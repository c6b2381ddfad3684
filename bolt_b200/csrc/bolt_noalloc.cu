// bolt_noalloc.cu - df/dt entry point that performs no device allocation.
//
// Some callers cannot allocate device memory at the point where they need a
// df/dt evaluation: code that runs inside a memory pool or allocator whose
// budget is fixed up front, code that must not synchronise the device (a
// cudaMalloc/cudaFree may), and embedders that own all device memory
// themselves.  bolt_dfdt_noalloc serves them: the caller passes f and the
// output buffer, and the only scratch the evaluation needs -- the FP64 velocity
// moment sums per q-cell that the BGK term reads, an error word and a
// non-finite flag -- lives in a fixed array in this library's device memory.
//
// Limits and behaviour (also stated in include/bolt_b200.h):
//   * the moment scratch holds BOLT_NOALLOC_MAX_QCELLS q-cells x species
//     (5 FP64 sums each, 2.5 MiB); larger grids are rejected with
//     BOLT_ERR_UNSUPPORTED before anything is launched;
//   * every GPU that loads the library holds this array until the process
//     exits;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.  The address is cached per device for the
//     life of the process and does not survive a cudaDeviceReset;
//   * all calls share the array, which keeps the last call's contents; the
//     moment sums are fully overwritten by each call and the error word and
//     flag are cleared at the start of each call, so calls that overlap on the
//     GPU (different streams, or different host threads) race and must not;
//   * bolt_noalloc_status reads (and clears) the error word and flag of the
//     last call, a bounded-wait timeout or a non-finite df/dt;
//   * fields must be disabled, tau is the constant params->tau, and the ghost
//     cells of f must be current.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/bolt_b200.h"
#include "launch.h"
#include "validate.h"

using namespace bolt;

namespace {

constexpr int kMaxDevices = 64;
constexpr size_t kMomDoubles = (size_t)kNumMom * BOLT_NOALLOC_MAX_QCELLS;

// moment sums [5][Ns][Nq2][Nq1], then the error word and the non-finite flag
static __device__ __align__(256) double g_noalloc_scratch[kMomDoubles + 32];

double* g_scratch_ptr[kMaxDevices];          // device address of g_noalloc_scratch
int g_scratch_rc[kMaxDevices];               // result of its lookup
std::once_flag g_scratch_once[kMaxDevices];  // one lookup per device

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn lookup_encode_fn() {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
        return reinterpret_cast<EncodeTiledFn>(p);
    return nullptr;
}

// looked up once per process, thread-safely (function-local static)
EncodeTiledFn encode_fn() {
    static const EncodeTiledFn fn = lookup_encode_fn();
    return fn;
}

int scratch_for_current_device(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return BOLT_ERR_CUDA;
    std::call_once(g_scratch_once[dev], [dev] {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            g_scratch_rc[dev] = BOLT_ERR_CUDA;
        } else {
            g_scratch_ptr[dev] = static_cast<double*>(p);
            g_scratch_rc[dev] = BOLT_OK;
        }
    });
    if (g_scratch_rc[dev]) return g_scratch_rc[dev];
    *out = g_scratch_ptr[dev];
    return BOLT_OK;
}

int* error_words(double* scratch) { return reinterpret_cast<int*>(scratch + kMomDoubles); }

}  // namespace

extern "C" int bolt_dfdt_noalloc(const BoltGrid* grid, const BoltParams* params,
                                 const void* f_dev, void* dfdt_dev, void* stream) {
    if (!grid || !params || !f_dev || !dfdt_dev) return BOLT_ERR_ARG;
    const BoltGrid& g = *grid;
    const BoltParams& p = *params;
    const int vrc = check_grid_params(g, p);
    if (vrc) return vrc;
    if (p.fields_enabled) return BOLT_ERR_UNSUPPORTED;
    if (p.source_enabled && !(p.tau > 0.0)) return BOLT_ERR_ARG;
    if ((long long)g.N_s * g.N_q1 * g.N_q2 > BOLT_NOALLOC_MAX_QCELLS) return BOLT_ERR_UNSUPPORTED;

    double* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    int* err = error_words(scratch);            // [0] error word, [1] non-finite flag
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(err, 0, 2 * sizeof(int), st) != cudaSuccess) return BOLT_ERR_CUDA;

    const int Np = g.N_p1 * g.N_p2 * g.N_p3;
    const int Nq1g = g.N_q1 + 2 * g.N_ghost, Nq2g = g.N_q2 + 2 * g.N_ghost;
    const size_t elem = p.dtype == BOLT_F32 ? 4 : 8;
    SpeciesGrid sg;
    memset(&sg, 0, sizeof(sg));
    for (int s = 0; s < g.N_s; ++s) {
        sg.p1_start[s] = g.p1_start[s]; sg.p2_start[s] = g.p2_start[s]; sg.p3_start[s] = g.p3_start[s];
        sg.dp1[s] = g.dp1[s]; sg.dp2[s] = g.dp2[s]; sg.dp3[s] = g.dp3[s];
        sg.mass[s] = p.mass[s]; sg.charge[s] = p.charge[s];
    }
    const int bgk = p.source_enabled ? 1 : 0;
    if (bgk) {
        cudaError_t e = elem == 8
            ? launch_moments5_f64(f_dev, scratch, g.N_s, g.N_p1, g.N_p2, g.N_p3, g.N_q1, g.N_q2,
                                  g.N_ghost, sg, st)
            : launch_moments5_f32(f_dev, scratch, g.N_s, g.N_p1, g.N_p2, g.N_p3, g.N_q1, g.N_q2,
                                  g.N_ghost, sg, st);
        if (e != cudaSuccess) return BOLT_ERR_CUDA;
    }

    // the context path's tiling and p-split rules (the split is chosen for the
    // current device's SM count; the result does not depend on it)
    const bool q2_needed = g.N_q2 > 1 || p.bc_q2 != BOLT_BC_PERIODIC;
    const int tiling = g.N_q2 == 1 ? (q2_needed ? TILING_1D_Q2 : TILING_1D) : TILING_2D;
    const TileShape t = tile_shape(tiling);
    const int ntiles1 = (g.N_q1 + t.tq1 - 1) / t.tq1, ntiles2 = (g.N_q2 + t.tq2 - 1) / t.tq2;
    const int ntab = g.N_p1 + g.N_p2 + g.N_p3;
    const int bgk_direct = (p.p_dim == 1 ||
                            (size_t)t.tq1 * t.tq2 * ntab * sizeof(double) > 64 * 1024) ? 1 : 0;
    const int nchunks = (Np + PW - 1) / PW;
    const size_t smem = qstage_smem(tiling, elem, bgk, bgk_direct, ntab);
    const PSplit sp = choose_psplit(nchunks, (long long)ntiles1 * ntiles2 * g.N_s,
                                    current_sm_count(), smem);

    QStageArgs a;
    memset(&a, 0, sizeof(a));
    const size_t rowbytes = (size_t)g.N_s * Np * elem;
    EncodeTiledFn enc = encode_fn();
    if (enc && g.N_ghost >= HALO && rowbytes % 16 == 0 && ((size_t)Np * elem) % 16 == 0 &&
        ((uintptr_t)f_dev) % 16 == 0) {
        cuuint64_t dims[3] = {(cuuint64_t)g.N_s * Np, (cuuint64_t)Nq1g, (cuuint64_t)Nq2g};
        cuuint64_t strides[2] = {(cuuint64_t)rowbytes, (cuuint64_t)rowbytes * Nq1g};
        cuuint32_t box[3] = {(cuuint32_t)PW, (cuuint32_t)(t.tq1 + 2 * HALO),
                             (cuuint32_t)(t.q2 ? t.tq2 + 2 * HALO : 1)};
        cuuint32_t estr[3] = {1, 1, 1};
        if (enc(&a.tmap, elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                3, const_cast<void*>(f_dev), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS)
            a.use_tma = 1;
    }
    a.fs = f_dev;
    a.out1 = dfdt_dev;                  // write-k mode: out1 <- df/dt
    a.mom_in = scratch;
    a.nsplit_in = 1;
    a.err = err;
    a.flag = err + 1;
    a.wait_cycles = kDefaultWaitCycles;
    a.tau = p.tau;
    a.dq1 = g.dq1; a.dq2 = g.dq2; a.kB = p.boltzmann_constant;
    a.Nq1 = g.N_q1; a.Nq2 = g.N_q2; a.Ng = g.N_ghost; a.Ns = g.N_s;
    a.Np1 = g.N_p1; a.Np2 = g.N_p2; a.Np3 = g.N_p3; a.Np = Np;
    a.Nq1g = Nq1g; a.Nq2g = Nq2g;
    a.nsplit = sp.nsplit;
    a.chunks_per_split = sp.chunks_per_split;
    a.ntiles1 = ntiles1;
    a.p_dim = p.p_dim;
    a.bgk_direct = bgk_direct;
    a.full_chunks = (Np % PW) == 0;
    a.sg = sg;
    dim3 grid_dim(ntiles1 * ntiles2, g.N_s * sp.nsplit);
    cudaError_t e = elem == 8
        ? launch_qstage_f64(a, p.recon_q, tiling, bgk, grid_dim, smem, st)
        : launch_qstage_f32(a, p.recon_q, tiling, bgk, grid_dim, smem, st);
    return e == cudaSuccess ? BOLT_OK : BOLT_ERR_CUDA;
}

extern "C" int bolt_noalloc_status(void* stream, int* status) {
    if (!status) return BOLT_ERR_ARG;
    *status = BOLT_OK;
    double* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    int w[2] = {0, 0};
    int* err = error_words(scratch);
    if (cudaMemcpyAsync(w, err, sizeof(w), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemsetAsync(err, 0, sizeof(w), st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return BOLT_ERR_CUDA;
    *status = w[0] ? w[0] : (w[1] ? BOLT_ERR_NONFINITE : BOLT_OK);
    return BOLT_OK;
}
