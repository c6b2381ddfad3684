// bolt_capi.cu - C ABI of the B200 FVM kinetic update (see include/bolt_b200.h).
//
// Host-side orchestration: context (scratch buffers, moment partial sums,
// fields), TMA descriptors, and the stage sequences of the RK2 midpoint
// stepper of fvm_operator.py:6-35 and of classic RK4 (integrators.py:15-28)
// around the fused stage kernels.
#include <cuda.h>
#include <cuda_runtime.h>

#include <nvtx3/nvToolsExt.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/bolt_b200.h"
#include "launch.h"
#include "validate.h"

using namespace bolt;

namespace {

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

// looked up once per process (a function-local static is initialised once,
// even when several host threads make their first call together)
EncodeTiledFn get_encode_fn() {
    static const EncodeTiledFn fn = lookup_encode_fn();
    return fn;
}

// tensor-map kinds: the stage input's halo box, and the paired kernel's
// 8x8x32 interior boxes (plain, or 128-byte swizzled for the out1 staging tile)
enum TmapKind { TMAP_HALO = 0, TMAP_TILE = 1, TMAP_TILE_SWZ = 2 };
constexpr int kTmapSlots = 16;

struct TmapEntry {
    const void* ptr;
    int kind;
    CUtensorMap map;
};

}  // namespace

struct BoltCtx {
    BoltGrid g;
    BoltParams p;
    SpeciesGrid sg;
    int Nq1g, Nq2g, Np;
    size_t elem;
    size_t fcount;          // elements of one ghosted f
    int tiling, recon_q, recon_p;
    int bgk, bgk_direct, ntab;
    int ntiles1, ntiles2, nsplit, chunks_per_split;
    int use_tma_ok;
    int p_only;             // 1 during bolt_fvm_p_step: df/dt without its q-part
    // scratch
    void* buf[3];
    void* kbuf;
    double* momP[2];        // partial moments [nsplit][5][Ns][Nq2][Nq1]
    double* jpart;          // partial currents [nsplit][3][Ns][Nq2][Nq1]
    int cur_mom;            // index of momP holding moments of the current f
    int cur_nsplit;         // nsplit of that buffer
    const void* mom_owner;  // f pointer whose moments momP[cur_mom] holds (null: stale)
    const void* ghost_owner;
    // fields
    double *cell, *yee, *ebefore, *J;
    int at_n;
    // electrostatic fields: density partials of the df/dt argument, FFT work
    // arrays and the cuFFT plans (0 when unused)
    double* es_part;
    double2 *es_rho, *es_e;
    int es_fwd, es_inv;
    // block neighbours' copies of (f, buf[0], buf[1]): [0] below, [1] above
    // (q2), [2] left, [3] right (q1); peer_on bit 1: q2 on, bit 2: q1 on
    void* peer[4][3];
    int peer_on;
    // misc
    const void* tau_arr;
    const void* dirichlet[4];
    int* hflag;             // pinned, mapped
    int* dflag;
    int* herr;              // device error word: pinned, mapped (host view)
    int* derr;              // (device view)
    double shear_q, shear_omega, time;   // shearing-box constants and strip time
    int ghost_stale_time;   // the time changed since the ghosts of f were sheared
    long long wait_cycles;  // budget of the stage kernels' tile waits
    int stall_test;         // test hook: the stage kernels issue no tile copies
    int sticky;
    long long launches;
    long long pair_launches;    // of which the paired stage kernel
    size_t scratch_bytes;
    TmapEntry tmaps[kTmapSlots];
    int ntmaps, next_tmap;
    // per-component device timing (bolt_set_timing): event pairs of launch
    // groups not yet read back, recycled events, accumulated milliseconds
    struct Timed {
        int cat;
        cudaEvent_t e0, e1;
    };
    std::vector<Timed>* timed;
    std::vector<cudaEvent_t>* free_events;
    double timing_ms[BOLT_TIMING_COUNT];
    int timing_on, timing_depth;
    int pair_enabled;       // paired kernel allowed (BOLT_NO_PAIR unset)
    int pair_shape_ok;      // grid/method meet the paired kernel's shape conditions
};

#define CK(x)                                             \
    do {                                                  \
        cudaError_t e_ = (x);                             \
        if (e_ != cudaSuccess) {                          \
            ctx->sticky = ctx->sticky ? ctx->sticky : BOLT_ERR_CUDA; \
            return BOLT_ERR_CUDA;                         \
        }                                                 \
    } while (0)

static int drain_timing(BoltCtx* ctx);

static inline int bc_dirichlet(int bc) {
    return bc == BOLT_BC_DIRICHLET || bc == BOLT_BC_MIRROR_DIRICHLET;
}
static inline int bc_mirror(int bc) { return bc_is_mirror(bc) ? 1 : 0; }

static int dev_alloc(BoltCtx* ctx, void** p, size_t bytes) {
    if (bytes == 0) {
        *p = nullptr;
        return BOLT_OK;
    }
    if (cudaMalloc(p, bytes) != cudaSuccess) {
        *p = nullptr;
        return BOLT_ERR_NOMEM;
    }
    // zeroed once: cells that no kernel writes (ghost cells of the work
    // buffers, which a copy may carry into f) hold finite values
    if (cudaMemset(*p, 0, bytes) != cudaSuccess) return BOLT_ERR_CUDA;
    ctx->scratch_bytes += bytes;
    return BOLT_OK;
}

static const CUtensorMap* get_tmap(BoltCtx* ctx, const void* ptr, int kind) {
    for (int i = 0; i < ctx->ntmaps; ++i)
        if (ctx->tmaps[i].ptr == ptr && ctx->tmaps[i].kind == kind) return &ctx->tmaps[i].map;
    EncodeTiledFn enc = get_encode_fn();
    if (!enc) return nullptr;
    TileShape t = tile_shape(ctx->tiling);
    cuuint64_t dims[3] = {(cuuint64_t)ctx->g.N_s * ctx->Np, (cuuint64_t)ctx->Nq1g,
                          (cuuint64_t)ctx->Nq2g};
    cuuint64_t strides[2] = {(cuuint64_t)ctx->g.N_s * ctx->Np * ctx->elem,
                             (cuuint64_t)ctx->g.N_s * ctx->Np * ctx->elem * ctx->Nq1g};
    cuuint32_t box[3] = {(cuuint32_t)PW, (cuuint32_t)(t.tq1 + 2 * HALO),
                         (cuuint32_t)(t.q2 ? t.tq2 + 2 * HALO : 1)};
    if (kind != TMAP_HALO) {
        box[1] = 8;
        box[2] = 8;
    }
    // the 128-byte swizzle covers rows of at most 128 bytes: FP64 staging
    // tiles go out as two boxes of 16 p
    if (kind == TMAP_TILE_SWZ && ctx->elem == 8) box[0] = 16;
    cuuint32_t estr[3] = {1, 1, 1};
    CUtensorMap m;
    CUresult r = enc(&m, ctx->elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                        : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                     3, const_cast<void*>(ptr), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE,
                     kind == TMAP_TILE_SWZ ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return nullptr;
    int slot;
    if (ctx->ntmaps < kTmapSlots) {
        slot = ctx->ntmaps++;
    } else {
        slot = ctx->next_tmap;
        ctx->next_tmap = (ctx->next_tmap + 1) % kTmapSlots;
    }
    ctx->tmaps[slot].ptr = ptr;
    ctx->tmaps[slot].kind = kind;
    ctx->tmaps[slot].map = m;
    return &ctx->tmaps[slot].map;
}

extern "C" {

const char* bolt_strerror(int code) {
    switch (code) {
        case BOLT_OK: return "ok";
        case BOLT_ERR_ARG: return "invalid argument";
        case BOLT_ERR_CUDA: return "CUDA error";
        case BOLT_ERR_NONFINITE: return "Solver Diverging!";
        case BOLT_ERR_TIMEOUT: return "device wait timed out";
        case BOLT_ERR_UNSUPPORTED: return "unsupported configuration";
        case BOLT_ERR_NOMEM: return "out of device memory";
        default: return "unknown error";
    }
}

int bolt_ctx_create(const BoltGrid* grid, const BoltParams* params, BoltCtx** out) {
    if (!grid || !params || !out) return BOLT_ERR_ARG;
    *out = nullptr;
    const BoltGrid& g = *grid;
    const BoltParams& p = *params;
    const int vrc = check_grid_params(g, p);
    if (vrc) return vrc;

    BoltCtx* ctx = new (std::nothrow) BoltCtx;
    if (!ctx) return BOLT_ERR_NOMEM;
    memset(ctx, 0, sizeof(BoltCtx));
    ctx->g = g;
    ctx->p = p;
    ctx->Nq1g = g.N_q1 + 2 * g.N_ghost;
    ctx->Nq2g = g.N_q2 + 2 * g.N_ghost;
    ctx->Np = g.N_p1 * g.N_p2 * g.N_p3;
    ctx->elem = p.dtype == BOLT_F32 ? 4 : 8;
    ctx->fcount = (size_t)ctx->Nq1g * ctx->Nq2g * g.N_s * ctx->Np;
    for (int s = 0; s < g.N_s; ++s) {
        ctx->sg.p1_start[s] = g.p1_start[s];
        ctx->sg.p2_start[s] = g.p2_start[s];
        ctx->sg.p3_start[s] = g.p3_start[s];
        ctx->sg.dp1[s] = g.dp1[s];
        ctx->sg.dp2[s] = g.dp2[s];
        ctx->sg.dp3[s] = g.dp3[s];
        ctx->sg.mass[s] = p.mass[s];
        ctx->sg.charge[s] = p.charge[s];
    }
    // q-tiling: the q2 stencil is skipped only when it contributes exactly
    // zero (one periodic q2 cell: identical neighbours give identical faces)
    // and no current along q2 is needed
    const bool q2_needed = g.N_q2 > 1 || p.bc_q2 != BOLT_BC_PERIODIC || p.fields_enabled;
    if (g.N_q2 == 1)
        ctx->tiling = q2_needed ? TILING_1D_Q2 : TILING_1D;
    else
        ctx->tiling = TILING_2D;
    TileShape t = tile_shape(ctx->tiling);
    ctx->ntiles1 = (g.N_q1 + t.tq1 - 1) / t.tq1;
    ctx->ntiles2 = (g.N_q2 + t.tq2 - 1) / t.tq2;
    ctx->recon_q = p.recon_q;
    ctx->recon_p = p.recon_p;
    ctx->bgk = p.source_enabled ? 1 : 0;
    ctx->ntab = g.N_p1 + g.N_p2 + g.N_p3;
    ctx->bgk_direct = (p.p_dim == 1 ||
                       (size_t)t.tq1 * t.tq2 * ctx->ntab * sizeof(double) > 64 * 1024) ? 1 : 0;
    // the paired kernel's shape conditions (the per-call ones are checked at
    // launch): FP32, or FP64 in its throughput form
    ctx->pair_shape_ok = (ctx->elem == 4 || p.dtype == BOLT_F64_FAST) &&
                         ctx->tiling == TILING_2D && !(ctx->bgk && ctx->bgk_direct) &&
                         g.N_q1 % 8 == 0 && g.N_q2 % 8 == 0 && ctx->Np % PW == 0 &&
                         g.N_p1 % 8 == 0 && 2 * g.N_ghost <= g.N_q1 &&
                         2 * g.N_ghost <= g.N_q2 && ctx->fcount < (1ull << 31);
    if (ctx->pair_shape_ok) {
        // its shared memory (exp tables grow with N_p1 + N_p2 + N_p3) must fit a CTA
        int dev = 0, optin = 232448;
        if (cudaGetDevice(&dev) == cudaSuccess)
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (qpair_smem(ctx->ntab, ctx->bgk, ctx->elem) > (size_t)optin) ctx->pair_shape_ok = 0;
    }
    // p-splits: the grid is (q-tiles, species x splits)
    {
        const size_t smem_est = ctx->pair_shape_ok
            ? qpair_smem(ctx->ntab, ctx->bgk, ctx->elem)
            : qstage_smem(ctx->tiling, ctx->elem, ctx->bgk, ctx->bgk_direct, ctx->ntab);
        const int nchunks = (ctx->Np + PW - 1) / PW;
        const long long base_ctas = (long long)ctx->ntiles1 * ctx->ntiles2 * g.N_s;
        PSplit sp = choose_psplit(nchunks, base_ctas, current_sm_count(), smem_est);
        // BOLT_CHUNKS_PER_SPLIT fixes the split instead (tests run one problem
        // under several splits; results differ only in the order of the FP64
        // moment partial sums)
        if (const char* env = getenv("BOLT_CHUNKS_PER_SPLIT")) {
            const int c = atoi(env);
            if (c >= 1) {
                sp.chunks_per_split = c < nchunks ? c : nchunks;
                sp.nsplit = (nchunks + sp.chunks_per_split - 1) / sp.chunks_per_split;
            }
        }
        ctx->chunks_per_split = sp.chunks_per_split;
        ctx->nsplit = sp.nsplit;
    }
    const size_t rowbytes = (size_t)g.N_s * ctx->Np * ctx->elem;
    ctx->use_tma_ok = (g.N_ghost >= HALO) && (rowbytes % 16 == 0) &&
                      (((size_t)ctx->Np * ctx->elem) % 16 == 0) && get_encode_fn() != nullptr;
    ctx->at_n = 1;
    ctx->pair_enabled = getenv("BOLT_NO_PAIR") == nullptr;

    int rc = BOLT_OK;
    const size_t fbytes = ctx->fcount * ctx->elem;
    const int nbuf = p.integrator == BOLT_RK4 ? 3 : 1;
    for (int i = 0; i < nbuf && rc == BOLT_OK; ++i) rc = dev_alloc(ctx, &ctx->buf[i], fbytes);
    if (rc == BOLT_OK && p.fields_enabled) rc = dev_alloc(ctx, &ctx->kbuf, fbytes);
    const size_t plane = (size_t)g.N_q1 * g.N_q2 * g.N_s;
    const int nsp = ctx->nsplit > 1 ? ctx->nsplit : 1;
    for (int i = 0; i < 2 && rc == BOLT_OK; ++i)
        rc = dev_alloc(ctx, (void**)&ctx->momP[i], (size_t)nsp * kNumMom * plane * sizeof(double));
    if (rc == BOLT_OK && p.fields_enabled) {
        const size_t fp = (size_t)ctx->Nq1g * ctx->Nq2g;
        rc = dev_alloc(ctx, (void**)&ctx->jpart, (size_t)nsp * 3 * plane * sizeof(double));
        if (rc == BOLT_OK) rc = dev_alloc(ctx, (void**)&ctx->cell, 6 * fp * sizeof(double));
        if (rc == BOLT_OK) rc = dev_alloc(ctx, (void**)&ctx->yee, 6 * fp * sizeof(double));
        if (rc == BOLT_OK) rc = dev_alloc(ctx, (void**)&ctx->ebefore, 3 * fp * sizeof(double));
        if (rc == BOLT_OK) rc = dev_alloc(ctx, (void**)&ctx->J, 3 * fp * sizeof(double));
        if (rc == BOLT_OK) {
            cudaMemset(ctx->cell, 0, 6 * fp * sizeof(double));
            cudaMemset(ctx->yee, 0, 6 * fp * sizeof(double));
        }
        if (rc == BOLT_OK && p.fields_type == BOLT_FIELDS_ELECTROSTATIC) {
            const size_t nq = (size_t)g.N_q1 * g.N_q2;
            rc = dev_alloc(ctx, (void**)&ctx->es_part, kNumMom * plane * sizeof(double));
            if (rc == BOLT_OK) rc = dev_alloc(ctx, (void**)&ctx->es_rho, nq * sizeof(double2));
            if (rc == BOLT_OK) rc = dev_alloc(ctx, (void**)&ctx->es_e, 2 * nq * sizeof(double2));
            if (rc == BOLT_OK && poisson_plans_create(g.N_q1, g.N_q2, &ctx->es_fwd, &ctx->es_inv))
                rc = BOLT_ERR_CUDA;
        }
    }
    // the divergence flag and the error word live in pinned host memory the
    // kernels write through its device mapping, so the host reads either
    // without synchronising
    if (rc == BOLT_OK) {
        if (cudaHostAlloc((void**)&ctx->hflag, 2 * sizeof(int), cudaHostAllocMapped) !=
                cudaSuccess ||
            cudaHostGetDevicePointer((void**)&ctx->dflag, ctx->hflag, 0) != cudaSuccess) {
            rc = BOLT_ERR_CUDA;
        } else {
            ctx->hflag[0] = ctx->hflag[1] = 0;
            ctx->herr = ctx->hflag + 1;
            ctx->derr = ctx->dflag + 1;
        }
    }
    ctx->wait_cycles = kDefaultWaitCycles;
    if (rc == BOLT_OK && cudaDeviceSynchronize() != cudaSuccess) rc = BOLT_ERR_CUDA;
    if (rc != BOLT_OK) {
        bolt_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return BOLT_OK;
}

void bolt_ctx_destroy(BoltCtx* ctx) {
    if (!ctx) return;
    for (int i = 0; i < 3; ++i) cudaFree(ctx->buf[i]);
    cudaFree(ctx->kbuf);
    cudaFree(ctx->momP[0]);
    cudaFree(ctx->momP[1]);
    cudaFree(ctx->jpart);
    cudaFree(ctx->cell);
    cudaFree(ctx->yee);
    cudaFree(ctx->ebefore);
    cudaFree(ctx->J);
    cudaFree(ctx->es_part);
    cudaFree(ctx->es_rho);
    cudaFree(ctx->es_e);
    poisson_plans_destroy(ctx->es_fwd, ctx->es_inv);
    if (ctx->hflag) cudaFreeHost(ctx->hflag);
    if (ctx->timed) {
        for (auto& t : *ctx->timed) {
            cudaEventDestroy(t.e0);
            cudaEventDestroy(t.e1);
        }
        delete ctx->timed;
    }
    if (ctx->free_events) {
        for (cudaEvent_t e : *ctx->free_events) cudaEventDestroy(e);
        delete ctx->free_events;
    }
    delete ctx;
}

int bolt_set_tau_array(BoltCtx* ctx, const void* tau_dev) {
    if (!ctx) return BOLT_ERR_ARG;
    ctx->tau_arr = tau_dev;
    return BOLT_OK;
}

int bolt_set_dirichlet(BoltCtx* ctx, int side, const void* values_dev) {
    if (!ctx || side < 0 || side > 3) return BOLT_ERR_ARG;
    ctx->dirichlet[side] = values_dev;
    ctx->ghost_owner = nullptr;
    return BOLT_OK;
}

// neighbours lo / hi along one axis (side 0: q2, 1: q1) of an external axis
static int set_peers(BoltCtx* ctx, int side, int bc, const void* const* lo,
                     const void* const* hi) {
    if (!ctx) return BOLT_ERR_ARG;
    const int bit = 1 << side;
    if (!lo || !hi) {
        ctx->peer_on &= ~bit;
        for (int i = 0; i < 3; ++i) ctx->peer[2 * side][i] = ctx->peer[2 * side + 1][i] = nullptr;
        return BOLT_OK;
    }
    if (bc != BOLT_BC_EXTERNAL || ctx->p.fields_enabled) return BOLT_ERR_UNSUPPORTED;
    const int nb = ctx->p.integrator == BOLT_RK4 ? 3 : 2;   // f and the stage inputs
    for (int i = 0; i < nb; ++i)
        if (!lo[i] || !hi[i]) return BOLT_ERR_ARG;
    for (int i = 0; i < 3; ++i) {
        ctx->peer[2 * side][i] = i < nb ? const_cast<void*>(lo[i]) : nullptr;
        ctx->peer[2 * side + 1][i] = i < nb ? const_cast<void*>(hi[i]) : nullptr;
    }
    ctx->peer_on |= bit;
    return BOLT_OK;
}

int bolt_set_peer_halos(BoltCtx* ctx, const void* const* below, const void* const* above) {
    return set_peers(ctx, 0, ctx ? ctx->p.bc_q2 : 0, below, above);
}

int bolt_set_peer_halos_q1(BoltCtx* ctx, const void* const* left, const void* const* right) {
    return set_peers(ctx, 1, ctx ? ctx->p.bc_q1 : 0, left, right);
}

int bolt_ipc_get(const void* dev_ptr, unsigned char* handle64) {
    if (!dev_ptr || !handle64) return BOLT_ERR_ARG;
    cudaIpcMemHandle_t h;
    if (cudaIpcGetMemHandle(&h, const_cast<void*>(dev_ptr)) != cudaSuccess) return BOLT_ERR_CUDA;
    static_assert(sizeof(h) == 64, "CUDA IPC handles are 64 bytes");
    memcpy(handle64, &h, sizeof(h));
    return BOLT_OK;
}

int bolt_ipc_open(const unsigned char* handle64, void** dev_ptr) {
    if (!handle64 || !dev_ptr) return BOLT_ERR_ARG;
    cudaIpcMemHandle_t h;
    memcpy(&h, handle64, sizeof(h));
    if (cudaIpcOpenMemHandle(dev_ptr, h, cudaIpcMemLazyEnablePeerAccess) != cudaSuccess)
        return BOLT_ERR_CUDA;
    return BOLT_OK;
}

int bolt_ipc_close(void* dev_ptr) {
    if (!dev_ptr) return BOLT_ERR_ARG;
    return cudaIpcCloseMemHandle(dev_ptr) == cudaSuccess ? BOLT_OK : BOLT_ERR_CUDA;
}

void* bolt_stage_buffer(BoltCtx* ctx, int i) {
    if (!ctx || i < 0 || i > 1) return nullptr;
    return ctx->buf[i];
}

long long bolt_launch_count(BoltCtx* ctx) { return ctx ? ctx->launches : 0; }
long long bolt_paired_launch_count(BoltCtx* ctx) { return ctx ? ctx->pair_launches : 0; }
int bolt_split_info(BoltCtx* ctx, int* nsplit, int* chunks_per_split) {
    if (!ctx || !nsplit || !chunks_per_split) return BOLT_ERR_ARG;
    *nsplit = ctx->nsplit;
    *chunks_per_split = ctx->chunks_per_split;
    return BOLT_OK;
}
size_t bolt_scratch_bytes(BoltCtx* ctx) { return ctx ? ctx->scratch_bytes : 0; }

int bolt_divergence_flag(BoltCtx* ctx) {
    if (!ctx || !ctx->hflag) return 0;
    return *(volatile int*)ctx->hflag ? 1 : 0;
}

int bolt_clear_divergence_flag(BoltCtx* ctx) {
    if (!ctx || !ctx->hflag) return BOLT_ERR_ARG;
    *(volatile int*)ctx->hflag = 0;
    return BOLT_OK;
}

int bolt_status_sync(BoltCtx* ctx, void* stream) {
    if (!ctx) return BOLT_ERR_ARG;
    if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return BOLT_ERR_CUDA;
    const int e = *(volatile int*)ctx->herr;
    if (e) return e;
    if (ctx->sticky) return ctx->sticky;
    return BOLT_OK;
}

int bolt_error_flag(BoltCtx* ctx) {
    if (!ctx || !ctx->herr) return BOLT_ERR_ARG;
    return *(volatile int*)ctx->herr;
}

int bolt_clear_error(BoltCtx* ctx) {
    if (!ctx || !ctx->herr) return BOLT_ERR_ARG;
    *(volatile int*)ctx->herr = 0;
    return BOLT_OK;
}

int bolt_set_wait_budget(BoltCtx* ctx, long long cycles) {
    if (!ctx) return BOLT_ERR_ARG;
    ctx->wait_cycles = cycles > 0 ? cycles : kDefaultWaitCycles;
    return BOLT_OK;
}

int bolt_set_timing(BoltCtx* ctx, int on) {
    if (!ctx) return BOLT_ERR_ARG;
    if (on && !ctx->timed) {
        ctx->timed = new (std::nothrow) std::vector<BoltCtx::Timed>();
        ctx->free_events = new (std::nothrow) std::vector<cudaEvent_t>();
        if (!ctx->timed || !ctx->free_events) return BOLT_ERR_NOMEM;
    }
    ctx->timing_on = on ? 1 : 0;
    ctx->timing_depth = 0;
    return BOLT_OK;
}

int bolt_timings(BoltCtx* ctx, double* ms_out) {
    if (!ctx || !ms_out) return BOLT_ERR_ARG;
    const int rc = drain_timing(ctx);
    for (int i = 0; i < BOLT_TIMING_COUNT; ++i) {
        ms_out[i] = ctx->timing_ms[i];
        ctx->timing_ms[i] = 0.0;
    }
    return rc;
}

int bolt_test_stall_waits(BoltCtx* ctx, int on) {
    if (!ctx) return BOLT_ERR_ARG;
    ctx->stall_test = on ? 1 : 0;
    return BOLT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// internal launch helpers
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// per-component timing: a TimedScope brackets one launch group with CUDA
// events (outermost scope only) and names it for NVTX-based profilers
// ---------------------------------------------------------------------------
static cudaEvent_t timing_event(BoltCtx* ctx) {
    if (!ctx->free_events->empty()) {
        cudaEvent_t e = ctx->free_events->back();
        ctx->free_events->pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// read back every recorded pair (synchronising on the last one)
static int drain_timing(BoltCtx* ctx) {
    if (!ctx->timed) return BOLT_OK;
    int rc = BOLT_OK;
    for (auto& t : *ctx->timed) {
        float ms = 0.0f;
        if (cudaEventSynchronize(t.e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, t.e0, t.e1) != cudaSuccess)
            rc = BOLT_ERR_CUDA;
        else
            ctx->timing_ms[t.cat] += ms;
        ctx->free_events->push_back(t.e0);
        ctx->free_events->push_back(t.e1);
    }
    ctx->timed->clear();
    return rc;
}

static const char* const kTimingNames[BOLT_TIMING_COUNT] = {
    "bolt: ghosts", "bolt: moments", "bolt: q-stage", "bolt: p-stage", "bolt: fields"};

struct TimedScope {
    BoltCtx* ctx;
    cudaStream_t st;
    int cat;
    bool rec;
    cudaEvent_t e0;
    TimedScope(BoltCtx* c, int category, cudaStream_t s) : ctx(c), st(s), cat(category) {
        nvtxRangePushA(kTimingNames[cat]);
        rec = ctx->timing_on && ctx->timing_depth++ == 0;
        if (rec) {
            e0 = timing_event(ctx);
            cudaEventRecord(e0, st);
        }
    }
    ~TimedScope() {
        if (ctx->timing_on) --ctx->timing_depth;
        if (rec) {
            cudaEvent_t e1 = timing_event(ctx);
            cudaEventRecord(e1, st);
            ctx->timed->push_back({cat, e0, e1});
            if (ctx->timed->size() >= 4096) drain_timing(ctx);   // bounded event use
        }
        nvtxRangePop();
    }
};

static int launch_ghosts(BoltCtx* ctx, void* f, cudaStream_t st) {
    TimedScope ts(ctx, BOLT_TIMING_GHOSTS, st);
    const BoltGrid& g = ctx->g;
    const int dir1 = bc_dirichlet(ctx->p.bc_q1), dir2 = bc_dirichlet(ctx->p.bc_q2);
    const int mir1 = bc_mirror(ctx->p.bc_q1), mir2 = bc_mirror(ctx->p.bc_q2);
    const int ext1 = ctx->p.bc_q1 == BOLT_BC_EXTERNAL, ext2 = ctx->p.bc_q2 == BOLT_BC_EXTERNAL;
    const int per1 = ctx->p.bc_q1 == BOLT_BC_PERIODIC, per2 = ctx->p.bc_q2 == BOLT_BC_PERIODIC;
    if (g.N_ghost == 0) return BOLT_OK;
    GhostShear sh;
    memset(&sh, 0, sizeof(sh));
    if (ctx->p.bc_q1 == BOLT_BC_SHEARING_BOX || ctx->p.bc_q2 == BOLT_BC_SHEARING_BOX) {
        // boundaries.py:19-22: shift q omega L t along the other axis, L the
        // length of the strip's own axis, reduced modulo the other's length
        const bool a1 = ctx->p.bc_q1 == BOLT_BC_SHEARING_BOX;
        const double L_own = a1 ? g.N_q1 * g.dq1 : g.N_q2 * g.dq2;
        sh.axis = a1 ? 1 : 2;
        sh.start = a1 ? g.q2_start : g.q1_start;
        sh.dq = a1 ? g.dq2 : g.dq1;
        sh.end = sh.start + (a1 ? g.N_q2 : g.N_q1) * sh.dq;
        sh.shift = fmod(ctx->shear_q * ctx->shear_omega * L_own * ctx->time, sh.end - sh.start);
        if (!(sh.shift == sh.shift)) sh.shift = 0.0;          // a non-finite time
    }
    if ((dir1 && (!ctx->dirichlet[0] || !ctx->dirichlet[1])) ||
        (dir2 && (!ctx->dirichlet[2] || !ctx->dirichlet[3])))
        return BOLT_ERR_ARG;
    cudaError_t e;
    if (ctx->elem == 8)
        e = launch_ghost_f64(f, ctx->dirichlet[0], ctx->dirichlet[1], ctx->dirichlet[2],
                             ctx->dirichlet[3], g.N_q1, g.N_q2, g.N_ghost, g.N_s, ctx->Np,
                             g.N_p1, g.N_p2, per1, per2, dir1, dir2, mir1, mir2, ext1, ext2, ctx->sg,
                             sh, st);
    else
        e = launch_ghost_f32(f, ctx->dirichlet[0], ctx->dirichlet[1], ctx->dirichlet[2],
                             ctx->dirichlet[3], g.N_q1, g.N_q2, g.N_ghost, g.N_s, ctx->Np,
                             g.N_p1, g.N_p2, per1, per2, dir1, dir2, mir1, mir2, ext1, ext2, ctx->sg,
                             sh, st);
    ctx->launches++;
    CK(e);
    return BOLT_OK;
}

static int launch_moments5(BoltCtx* ctx, const void* f, double* part, cudaStream_t st) {
    TimedScope ts(ctx, BOLT_TIMING_MOMENTS, st);
    const BoltGrid& g = ctx->g;
    cudaError_t e = ctx->elem == 8
        ? launch_moments5_f64(f, part, g.N_s, g.N_p1, g.N_p2, g.N_p3, g.N_q1, g.N_q2, g.N_ghost,
                              ctx->sg, st)
        : launch_moments5_f32(f, part, g.N_s, g.N_p1, g.N_p2, g.N_p3, g.N_q1, g.N_q2, g.N_ghost,
                              ctx->sg, st);
    ctx->launches++;
    CK(e);
    return BOLT_OK;
}

struct StageIO {
    void* peer_lo;          // neighbours' copies of out1 (q2 cut) or null
    void* peer_hi;
    void* peer_left;        // neighbours' copies of out1 (q1 cut) or null
    void* peer_right;
    const void* fs;
    const void* base1;
    double c1;
    void* out1;
    const void* base2;
    double c2;
    void* out2;
    const double* mom_in;
    int nsplit_in;
    double* mom_out;
    int* flag;
};

// q-part of one stage.  write_k: out1 <- k_q (no moments, no ghosts).
// region -1: every q-tile; 0: the tiles whose stencils stay inside the block
// along its external axes; 1: the other tiles (0 and 1 need the paired
// kernel: BOLT_ERR_UNSUPPORTED, with nothing launched, where it does not run)
static int launch_qstage(BoltCtx* ctx, const StageIO& io, int write_k, int want_j,
                         cudaStream_t st, int region = -1) {
    TimedScope ts(ctx, BOLT_TIMING_QSTAGE, st);
    const BoltGrid& g = ctx->g;
    QStageArgs a;
    memset(&a, 0, sizeof(a));
    a.use_tma = 0;
    if (ctx->use_tma_ok && (((uintptr_t)io.fs) % 16 == 0)) {
        const CUtensorMap* m = get_tmap(ctx, io.fs, TMAP_HALO);
        if (m) {
            a.tmap = *m;
            a.use_tma = 1;
        }
    }
    a.fs = io.fs;
    a.base1 = write_k ? nullptr : io.base1;
    a.base2 = write_k ? nullptr : io.base2;
    a.out1 = io.out1;
    a.out2 = write_k ? nullptr : io.out2;
    a.peer_lo = write_k ? nullptr : io.peer_lo;
    a.peer_hi = write_k ? nullptr : io.peer_hi;
    a.peer_left = write_k ? nullptr : io.peer_left;
    a.peer_right = write_k ? nullptr : io.peer_right;
    a.tau_arr = ctx->tau_arr;
    a.mom_in = io.mom_in;
    a.mom_out = write_k ? nullptr : io.mom_out;
    a.j_out = want_j ? ctx->jpart : nullptr;
    a.flag = write_k ? nullptr : io.flag;
    a.err = ctx->derr;
    a.wait_cycles = ctx->wait_cycles;
    a.stall_test = ctx->stall_test;
    a.c1 = io.c1;
    a.c2 = io.c2;
    a.tau = ctx->p.tau;
    a.dq1 = g.dq1;
    a.dq2 = g.dq2;
    a.kB = ctx->p.boltzmann_constant;
    a.Nq1 = g.N_q1; a.Nq2 = g.N_q2; a.Ng = g.N_ghost; a.Ns = g.N_s;
    a.Np1 = g.N_p1; a.Np2 = g.N_p2; a.Np3 = g.N_p3; a.Np = ctx->Np;
    a.Nq1g = ctx->Nq1g; a.Nq2g = ctx->Nq2g;
    const TileShape t = tile_shape(ctx->tiling);
    a.periodic1 = !write_k && ctx->p.bc_q1 == BOLT_BC_PERIODIC && g.N_ghost > 0;
    a.periodic2 = !write_k && ctx->p.bc_q2 == BOLT_BC_PERIODIC && g.N_ghost > 0 && t.q2;
    a.nsplit_in = io.nsplit_in;
    a.nsplit = ctx->nsplit;
    a.chunks_per_split = ctx->chunks_per_split;
    a.ntiles1 = ctx->ntiles1;
    a.ntiles2 = ctx->ntiles2;
    a.ext1 = ctx->p.bc_q1 == BOLT_BC_EXTERNAL;
    a.ext2 = ctx->p.bc_q2 == BOLT_BC_EXTERNAL;
    a.tile_sel = region < 0 ? 0 : region + 1;
    a.p_dim = ctx->p.p_dim;
    a.want_j = want_j;
    a.bgk_direct = ctx->bgk_direct;
    a.full_chunks = (ctx->Np % PW) == 0;
    a.sg = ctx->sg;
    dim3 grid(ctx->ntiles1 * ctx->ntiles2, g.N_s * ctx->nsplit);
    // the paired kernel (FP32, or FP64 throughput form) covers the fused 2-D stage with every
    // buffer reachable by TMA; everything else (FP64, other reconstructions,
    // 1-D tilings, write-k mode, currents, tau arrays) runs the scalar kernel
    // (so do the write-k stages of field-coupled steps, unless they also
    // accumulate currents; bolt_dfdt without fields keeps the scalar kernel,
    // the one bolt_dfdt_noalloc runs, so the two agree to the bit)
    bool pair = ctx->pair_shape_ok && ctx->pair_enabled && !want_j && a.use_tma &&
                (write_k ? ctx->p.fields_enabled != 0 : a.base1 != nullptr) &&
                ctx->tau_arr == nullptr;
    if (pair) {
        const void* ptrs[4] = {a.base1, a.out1, a.base2, a.out2};
        for (int i = 0; i < 4; ++i)
            if (ptrs[i] && ((uintptr_t)ptrs[i]) % 16 != 0) pair = false;
        if ((a.base2 == nullptr) != (a.out2 == nullptr)) pair = false;
        // stage shapes of the paired kernel: bases = stage input, or out2 is
        // its own base (accumulated in place), or no out2
        const bool bx = a.base1 == a.fs && (!a.base2 || a.base2 == a.fs);
        if (a.base2 && !bx && a.base2 != a.out2) pair = false;
    }
    if (pair) {
        // copy each map out at once: a later lookup may recycle its cache slot
        const CUtensorMap* m;
        if (a.base1) {
            if ((m = get_tmap(ctx, a.base1, TMAP_TILE))) a.tm_b1 = *m; else pair = false;
        }
        if (pair && (m = get_tmap(ctx, a.out1, TMAP_TILE_SWZ))) a.tm_o1 = *m; else pair = false;
        if (!a.base1) a.tm_b1 = a.tm_o1;            // unused (no base tiles): a valid map
        a.tm_o2 = a.tm_o1;
        if (pair && a.out2) {
            if ((m = get_tmap(ctx, a.out2, TMAP_TILE))) a.tm_o2 = *m; else pair = false;
        }
    }
    if (region >= 0) {
        if (!pair) return BOLT_ERR_UNSUPPORTED;
        const int n1 = ctx->ntiles1, n2 = ctx->ntiles2;
        const int inner = std::max(0, n1 - 2 * a.ext1) * std::max(0, n2 - 2 * a.ext2);
        const int count = region == 0 ? inner : n1 * n2 - inner;
        if (count == 0) return BOLT_OK;
        grid.x = (unsigned)count;
    }
    const size_t smem = pair ? qpair_smem(ctx->ntab, ctx->bgk, ctx->elem)
                             : qstage_smem(ctx->tiling, ctx->elem, ctx->bgk, ctx->bgk_direct,
                                           ctx->ntab);
    cudaError_t e = ctx->elem == 8
        ? (pair ? launch_qpair_f64(a, ctx->bgk, ctx->recon_q, grid, smem, st)
                : launch_qstage_f64(a, ctx->recon_q, ctx->tiling, ctx->bgk, grid, smem, st))
        : (pair ? launch_qpair_f32(a, ctx->bgk, ctx->recon_q, grid, smem, st)
                : launch_qstage_f32(a, ctx->recon_q, ctx->tiling, ctx->bgk, grid, smem, st));
    ctx->launches++;
    if (pair) ctx->pair_launches++;
    CK(e);
    return BOLT_OK;
}

static int launch_pstage(BoltCtx* ctx, const StageIO& io, const void* kq, cudaStream_t st,
                         int term = 0) {
    TimedScope ts(ctx, BOLT_TIMING_PSTAGE, st);
    const BoltGrid& g = ctx->g;
    PStageArgs a;
    memset(&a, 0, sizeof(a));
    a.fs = io.fs;
    a.kq = kq;
    a.base1 = io.base1;
    a.base2 = io.base2;
    a.out1 = io.out1;
    a.out2 = io.out2;
    a.cell = ctx->cell;
    a.mom_out = io.mom_out;
    a.flag = io.flag;
    a.c1 = io.c1;
    a.c2 = io.c2;
    a.Nq1 = g.N_q1; a.Nq2 = g.N_q2; a.Ng = g.N_ghost; a.Ns = g.N_s;
    a.Np1 = g.N_p1; a.Np2 = g.N_p2; a.Np3 = g.N_p3; a.Np = ctx->Np;
    a.Nq1g = ctx->Nq1g; a.Nq2g = ctx->Nq2g;
    a.periodic1 = io.base1 != nullptr && ctx->p.bc_q1 == BOLT_BC_PERIODIC && g.N_ghost > 0;
    a.periodic2 = io.base1 != nullptr && ctx->p.bc_q2 == BOLT_BC_PERIODIC && g.N_ghost > 0;
    a.term = term;
    if (term) {
        a.periodic1 = a.periodic2 = 0;
        a.mom_out = nullptr;
        a.flag = nullptr;
    }
    a.sg = ctx->sg;
    const size_t smem = pstage_smem(ctx->Np, ctx->elem, g.N_p1 + g.N_p2 + g.N_p3);
    if (smem > 200 * 1024) return BOLT_ERR_UNSUPPORTED;
    dim3 grid(g.N_q1 * g.N_q2, g.N_s);
    cudaError_t e = ctx->elem == 8 ? launch_pstage_f64(a, ctx->recon_p, grid, smem, st)
                                   : launch_pstage_f32(a, ctx->recon_p, grid, smem, st);
    ctx->launches++;
    CK(e);
    return BOLT_OK;
}

// the FDTD update (part -1), or one of its three parts (a field-evolving
// stage of a block whose Yee ghosts are exchanged between the parts)
static int launch_fields(BoltCtx* ctx, double dt, int nsplit_j, cudaStream_t st,
                         const double* j_given = nullptr, int part = -1) {
    TimedScope ts(ctx, BOLT_TIMING_FIELDS, st);
    const BoltGrid& g = ctx->g;
    FieldArgs a;
    memset(&a, 0, sizeof(a));
    a.yee = ctx->yee;
    a.cell = ctx->cell;
    a.ebefore = ctx->ebefore;
    a.J = ctx->J;
    a.jpart = ctx->jpart;
    a.j_given = j_given;
    a.nsplit = nsplit_j;
    a.Ns = g.N_s; a.Nq1 = g.N_q1; a.Nq2 = g.N_q2; a.Ng = g.N_ghost;
    a.Nq1g = ctx->Nq1g; a.Nq2g = ctx->Nq2g;
    a.ext1 = ctx->p.bc_q1 == BOLT_BC_EXTERNAL;
    a.ext2 = ctx->p.bc_q2 == BOLT_BC_EXTERNAL;
    a.dq1 = g.dq1; a.dq2 = g.dq2; a.dt = dt; a.eps = ctx->p.eps; a.mu = ctx->p.mu;
    for (int s = 0; s < g.N_s; ++s) {
        a.charge[s] = ctx->p.charge[s];
        a.measure[s] = (g.dp3[s] * g.dp2[s]) * g.dp1[s];
    }
    a.mom_scale = ctx->sg.polar2d ? ctx->sg.mom_scale : 1.0;
    if (part < 0) CK(launch_fdtd(a, st, &ctx->launches));
    else CK(launch_fdtd_part(a, part, st, &ctx->launches));
    return BOLT_OK;
}

static int electrostatic(const BoltCtx* ctx) {
    return ctx->p.fields_enabled && ctx->p.fields_type == BOLT_FIELDS_ELECTROSTATIC;
}

// electrostatic fields of the df/dt argument f (df_dt_fvm.py:234-242): its
// species densities, then the FFT Poisson solve into the cell-centred E1, E2
static int launch_electrostatic(BoltCtx* ctx, const void* f, cudaStream_t st) {
    TimedScope ts(ctx, BOLT_TIMING_FIELDS, st);
    const BoltGrid& g = ctx->g;
    int rc = launch_moments5(ctx, f, ctx->es_part, st);
    if (rc) return rc;
    PoissonArgs a;
    memset(&a, 0, sizeof(a));
    a.part = ctx->es_part;
    a.rho_hat = ctx->es_rho;
    a.e_hat = ctx->es_e;
    a.cell = ctx->cell;
    a.Nq1 = g.N_q1; a.Nq2 = g.N_q2; a.Ng = g.N_ghost; a.Ns = g.N_s;
    a.dq1 = g.dq1; a.dq2 = g.dq2; a.eps = ctx->p.eps;
    for (int s = 0; s < g.N_s; ++s) {
        a.charge[s] = ctx->p.charge[s];
        a.measure[s] = (g.dp3[s] * g.dp2[s]) * g.dp1[s];
    }
    a.mom_scale = ctx->sg.polar2d ? ctx->sg.mom_scale : 1.0;
    CK(launch_poisson(a, ctx->es_fwd, ctx->es_inv, st, &ctx->launches));
    return BOLT_OK;
}

// one df/dt evaluation + stage update: q-part (fused combine when there is no
// p-advection), then p-part when fields are enabled.  part -1 runs the whole
// stage; a field-evolving stage of a block runs as parts 0..2 with the Yee
// ghosts exchanged between them (0: q-part, currents, halo; 1: E update;
// 2: B update, cell fields, p-part)
static int run_stage(BoltCtx* ctx, StageIO io, int evolve, double dt, cudaStream_t st,
                     int part = -1, int region = -1) {
    int rc;
    if (!ctx->p.fields_enabled) {
        rc = launch_qstage(ctx, io, 0, 0, st, region);
    } else if (electrostatic(ctx)) {
        rc = launch_electrostatic(ctx, io.fs, st);
        StageIO qio = io;
        qio.out1 = ctx->kbuf;
        if (rc == BOLT_OK && ctx->p_only) {
            // the q-part (and the source) belong to the semi-Lagrangian q-step
            const cudaError_t e = cudaMemsetAsync(ctx->kbuf, 0, ctx->fcount * ctx->elem, st);
            if (e != cudaSuccess) rc = BOLT_ERR_CUDA;
        } else if (rc == BOLT_OK) {
            rc = launch_qstage(ctx, qio, 1, 0, st);
        }
        if (rc == BOLT_OK) rc = launch_pstage(ctx, io, ctx->kbuf, st);
    } else {
        StageIO qio = io;
        qio.out1 = ctx->kbuf;
        rc = BOLT_OK;
        if (part <= 0) rc = launch_qstage(ctx, qio, 1, evolve, st);
        if (rc == BOLT_OK && evolve) rc = launch_fields(ctx, dt, ctx->nsplit, st, nullptr, part);
        if (rc == BOLT_OK && (part < 0 || part == 2)) rc = launch_pstage(ctx, io, ctx->kbuf, st);
    }
    return rc;
}

static int ensure_state(BoltCtx* ctx, void* f, cudaStream_t st) {
    int rc = BOLT_OK;
    if (ctx->ghost_owner != f) {
        rc = launch_ghosts(ctx, f, st);
        if (rc) return rc;
        ctx->ghost_owner = f;
        ctx->mom_owner = nullptr;
    } else if (ctx->ghost_stale_time) {
        // shearing-box strips of the new time (the interior, and so the
        // moments, are unchanged)
        rc = launch_ghosts(ctx, f, st);
        if (rc) return rc;
    }
    ctx->ghost_stale_time = 0;
    if (ctx->bgk && ctx->mom_owner != f) {
        rc = launch_moments5(ctx, f, ctx->momP[ctx->cur_mom], st);
        if (rc) return rc;
        ctx->cur_nsplit = 1;
        ctx->mom_owner = f;
    }
    return rc;
}

// Stage k of one step of f (RK2: k = 0, 1; RK4: k = 0..3, in order).  Stage
// k reads the moments written by stage k-1 (the ping-pong pair momP flips
// every stage, so after a whole step the moments of the new f are back in
// momP[cur_mom]); the last stage finalises the bookkeeping.
static int stage_count(const BoltCtx* ctx) { return ctx->p.integrator == BOLT_RK2 ? 2 : 4; }

static void* stage_input(BoltCtx* ctx, void* f, int k) {
    if (k == 0) return f;
    if (ctx->p.integrator == BOLT_RK2) return ctx->buf[0];
    return k == 2 ? ctx->buf[1] : ctx->buf[0];
}

static const char* const kStageNames[4] = {"bolt: RK stage 1", "bolt: RK stage 2",
                                           "bolt: RK stage 3", "bolt: RK stage 4"};

// one NVTX range per RK stage (pushed and popped around run_rk_stage)
struct StageRange {
    explicit StageRange(int k) { nvtxRangePushA(kStageNames[k & 3]); }
    ~StageRange() { nvtxRangePop(); }
};

// whether stage k of the next step advances FDTD fields (RK4: stage 2;
// RK2: the stage entered with the time-level flag at 0)
static int stage_evolves(const BoltCtx* ctx, int k) {
    if (!ctx->p.fields_enabled || ctx->p.fields_type != BOLT_FIELDS_ELECTRODYNAMIC) return 0;
    return ctx->p.integrator == BOLT_RK2 ? !ctx->at_n : k == 1;
}

// parts of stage k: 3 when it advances the fields of a block (Yee ghosts
// exchanged in between), else 1
static int stage_parts(const BoltCtx* ctx, int k) {
    const bool ext = ctx->p.bc_q1 == BOLT_BC_EXTERNAL || ctx->p.bc_q2 == BOLT_BC_EXTERNAL;
    return ext && stage_evolves(ctx, k) ? 3 : 1;
}

// region (see launch_qstage): -1 the whole stage; 0 the q-tiles whose stencils
// stay inside a block along its external axes; 1 the other tiles; 2 the rest
// of the stage (the ghost pass of non-periodic axes, the step's bookkeeping),
// after both.  0-2 need a stage without fields on the paired kernel, no peer
// halos, and (stage 0) the ghosts and moments of f current; otherwise they
// return BOLT_ERR_UNSUPPORTED having launched nothing.
static int run_rk_stage(BoltCtx* ctx, void* f, double dt, int k, cudaStream_t st,
                        int part = -1, int region = -1) {
    StageRange range(k);
    int rc = BOLT_OK;
    if (region >= 0) {
        const bool current = ctx->ghost_owner == f && !ctx->ghost_stale_time &&
                             (!ctx->bgk || ctx->mom_owner == f);
        if (ctx->p.fields_enabled || ctx->peer_on || (k == 0 && !current))
            return BOLT_ERR_UNSUPPORTED;
    }
    // with parts: the bookkeeping happens once, after the last part
    const bool first_part = part <= 0, last_part = part < 0 || part == 2;
    if (k == 0 && first_part) {
        rc = ensure_state(ctx, f, st);
        if (rc) return rc;
    }
    // the stage kernels write periodic images only; any other q1 / q2
    // condition (external axes excepted) needs the ghost pass after the stage
    const int dir = (ctx->p.bc_q1 != BOLT_BC_PERIODIC && ctx->p.bc_q1 != BOLT_BC_EXTERNAL) ||
                    (ctx->p.bc_q2 != BOLT_BC_PERIODIC && ctx->p.bc_q2 != BOLT_BC_EXTERNAL);
    const int fe = ctx->p.fields_enabled;
    const int mo_split = fe ? 1 : ctx->nsplit;     // nsplit of partials written by a stage
    double* m_in = ctx->momP[ctx->cur_mom ^ (k & 1)];
    double* m_out = ctx->momP[ctx->cur_mom ^ (k & 1) ^ 1];
    const int nin = k == 0 ? ctx->cur_nsplit : mo_split;
    StageIO io;
    memset(&io, 0, sizeof(io));
    io.mom_in = m_in;
    io.nsplit_in = nin;
    io.mom_out = ctx->bgk ? m_out : nullptr;
    const int last = k == stage_count(ctx) - 1;
    io.flag = last ? ctx->dflag : nullptr;
    void* out1;
    int ev;
    // a block with peers: the stage also stores its boundary rows (q2) and
    // columns (q1) into the neighbours' copy of out1 (f, buf[0] or buf[1])
    auto peers_of = [&](void* out) {
        io.peer_lo = io.peer_hi = io.peer_left = io.peer_right = nullptr;
        if (!ctx->peer_on) return;
        const int idx = out == f ? 0 : (out == ctx->buf[0] ? 1 : (out == ctx->buf[1] ? 2 : -1));
        if (idx < 0) return;
        if (ctx->peer_on & 1) {
            io.peer_lo = ctx->peer[0][idx];
            io.peer_hi = ctx->peer[1][idx];
        }
        if (ctx->peer_on & 2) {
            io.peer_left = ctx->peer[2][idx];
            io.peer_right = ctx->peer[3][idx];
        }
    };
    if (ctx->p.integrator == BOLT_RK2) {
        // fvm_operator.py:22-33: f_half = f + k1*(dt/2); f = f_initial + k2*dt
        void* A = ctx->buf[0];
        io.fs = k == 0 ? f : A;
        io.base1 = f;
        io.c1 = k == 0 ? dt / 2 : dt;
        io.out1 = out1 = k == 0 ? A : f;
        peers_of(out1);
        ev = fe && !ctx->at_n;
        if (region != 2) rc = run_stage(ctx, io, ev, dt, st, ev ? part : -1, region);
        if (region == 0 || region == 1) return rc;
        if (fe && last_part) ctx->at_n ^= 1;
    } else {
        // classic RK4 (integrators.py:15-28) in accumulator form:
        //   f1 = f + (dt/2) k1, acc = f + (dt/6) k1
        //   f2 = f + (dt/2) k2, acc += (dt/3) k2
        //   f3 = f + dt k3,     acc += (dt/3) k3
        //   f  = acc + (dt/6) k4
        // fields (if any) advance once per step, in stage 2
        void* A = ctx->buf[0];
        void* B = ctx->buf[1];
        void* C = ctx->buf[2];
        const double c_half = 0.5 * dt, c_six = dt / 6.0, c_three = dt / 3.0;
        struct S {
            const void* fs; const void* b1; double c1; void* o1; const void* b2; double c2;
            void* o2; int ev;
        } stages[4] = {
            {f, f, c_half, A, f, c_six, C, 0},
            {A, f, c_half, B, C, c_three, C, 1},
            {B, f, dt, A, C, c_three, C, 0},
            {A, C, c_six, f, nullptr, 0.0, nullptr, 0},
        };
        io.fs = stages[k].fs; io.base1 = stages[k].b1; io.c1 = stages[k].c1;
        io.out1 = out1 = stages[k].o1; io.base2 = stages[k].b2; io.c2 = stages[k].c2;
        io.out2 = stages[k].o2;
        peers_of(out1);
        if (region != 2)
            rc = run_stage(ctx, io, fe && stages[k].ev, dt, st, fe && stages[k].ev ? part : -1,
                           region);
        if (region == 0 || region == 1) return rc;
    }
    if (!last_part) return rc;
    if (!rc && dir) rc = launch_ghosts(ctx, out1, st);
    if (rc) return rc;
    if (last) {
        ctx->cur_nsplit = mo_split;
        ctx->ghost_owner = f;
        ctx->mom_owner = ctx->bgk ? f : nullptr;
    }
    return BOLT_OK;
}

static int step_once(BoltCtx* ctx, void* f, double dt, cudaStream_t st) {
    for (int k = 0; k < stage_count(ctx); ++k) {
        const int rc = run_rk_stage(ctx, f, dt, k, st);
        if (rc) return rc;
    }
    return BOLT_OK;
}

extern "C" {

int bolt_fill_ghosts(BoltCtx* ctx, void* f_dev, void* stream) {
    if (!ctx || !f_dev) return BOLT_ERR_ARG;
    int rc = launch_ghosts(ctx, f_dev, (cudaStream_t)stream);
    if (rc) return rc;
    ctx->ghost_owner = f_dev;
    ctx->mom_owner = nullptr;
    ctx->ghost_stale_time = 0;
    return BOLT_OK;
}

// ---- advective semi-Lagrangian step in q (asl_operators.py:20-83) ----------
// op_advect_q from f_in into out's interior (out != f_in)
static int asl_advect(BoltCtx* ctx, void* f_in, void* out, double dt, cudaStream_t st) {
    const BoltGrid& g = ctx->g;
    if ((ctx->p.fields_enabled && !electrostatic(ctx)) || g.N_ghost < 2)
        return BOLT_ERR_UNSUPPORTED;
    // op_advect_q: communicate_f + apply_bcs_f, then the interpolation
    int rc = launch_ghosts(ctx, f_in, st);
    if (rc) return rc;
    AslArgs a;
    memset(&a, 0, sizeof(a));
    a.f = f_in;
    a.out = out;
    a.dt = dt;
    a.q1_start = g.q1_start;
    a.q2_start = g.q2_start;
    a.dq1 = g.dq1;
    a.dq2 = g.dq2;
    a.Nq1 = g.N_q1; a.Nq2 = g.N_q2; a.Ng = g.N_ghost; a.Ns = g.N_s;
    a.Np1 = g.N_p1; a.Np2 = g.N_p2; a.Np3 = g.N_p3; a.Np = ctx->Np;
    a.sg = ctx->sg;
    // a non-finite interpolated value raises the divergence flag
    cudaError_t e = ctx->elem == 8 ? launch_asl_q_f64(a, ctx->dflag, st)
                                   : launch_asl_q_f32(a, ctx->dflag, st);
    ctx->launches++;
    CK(e);
    ctx->ghost_owner = nullptr;
    ctx->mom_owner = nullptr;
    return BOLT_OK;
}

int bolt_asl_advect_q(BoltCtx* ctx, void* f_dev, double dt, void* stream) {
    if (!ctx || !f_dev) return BOLT_ERR_ARG;
    const BoltGrid& g = ctx->g;
    cudaStream_t st = (cudaStream_t)stream;
    int rc = asl_advect(ctx, f_dev, ctx->buf[0], dt, st);
    if (rc) return rc;
    // the interpolated interior back into f: the interior q2 rows as one
    // contiguous copy (a 2-D copy of the interior cells alone ran at a third
    // of the bandwidth); it carries the work buffer's stale q1 ghost cells
    // into f's, which are stale until the next refresh in any case
    const size_t row = (size_t)g.N_s * ctx->Np * ctx->elem;
    const size_t pitch = row * ctx->Nq1g;
    const size_t off = (size_t)g.N_ghost * pitch;
    CK(cudaMemcpyAsync(static_cast<char*>(f_dev) + off,
                       static_cast<const char*>(ctx->buf[0]) + off, pitch * g.N_q2,
                       cudaMemcpyDeviceToDevice, st));
    ctx->ghost_owner = nullptr;
    ctx->mom_owner = nullptr;
    return BOLT_OK;
}

int bolt_fvm_p_step(BoltCtx* ctx, void* f_dev, double dt, void* stream) {
    if (!ctx || !f_dev) return BOLT_ERR_ARG;
    if (!electrostatic(ctx)) return BOLT_ERR_UNSUPPORTED;
    ctx->p_only = 1;
    const int rc = step_once(ctx, f_dev, dt, (cudaStream_t)stream);
    ctx->p_only = 0;
    return rc;
}

int bolt_asl_advect_q_to(BoltCtx* ctx, void* f_in, void* out, double dt, void* stream) {
    if (!ctx || !f_in || !out || out == f_in) return BOLT_ERR_ARG;
    return asl_advect(ctx, f_in, out, dt, (cudaStream_t)stream);
}

// op_solve_src from f_in into out's interior; scratch (!= f_in, may be out)
// holds the RK2 half step
static int asl_source(BoltCtx* ctx, const void* f_in, void* out, void* scratch, double dt,
                      int instantaneous, cudaStream_t st) {
    const BoltGrid& g = ctx->g;
    if ((ctx->p.fields_enabled && !electrostatic(ctx)) || !ctx->bgk || ctx->tau_arr ||
        ctx->ntab > 768)
        return BOLT_ERR_UNSUPPORTED;
    QStageArgs a;
    memset(&a, 0, sizeof(a));
    a.Nq1 = g.N_q1; a.Nq2 = g.N_q2; a.Ng = g.N_ghost; a.Ns = g.N_s;
    a.Np1 = g.N_p1; a.Np2 = g.N_p2; a.Np3 = g.N_p3; a.Np = ctx->Np;
    a.Nq1g = ctx->Nq1g; a.Nq2g = ctx->Nq2g;
    a.sg = ctx->sg;
    a.kB = ctx->p.boltzmann_constant;
    a.p_dim = ctx->p.p_dim;
    a.tau = ctx->p.tau;
    a.nsplit_in = 1;
    // one source evaluation; the moments of `in` come from a moment pass
    // (mom_in null) or from the previous evaluation, which wrote them with
    // its output (mom_out)
    auto src = [&](const void* in, const void* base, void* dst, double c, int mode,
                   double* mom_in, double* mom_out) {
        if (!mom_in) {
            int r = launch_moments5(ctx, in, ctx->momP[0], st);
            if (r) return r;
            mom_in = ctx->momP[0];
        }
        a.mom_in = mom_in;
        cudaError_t e = ctx->elem == 8
            ? launch_asl_src_f64(a, in, base, dst, c, mode, ctx->dflag, mom_out, st)
            : launch_asl_src_f32(a, in, base, dst, c, mode, ctx->dflag, mom_out, st);
        ctx->launches++;
        CK(e);
        return BOLT_OK;
    };
    int rc;
    if (instantaneous) {
        // f <- f_MB (asl_operators.py:56-64, collision_operator.py:126-128)
        rc = src(f_in, f_in, out, 0.0, 1, nullptr, nullptr);
    } else {
        // integrators.RK2: f_half = f + S(f) dt/2; f = f + S(f_half) dt
        // (each element of the second evaluation reads f_half and f, then
        // writes out, in one thread: out may be either of them)
        rc = src(f_in, f_in, scratch, 0.5 * dt, 0, nullptr, ctx->momP[1]);
        if (!rc) rc = src(scratch, f_in, out, dt, 0, ctx->momP[1], nullptr);
    }
    // the written interiors changed: ghost cells and cached moments are stale
    ctx->ghost_owner = nullptr;
    ctx->mom_owner = nullptr;
    return rc;
}

int bolt_asl_source(BoltCtx* ctx, void* f_dev, double dt, int instantaneous, void* stream) {
    if (!ctx || !f_dev) return BOLT_ERR_ARG;
    return asl_source(ctx, f_dev, f_dev, ctx->buf[0], dt, instantaneous, (cudaStream_t)stream);
}

int bolt_asl_source_to(BoltCtx* ctx, const void* f_in, void* out, void* scratch, double dt,
                       int instantaneous, void* stream) {
    if (!ctx || !f_in || !out || (!instantaneous && (!scratch || scratch == f_in)))
        return BOLT_ERR_ARG;
    return asl_source(ctx, f_in, out, scratch, dt, instantaneous, (cudaStream_t)stream);
}

int bolt_work_buffer(BoltCtx* ctx, int i, void** ptr) {
    if (!ctx || !ptr || i < 0 || i >= 3 || !ctx->buf[i]) return BOLT_ERR_ARG;
    *ptr = ctx->buf[i];
    return BOLT_OK;
}

int bolt_set_shear(BoltCtx* ctx, double q, double omega) {
    if (!ctx) return BOLT_ERR_ARG;
    ctx->shear_q = q;
    ctx->shear_omega = omega;
    ctx->ghost_stale_time = 1;
    return BOLT_OK;
}

int bolt_set_p_space_grid(BoltCtx* ctx, int grid, double initial_mu) {
    if (!ctx || (grid != BOLT_PGRID_CARTESIAN && grid != BOLT_PGRID_POLAR2D)) return BOLT_ERR_ARG;
    if (grid == BOLT_PGRID_POLAR2D) {
        if (!(initial_mu == initial_mu)) return BOLT_ERR_ARG;
        // a q1 mirror edge splits the angle axis into two halves
        if ((ctx->p.bc_q1 == BOLT_BC_MIRROR || ctx->p.bc_q1 == BOLT_BC_MIRROR_DIRICHLET) &&
            ctx->g.N_p2 % 2)
            return BOLT_ERR_UNSUPPORTED;
    }
    ctx->sg.polar2d = grid == BOLT_PGRID_POLAR2D ? 1 : 0;
    ctx->sg.mom_scale = grid == BOLT_PGRID_POLAR2D ? initial_mu : 0.0;
    return BOLT_OK;
}

int bolt_set_time(BoltCtx* ctx, double t) {
    if (!ctx) return BOLT_ERR_ARG;
    const bool shearing = ctx->p.bc_q1 == BOLT_BC_SHEARING_BOX ||
                          ctx->p.bc_q2 == BOLT_BC_SHEARING_BOX;
    if (shearing && t != ctx->time) ctx->ghost_stale_time = 1;
    ctx->time = t;
    return BOLT_OK;
}

int bolt_invalidate(BoltCtx* ctx) {
    if (!ctx) return BOLT_ERR_ARG;
    ctx->ghost_owner = nullptr;
    ctx->mom_owner = nullptr;
    return BOLT_OK;
}

int bolt_step(BoltCtx* ctx, void* f_dev, double dt, void* stream) {
    if (!ctx || !f_dev) return BOLT_ERR_ARG;
    return step_once(ctx, f_dev, dt, (cudaStream_t)stream);
}

int bolt_stage_count(BoltCtx* ctx) { return ctx ? stage_count(ctx) : -1; }

void* bolt_stage_input(BoltCtx* ctx, void* f_dev, int k) {
    if (!ctx || k < 0 || k >= stage_count(ctx)) return nullptr;
    return stage_input(ctx, f_dev, k);
}

int bolt_stage(BoltCtx* ctx, void* f_dev, double dt, int k, void* stream) {
    if (!ctx || !f_dev || k < 0 || k >= stage_count(ctx)) return BOLT_ERR_ARG;
    return run_rk_stage(ctx, f_dev, dt, k, (cudaStream_t)stream);
}

int bolt_stage_region(BoltCtx* ctx, void* f_dev, double dt, int k, int region, void* stream) {
    if (!ctx || !f_dev || k < 0 || k >= stage_count(ctx) || region < 0 || region > 2)
        return BOLT_ERR_ARG;
    return run_rk_stage(ctx, f_dev, dt, k, (cudaStream_t)stream, -1, region);
}

int bolt_stage_parts(BoltCtx* ctx, int k) {
    if (!ctx || k < 0 || k >= stage_count(ctx)) return -1;
    return stage_parts(ctx, k);
}

int bolt_stage_part(BoltCtx* ctx, void* f_dev, double dt, int k, int part, void* stream) {
    if (!ctx || !f_dev || k < 0 || k >= stage_count(ctx)) return BOLT_ERR_ARG;
    const int n = stage_parts(ctx, k);
    if (part < 0 || part >= n) return BOLT_ERR_ARG;
    return run_rk_stage(ctx, f_dev, dt, k, (cudaStream_t)stream, n == 1 ? -1 : part);
}

double* bolt_fields_yee(BoltCtx* ctx) { return ctx ? ctx->yee : nullptr; }

int bolt_run(BoltCtx* ctx, void* f_dev, double dt, int n_steps, void* stream) {
    if (!ctx || !f_dev || n_steps < 0) return BOLT_ERR_ARG;
    for (int i = 0; i < n_steps; ++i) {
        int rc = step_once(ctx, f_dev, dt, (cudaStream_t)stream);
        if (rc) return rc;
    }
    return BOLT_OK;
}

static int dfdt_impl(BoltCtx* ctx, const void* f_dev, void* dfdt_dev, int evolve_fields,
                     double dt, int term, cudaStream_t st);

int bolt_dfdt(BoltCtx* ctx, const void* f_dev, void* dfdt_dev, int evolve_fields, double dt,
              void* stream) {
    if (!ctx || !f_dev || !dfdt_dev) return BOLT_ERR_ARG;
    return dfdt_impl(ctx, f_dev, dfdt_dev, evolve_fields, dt, 0, (cudaStream_t)stream);
}

int bolt_dfdt_term(BoltCtx* ctx, const void* f_dev, void* out_dev, int term, int evolve_fields,
                   double dt, void* stream) {
    if (!ctx || !f_dev || !out_dev || term < 1 || term > 3) return BOLT_ERR_ARG;
    if (!ctx->p.fields_enabled) return BOLT_ERR_UNSUPPORTED;
    return dfdt_impl(ctx, f_dev, out_dev, evolve_fields, dt, term, (cudaStream_t)stream);
}

}  // extern "C"

// df/dt of f (term 0) or, with fields, one p-flux divergence (term 1..3)
// after the same field evaluation df_dt_fvm performs
static int dfdt_impl(BoltCtx* ctx, const void* f_dev, void* dfdt_dev, int evolve_fields,
                     double dt, int term, cudaStream_t st) {
    int rc = BOLT_OK;
    double* m = ctx->momP[ctx->cur_mom ^ 1];
    if (ctx->bgk) rc = launch_moments5(ctx, f_dev, m, st);
    if (rc) return rc;
    StageIO io;
    memset(&io, 0, sizeof(io));
    io.fs = f_dev;
    io.mom_in = m;
    io.nsplit_in = 1;
    if (!ctx->p.fields_enabled) {
        io.out1 = dfdt_dev;
        return launch_qstage(ctx, io, 1, 0, st);
    }
    if (electrostatic(ctx)) {
        rc = launch_electrostatic(ctx, f_dev, st);
        evolve_fields = 0;
    }
    if (rc) return rc;
    StageIO qio = io;
    qio.out1 = ctx->kbuf;
    rc = launch_qstage(ctx, qio, 1, evolve_fields, st);
    if (!rc && evolve_fields) rc = launch_fields(ctx, dt, ctx->nsplit, st);
    if (!rc) {
        io.out1 = dfdt_dev;
        rc = launch_pstage(ctx, io, ctx->kbuf, st, term);
    }
    return rc;
}

extern "C" {

int bolt_moments(BoltCtx* ctx, const void* f_dev, int moment_id, double* out_dev,
                 void* stream) {
    if (!ctx || !f_dev || !out_dev || moment_id < 0 || moment_id > 10) return BOLT_ERR_ARG;
    const BoltGrid& g = ctx->g;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = ctx->elem == 8
        ? launch_moment_f64(f_dev, moment_id, out_dev, g.N_s, g.N_p1, g.N_p2, g.N_p3, ctx->Nq1g,
                            ctx->Nq2g, ctx->sg, st)
        : launch_moment_f32(f_dev, moment_id, out_dev, g.N_s, g.N_p1, g.N_p2, g.N_p3, ctx->Nq1g,
                            ctx->Nq2g, ctx->sg, st);
    ctx->launches++;
    CK(e);
    return BOLT_OK;
}

int bolt_fields_set(BoltCtx* ctx, const double* cell_dev, const double* yee_dev, void* stream) {
    if (!ctx || !ctx->p.fields_enabled) return BOLT_ERR_ARG;
    const size_t bytes = 6 * (size_t)ctx->Nq1g * ctx->Nq2g * sizeof(double);
    cudaStream_t st = (cudaStream_t)stream;
    if (cell_dev) CK(cudaMemcpyAsync(ctx->cell, cell_dev, bytes, cudaMemcpyDeviceToDevice, st));
    if (yee_dev) CK(cudaMemcpyAsync(ctx->yee, yee_dev, bytes, cudaMemcpyDeviceToDevice, st));
    return BOLT_OK;
}

int bolt_fields_get(BoltCtx* ctx, double* cell_dev, double* yee_dev, void* stream) {
    if (!ctx || !ctx->p.fields_enabled) return BOLT_ERR_ARG;
    const size_t bytes = 6 * (size_t)ctx->Nq1g * ctx->Nq2g * sizeof(double);
    cudaStream_t st = (cudaStream_t)stream;
    if (cell_dev) CK(cudaMemcpyAsync(cell_dev, ctx->cell, bytes, cudaMemcpyDeviceToDevice, st));
    if (yee_dev) CK(cudaMemcpyAsync(yee_dev, ctx->yee, bytes, cudaMemcpyDeviceToDevice, st));
    return BOLT_OK;
}

int bolt_fields_evolve(BoltCtx* ctx, const double* J_dev, double dt, void* stream) {
    if (!ctx || !J_dev || !ctx->p.fields_enabled ||
        ctx->p.fields_type != BOLT_FIELDS_ELECTRODYNAMIC)
        return BOLT_ERR_ARG;
    return launch_fields(ctx, dt, 0, (cudaStream_t)stream, J_dev);
}

int bolt_get_at_n(BoltCtx* ctx) { return ctx ? ctx->at_n : -1; }

int bolt_set_at_n(BoltCtx* ctx, int at_n) {
    if (!ctx) return BOLT_ERR_ARG;
    ctx->at_n = at_n ? 1 : 0;
    return BOLT_OK;
}

}  // extern "C"
