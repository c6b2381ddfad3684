// bolt_batch.cu - C ABI of the ragged batch of independent 1D1V runs
// (include/bolt_b200.h, "Ragged batch").
//
// Packing: run r's ghosted f (N_q1 + 6 rows of N_p1 FP32 values, periodic q1)
// starts at an element offset that is a multiple of 32 (128 bytes) in each of
// the four f-sized buffers (f, RK4 stage buffers A, B and the accumulator C);
// FP64 moment sums are packed by q-cell, [cell][5].  Work items (run, q-tile)
// are consumed by persistent CTAs through an atomic queue that a memset node
// resets before every stage.  The schedule -- q-cells per tile (8, 16, 32 or 64:
// CTAs of 2, 4, 8 or 16 warps), CTAs per SM and the queue order (decreasing cost
// = cells x p-chunks, or run by run) -- is set by bolt_batch_set_schedule; the
// batch's autotuner (bolt_b200.batch) times the candidates on the batch
// itself.  bolt_batch_run captures nsteps RK4 steps of all runs (4 stage
// launches each) into one CUDA graph on the batch's own stream and launches
// it on the caller's stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/bolt_b200.h"
#include "batch_kernels.cuh"

using namespace bolt;

struct BoltBatch {
    int nruns;
    int source;
    std::vector<BatchRunDev> runs;
    BatchRunDev* d_runs;
    int2* d_items;
    int nitems;
    size_t fcount;          // elements of one packed f buffer
    int nq_total;           // q-cells of all runs
    float* buf[4];          // f, A, B, C
    double* mom[2];         // moment sums: [0] of f (and of B), [1] of A
    int* counters;          // one work-queue head per stage of a step
    int* hflag;             // non-finite flag, host-mapped
    int* dflag;
    int nctas;
    int tile_warps;         // schedule: warps per CTA (4 q-cells each)
    int ctas_per_sm;        //           persistent CTAs per SM (clamped to occupancy)
    int lpt;                //           1: items by decreasing cost, 0: run by run
    int sms;
    cudaStream_t cap;       // capture stream
    cudaGraphExec_t exec;
    int exec_steps;
    int prepared;           // ghosts filled and moments of f current
};

namespace {

int batch_ck(cudaError_t e) { return e == cudaSuccess ? BOLT_OK : BOLT_ERR_CUDA; }

template <int NW>
int stage_occupancy() {
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_stage_kernel<NW>, NW * 32, 0);
    return std::max(1, per_sm);
}

int occupancy(int tile_warps) {
    switch (tile_warps) {
        case 2: return stage_occupancy<2>();
        case 4: return stage_occupancy<4>();
        case 8: return stage_occupancy<8>();
        default: return stage_occupancy<16>();
    }
}

// work items of the current schedule -> d_items, nitems, nctas (drops the
// captured graph: its launches carry the old grid and item list)
int build_schedule(BoltBatch* b) {
    const int tq = b->tile_warps * kBatchCellsPerWarp;
    std::vector<int2> items;
    std::vector<long long> cost;
    for (int r = 0; r < b->nruns; ++r) {
        const BatchRunDev& R = b->runs[r];
        for (int t = 0; t * tq < R.Nq1; ++t) {
            items.push_back(make_int2(r, t));
            cost.push_back((long long)std::min(tq, R.Nq1 - t * tq) * (R.Np1 / PW));
        }
    }
    std::vector<int> order(items.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    if (b->lpt)
        std::stable_sort(order.begin(), order.end(),
                         [&](int x, int y) { return cost[x] > cost[y]; });
    std::vector<int2> sorted(items.size());
    for (size_t i = 0; i < order.size(); ++i) sorted[i] = items[order[i]];
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
        b->exec_steps = 0;
    }
    if ((int)sorted.size() != b->nitems || !b->d_items) {
        cudaFree(b->d_items);
        b->d_items = nullptr;
        if (cudaMalloc((void**)&b->d_items, sorted.size() * sizeof(int2)) != cudaSuccess)
            return BOLT_ERR_NOMEM;
    }
    b->nitems = (int)sorted.size();
    int rc = batch_ck(cudaMemcpy(b->d_items, sorted.data(), sorted.size() * sizeof(int2),
                                 cudaMemcpyHostToDevice));
    const int per_sm = std::min(b->ctas_per_sm, occupancy(b->tile_warps));
    b->nctas = std::max(1, std::min(b->nitems, b->sms * per_sm));
    return rc;
}

void launch_stage(const BoltBatch* b, const BatchStageArgs& a, cudaStream_t st) {
    switch (b->tile_warps) {
        case 2: batch_stage_kernel<2><<<b->nctas, 2 * 32, 0, st>>>(a); break;
        case 4: batch_stage_kernel<4><<<b->nctas, 4 * 32, 0, st>>>(a); break;
        case 8: batch_stage_kernel<8><<<b->nctas, 8 * 32, 0, st>>>(a); break;
        default: batch_stage_kernel<16><<<b->nctas, 16 * 32, 0, st>>>(a); break;
    }
}

void launch_moments(const BoltBatch* b, cudaStream_t st) {
    switch (b->tile_warps) {
        case 2:
            batch_moments_kernel<2><<<b->nctas, 2 * 32, 0, st>>>(
                b->d_runs, b->d_items, b->nitems, b->counters, b->buf[0], b->mom[0]);
            break;
        case 4:
            batch_moments_kernel<4><<<b->nctas, 4 * 32, 0, st>>>(
                b->d_runs, b->d_items, b->nitems, b->counters, b->buf[0], b->mom[0]);
            break;
        case 8:
            batch_moments_kernel<8><<<b->nctas, 8 * 32, 0, st>>>(
                b->d_runs, b->d_items, b->nitems, b->counters, b->buf[0], b->mom[0]);
            break;
        default:
            batch_moments_kernel<16><<<b->nctas, 16 * 32, 0, st>>>(
                b->d_runs, b->d_items, b->nitems, b->counters, b->buf[0], b->mom[0]);
            break;
    }
}

void batch_free(BoltBatch* b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->cap) cudaStreamDestroy(b->cap);
    for (int i = 0; i < 4; ++i) cudaFree(b->buf[i]);
    cudaFree(b->mom[0]);
    cudaFree(b->mom[1]);
    cudaFree(b->counters);
    cudaFree(b->d_runs);
    cudaFree(b->d_items);
    if (b->hflag) cudaFreeHost(b->hflag);
    delete b;
}

// one RK4 step of every run: the stage sequence of bolt_capi.cu's RK4
// (A = f + dt/2 k(f), C = f + dt/6 k(f); B = f + dt/2 k(A), C += dt/3 k(A);
//  A = f + dt k(B), C += dt/3 k(B); f = C + dt/6 k(A))
int enqueue_step(BoltBatch* b, cudaStream_t st) {
    float *f = b->buf[0], *A = b->buf[1], *B = b->buf[2], *C = b->buf[3];
    struct S { const float *fs, *b1, *b2; float *o1, *o2; double a1, a2; int mi, mo; };
    const S stages[4] = {
        {f, f, f, A, C, 0.5, 1.0 / 6.0, 0, 1},
        {A, f, C, B, C, 0.5, 1.0 / 3.0, 1, 0},
        {B, f, C, A, C, 1.0, 1.0 / 3.0, 0, 1},
        {A, C, nullptr, f, nullptr, 1.0 / 6.0, 0.0, 1, 0},
    };
    for (int s = 0; s < 4; ++s) {
        if (cudaMemsetAsync(b->counters + s, 0, sizeof(int), st) != cudaSuccess)
            return BOLT_ERR_CUDA;
        BatchStageArgs a;
        a.runs = b->d_runs;
        a.items = b->d_items;
        a.nitems = b->nitems;
        a.counter = b->counters + s;
        a.fs = stages[s].fs;
        a.base1 = stages[s].b1;
        a.base2 = stages[s].b2;
        a.out1 = stages[s].o1;
        a.out2 = stages[s].o2;
        a.mom_in = b->mom[stages[s].mi];
        a.mom_out = b->mom[stages[s].mo];
        a.flag = b->dflag;
        a.a1 = stages[s].a1;
        a.a2 = stages[s].a2;
        a.source = b->source;
        launch_stage(b, a, st);
        if (cudaGetLastError() != cudaSuccess) return BOLT_ERR_CUDA;
    }
    return BOLT_OK;
}

}  // namespace

extern "C" {

int bolt_batch_create(const BoltBatchRun* runs, int nruns, int source_enabled, BoltBatch** out) {
    if (!runs || nruns <= 0 || !out) return BOLT_ERR_ARG;
    *out = nullptr;
    for (int r = 0; r < nruns; ++r) {
        const BoltBatchRun& R = runs[r];
        if (R.N_q1 < 2 * kBatchNg || R.N_q1 % 4 != 0 || R.N_p1 <= 0 || R.N_p1 % PW != 0)
            return BOLT_ERR_UNSUPPORTED;
        if (!(R.q1_end > R.q1_start) || !(R.p1_end > R.p1_start) || !(R.dp2 > 0) ||
            !(R.dp3 > 0) || !(R.mass > 0) || !(R.boltzmann_constant > 0) || !(R.dt > 0) ||
            (source_enabled && !(R.tau > 0)))
            return BOLT_ERR_ARG;
    }
    BoltBatch* b = new (std::nothrow) BoltBatch();
    if (!b) return BOLT_ERR_NOMEM;
    b->nruns = nruns;
    b->source = source_enabled ? 1 : 0;
    b->runs.resize(nruns);
    long long off = 0;
    int qoff = 0;
    for (int r = 0; r < nruns; ++r) {
        const BoltBatchRun& R = runs[r];
        BatchRunDev& D = b->runs[r];
        D.f_off = off;
        D.mom_off = qoff;
        D.Nq1 = R.N_q1;
        D.Np1 = R.N_p1;
        D.dp1 = (R.p1_end - R.p1_start) / R.N_p1;
        D.p1_start = R.p1_start;
        D.v2c = R.p2_center;
        D.v3c = R.p3_center;
        D.measure = (R.dp3 * R.dp2) * D.dp1;
        D.mass = R.mass;
        D.kB = R.boltzmann_constant;
        D.dt = R.dt;
        D.inv_dq1 = 1.0 / ((R.q1_end - R.q1_start) / R.N_q1);
        D.inv_tau = source_enabled ? 1.0 / R.tau : 0.0;
        off += ((long long)(R.N_q1 + 2 * kBatchNg) * R.N_p1 + 31) / 32 * 32;
        qoff += R.N_q1;
    }
    b->fcount = (size_t)off;
    b->nq_total = qoff;
    // default schedule: 32-cell tiles, as many CTAs as fit, longest items first
    b->tile_warps = 8;
    b->ctas_per_sm = 64;
    b->lpt = 1;

    int rc = BOLT_OK;
    auto alloc = [&](void** p, size_t bytes) {
        if (rc == BOLT_OK && cudaMalloc(p, bytes) != cudaSuccess) rc = BOLT_ERR_NOMEM;
    };
    for (int i = 0; i < 4; ++i) alloc((void**)&b->buf[i], b->fcount * sizeof(float));
    alloc((void**)&b->mom[0], (size_t)qoff * kNumMom * sizeof(double));
    alloc((void**)&b->mom[1], (size_t)qoff * kNumMom * sizeof(double));
    alloc((void**)&b->counters, 4 * sizeof(int));
    alloc((void**)&b->d_runs, nruns * sizeof(BatchRunDev));
    if (rc == BOLT_OK && cudaHostAlloc((void**)&b->hflag, sizeof(int), cudaHostAllocMapped) !=
                             cudaSuccess)
        rc = BOLT_ERR_NOMEM;
    if (rc == BOLT_OK) {
        *b->hflag = 0;
        rc = batch_ck(cudaHostGetDevicePointer((void**)&b->dflag, b->hflag, 0));
    }
    if (rc == BOLT_OK)
        rc = batch_ck(cudaMemcpy(b->d_runs, b->runs.data(), nruns * sizeof(BatchRunDev),
                                 cudaMemcpyHostToDevice));
    for (int i = 0; i < 4 && rc == BOLT_OK; ++i)
        rc = batch_ck(cudaMemset(b->buf[i], 0, b->fcount * sizeof(float)));
    if (rc == BOLT_OK) rc = batch_ck(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
    if (rc == BOLT_OK) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        b->sms = sms;
        rc = build_schedule(b);
    }
    if (rc != BOLT_OK) {
        batch_free(b);
        return rc;
    }
    *out = b;
    return BOLT_OK;
}

void bolt_batch_destroy(BoltBatch* b) { batch_free(b); }

void* bolt_batch_f(BoltBatch* b) { return b ? b->buf[0] : nullptr; }

long long bolt_batch_f_count(const BoltBatch* b) { return b ? (long long)b->fcount : -1; }

long long bolt_batch_f_offset(const BoltBatch* b, int run) {
    if (!b || run < 0 || run >= b->nruns) return -1;
    return b->runs[run].f_off;
}

int bolt_batch_q_offset(const BoltBatch* b, int run) {
    if (!b || run < 0 || run >= b->nruns) return -1;
    return b->runs[run].mom_off;
}

int bolt_batch_q_count(const BoltBatch* b) { return b ? b->nq_total : -1; }

int bolt_batch_prepare(BoltBatch* b, void* stream) {
    if (!b) return BOLT_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    dim3 g(8, b->nruns);
    batch_ghost_kernel<<<g, 256, 0, st>>>(b->d_runs, b->nruns, b->buf[0]);
    if (cudaGetLastError() != cudaSuccess) return BOLT_ERR_CUDA;
    if (cudaMemsetAsync(b->counters, 0, sizeof(int), st) != cudaSuccess) return BOLT_ERR_CUDA;
    launch_moments(b, st);
    if (cudaGetLastError() != cudaSuccess) return BOLT_ERR_CUDA;
    b->prepared = 1;
    return BOLT_OK;
}

int bolt_batch_set_schedule(BoltBatch* b, int tile_cells, int ctas_per_sm, int lpt_order) {
    if (!b || ctas_per_sm < 1) return BOLT_ERR_ARG;
    if (tile_cells != 8 && tile_cells != 16 && tile_cells != 32 && tile_cells != 64)
        return BOLT_ERR_ARG;
    if (cudaDeviceSynchronize() != cudaSuccess) return BOLT_ERR_CUDA;  // no launch uses the items
    b->tile_warps = tile_cells / kBatchCellsPerWarp;
    b->ctas_per_sm = ctas_per_sm;
    b->lpt = lpt_order ? 1 : 0;
    return build_schedule(b);
}

int bolt_batch_get_schedule(const BoltBatch* b, int* tile_cells, int* ctas, int* lpt_order) {
    if (!b) return BOLT_ERR_ARG;
    if (tile_cells) *tile_cells = b->tile_warps * kBatchCellsPerWarp;
    if (ctas) *ctas = b->nctas;
    if (lpt_order) *lpt_order = b->lpt;
    return BOLT_OK;
}

int bolt_batch_run(BoltBatch* b, int nsteps, void* stream) {
    if (!b || nsteps < 0) return BOLT_ERR_ARG;
    if (!b->prepared) return BOLT_ERR_ARG;
    if (nsteps == 0) return BOLT_OK;
    if (!b->exec || b->exec_steps != nsteps) {
        if (b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
        }
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return BOLT_ERR_CUDA;
        int rc = BOLT_OK;
        for (int s = 0; s < nsteps && rc == BOLT_OK; ++s) rc = enqueue_step(b, b->cap);
        cudaError_t e = cudaStreamEndCapture(b->cap, &g);
        if (rc != BOLT_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return BOLT_ERR_CUDA;
        }
        e = cudaGraphInstantiate(&b->exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            b->exec = nullptr;
            return BOLT_ERR_CUDA;
        }
        b->exec_steps = nsteps;
    }
    return batch_ck(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
}

int bolt_batch_moments(BoltBatch* b, double* out_dev, void* stream) {
    if (!b || !out_dev || !b->prepared) return BOLT_ERR_ARG;
    return batch_ck(cudaMemcpyAsync(out_dev, b->mom[0],
                                    (size_t)b->nq_total * kNumMom * sizeof(double),
                                    cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
}

int bolt_batch_divergence_flag(BoltBatch* b) {
    if (!b) return -1;
    const int v = *(volatile int*)b->hflag;
    *(volatile int*)b->hflag = 0;
    return v;
}

}  // extern "C"
