// bolt_adjoint.cu - C ABI of the 1D1V RK4 forward step and its hand-written
// adjoint (include/bolt_b200.h, "Adjoint"), FP32 or FP64.
//
// Adjoint of one RK4 step f' = f + dt/6 (k1 + 2k2 + 2k3 + k4), given the
// adjoint lam of f': recompute k1..k4 from f, then with g_s = L'(stage s)^T a_s
//   a4 = dt/6 lam                 g4 at f + dt k3
//   a3 = dt/3 lam + dt g4         g3 at f + dt/2 k2
//   a2 = dt/3 lam + dt/2 g3       g2 at f + dt/2 k1
//   a1 = dt/6 lam + dt/2 g2       g1 at f
//   lam <- lam + g1 + g2 + g3 + g4,  dJ/dtau += sum_s <a_s, dL/dtau(stage s)>
// The objective J = sum_{n >= 1} dt |nhat_1(f_n)|^2 adds dt d|nhat_1|^2/df to
// lam at every step boundary it sees.
#include <cuda_runtime.h>

#include <cstdlib>
#include <new>

#include "../../include/bolt_b200.h"
#include "adjoint_kernels.cuh"

using namespace bolt;

struct BoltAdj1D {
    int dtype;
    int recon;               // kAdjWeno5 or kAdjMinmod
    Adj1DArgs P;
    double dt;
    long long n;             // N_q1 * N_p1
    void* k[4];
    void* a;
    void* gacc;              // running lam + sum g
    void* gs;                // one stage's g (the second stage adjoint field of the
                             // cooperative step)
    double* dtau_part;       // [4][N_q1]
    double* dens;            // [N_q1]
    double* reim;            // [3]
    int coop_grid;           // CTAs of the cooperative whole-step launches (0: separate launches)
};

namespace {

template <typename T>
__global__ void adj_axpby_kernel(long long n, T* out, T alpha, const T* x, T beta, const T* y) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x)
        out[e] = y ? alpha * x[e] + beta * y[e] : alpha * x[e];
}

__global__ void adj_sum_kernel(const double* part, int n, double* acc) {
    __shared__ double red[kAdjThreads / 32];
    double s = 0;
    for (int i = threadIdx.x; i < n; i += kAdjThreads) s += part[i];
    s = adj_block_sum(s, red);
    if (threadIdx.x == 0) *acc += s;
}

int ew_blocks(long long n) {
    long long b = (n + 255) / 256;
    return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

// CTAs the cooperative step kernels may use (every one co-resident), or 0
// when the device has no cooperative launch
template <typename T, int R>
int coop_grid_for(int Nq1) {
    int dev = 0, coop = 0, sms = 0, per_a = 0, per_b = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (!coop || sms <= 0) return 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_a, adj_step_coop_kernel<T, R>,
                                                  kAdjThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_b, adj_step_adjoint_coop_kernel<T, R>,
                                                  kAdjThreads, 0);
    const int per = per_a < per_b ? per_a : per_b;
    if (per <= 0) return 0;
    return Nq1 < sms * per ? Nq1 : sms * per;
}

template <typename T, int R>
int step_coop(BoltAdj1D* c, T* f, double* J, cudaStream_t st) {
    Adj1DArgs P = c->P;
    T* k1 = (T*)c->k[0]; T* k2 = (T*)c->k[1]; T* k3 = (T*)c->k[2]; T* k4 = (T*)c->k[3];
    T dt = T(c->dt);
    double* dens = c->dens;
    double Jw = c->dt;
    void* args[] = {&P, &f, &k1, &k2, &k3, &k4, &dt, &J, &dens, &Jw};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)adj_step_coop_kernel<T, R>,
                                                dim3(c->coop_grid), dim3(kAdjThreads), args, 0, st);
    return e == cudaSuccess ? BOLT_OK : BOLT_ERR_CUDA;
}

template <typename T, int R>
int adjoint_coop(BoltAdj1D* c, const T* f, T* lam, int obj_at_start, double* dtau,
                 cudaStream_t st) {
    Adj1DArgs P = c->P;
    T* k1 = (T*)c->k[0]; T* k2 = (T*)c->k[1]; T* k3 = (T*)c->k[2];
    T* A = (T*)c->a; T* B = (T*)c->gs; T* gacc = (T*)c->gacc;
    T dt = T(c->dt);
    double* part = c->dtau_part;
    double* dens = c->dens;
    double* reim = c->reim;
    double wobj = c->dt;
    void* args[] = {&P, &f, &lam, &k1, &k2, &k3, &A, &B, &gacc, &dt, &part, &dtau,
                    &obj_at_start, &dens, &reim, &wobj};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)adj_step_adjoint_coop_kernel<T, R>,
                                                dim3(c->coop_grid), dim3(kAdjThreads), args, 0, st);
    return e == cudaSuccess ? BOLT_OK : BOLT_ERR_CUDA;
}

template <typename T, int R>
int step_impl(BoltAdj1D* c, T* f, double* J, cudaStream_t st) {
    if (c->coop_grid > 0) return step_coop<T, R>(c, f, J, st);
    const Adj1DArgs& P = c->P;
    const T dt = T(c->dt);
    T* k1 = (T*)c->k[0]; T* k2 = (T*)c->k[1]; T* k3 = (T*)c->k[2]; T* k4 = (T*)c->k[3];
    adj_stage_kernel<T, R><<<P.Nq1, kAdjThreads, 0, st>>>(P, f, (const T*)nullptr, T(0), k1);
    adj_stage_kernel<T, R><<<P.Nq1, kAdjThreads, 0, st>>>(P, f, k1, dt / T(2), k2);
    adj_stage_kernel<T, R><<<P.Nq1, kAdjThreads, 0, st>>>(P, f, k2, dt / T(2), k3);
    adj_stage_kernel<T, R><<<P.Nq1, kAdjThreads, 0, st>>>(P, f, k3, dt, k4);
    adj_combine_kernel<T><<<ew_blocks(c->n), 256, 0, st>>>(c->n, f, k1, k2, k3, k4, dt / T(6));
    if (J) {
        adj_density_kernel<T><<<P.Nq1, kAdjThreads, 0, st>>>(P, f, c->dens);
        adj_mode_kernel<<<1, kAdjThreads, 0, st>>>(P, c->dens, c->dt, J, nullptr);
    }
    return cudaGetLastError() == cudaSuccess ? BOLT_OK : BOLT_ERR_CUDA;
}

template <typename T, int R>
int adjoint_impl(BoltAdj1D* c, const T* f, T* lam, int obj_at_start, double* dtau,
                 cudaStream_t st) {
    if (c->coop_grid > 0) return adjoint_coop<T, R>(c, f, lam, obj_at_start, dtau, st);
    const Adj1DArgs& P = c->P;
    const T dt = T(c->dt);
    const long long n = c->n;
    const int eb = ew_blocks(n);
    T* k1 = (T*)c->k[0]; T* k2 = (T*)c->k[1]; T* k3 = (T*)c->k[2];
    T* a = (T*)c->a; T* gacc = (T*)c->gacc; T* gs = (T*)c->gs;
    // recompute the stages from f
    adj_stage_kernel<T, R><<<P.Nq1, kAdjThreads, 0, st>>>(P, f, (const T*)nullptr, T(0), k1);
    adj_stage_kernel<T, R><<<P.Nq1, kAdjThreads, 0, st>>>(P, f, k1, dt / T(2), k2);
    adj_stage_kernel<T, R><<<P.Nq1, kAdjThreads, 0, st>>>(P, f, k2, dt / T(2), k3);
    // stage 4 (state f + dt k3)
    adj_axpby_kernel<T><<<eb, 256, 0, st>>>(n, a, dt / T(6), lam, T(0), (const T*)nullptr);
    adj_vjp_kernel<T, R><<<P.Nq1, kAdjThreads, 0, st>>>(P, f, k3, dt, a, gs, c->dtau_part);
    if (dtau) adj_sum_kernel<<<1, kAdjThreads, 0, st>>>(c->dtau_part, P.Nq1, dtau);
    adj_axpby_kernel<T><<<eb, 256, 0, st>>>(n, gacc, T(1), lam, T(1), gs);
    // stage 3 (state f + dt/2 k2)
    adj_axpby_kernel<T><<<eb, 256, 0, st>>>(n, a, dt / T(3), lam, dt, gs);
    adj_vjp_kernel<T, R><<<P.Nq1, kAdjThreads, 0, st>>>(P, f, k2, dt / T(2), a, gs, c->dtau_part);
    if (dtau) adj_sum_kernel<<<1, kAdjThreads, 0, st>>>(c->dtau_part, P.Nq1, dtau);
    adj_axpby_kernel<T><<<eb, 256, 0, st>>>(n, gacc, T(1), gacc, T(1), gs);
    // stage 2 (state f + dt/2 k1)
    adj_axpby_kernel<T><<<eb, 256, 0, st>>>(n, a, dt / T(3), lam, dt / T(2), gs);
    adj_vjp_kernel<T, R><<<P.Nq1, kAdjThreads, 0, st>>>(P, f, k1, dt / T(2), a, gs, c->dtau_part);
    if (dtau) adj_sum_kernel<<<1, kAdjThreads, 0, st>>>(c->dtau_part, P.Nq1, dtau);
    adj_axpby_kernel<T><<<eb, 256, 0, st>>>(n, gacc, T(1), gacc, T(1), gs);
    // stage 1 (state f)
    adj_axpby_kernel<T><<<eb, 256, 0, st>>>(n, a, dt / T(6), lam, dt / T(2), gs);
    adj_vjp_kernel<T, R><<<P.Nq1, kAdjThreads, 0, st>>>(P, f, (const T*)nullptr, T(0), a, gs,
                                                     c->dtau_part);
    if (dtau) adj_sum_kernel<<<1, kAdjThreads, 0, st>>>(c->dtau_part, P.Nq1, dtau);
    adj_axpby_kernel<T><<<eb, 256, 0, st>>>(n, lam, T(1), gacc, T(1), gs);
    if (obj_at_start) {
        adj_density_kernel<T><<<P.Nq1, kAdjThreads, 0, st>>>(P, f, c->dens);
        double* scratch_J = c->reim + 2;                    // the forward value is not needed
        adj_mode_kernel<<<1, kAdjThreads, 0, st>>>(P, c->dens, 0.0, scratch_J, c->reim);
        adj_mode_adjoint_kernel<T><<<eb, 256, 0, st>>>(P, c->reim, c->dt, lam);
    }
    return cudaGetLastError() == cudaSuccess ? BOLT_OK : BOLT_ERR_CUDA;
}

void adj_free(BoltAdj1D* c) {
    if (!c) return;
    for (int i = 0; i < 4; ++i) cudaFree(c->k[i]);
    cudaFree(c->a);
    cudaFree(c->gacc);
    cudaFree(c->gs);
    cudaFree(c->dtau_part);
    cudaFree(c->dens);
    cudaFree(c->reim);
    delete c;
}

}  // namespace

extern "C" {

int bolt_adj1d_create(const BoltAdj1DSpec* s, int dtype, BoltAdj1D** out) {
    if (!s || !out || (dtype != BOLT_F32 && dtype != BOLT_F64)) return BOLT_ERR_ARG;
    *out = nullptr;
    if (s->N_q1 < 6 || s->N_p1 < 1 || s->N_p1 > kAdjMaxNp || !(s->q1_end > s->q1_start) ||
        !(s->p1_end > s->p1_start) || !(s->dp2 > 0) || !(s->dp3 > 0) || !(s->mass > 0) ||
        !(s->boltzmann_constant > 0) || !(s->dt > 0) || s->tau < 0)
        return BOLT_ERR_ARG;
    if (s->recon != BOLT_RECON_WENO5 && s->recon != BOLT_RECON_MINMOD) return BOLT_ERR_UNSUPPORTED;
    BoltAdj1D* c = new (std::nothrow) BoltAdj1D();
    if (!c) return BOLT_ERR_NOMEM;
    c->dtype = dtype;
    c->recon = s->recon == BOLT_RECON_MINMOD ? kAdjMinmod : kAdjWeno5;
    c->dt = s->dt;
    c->n = (long long)s->N_q1 * s->N_p1;
    Adj1DArgs& P = c->P;
    P.Nq1 = s->N_q1;
    P.Np1 = s->N_p1;
    P.dq1 = (s->q1_end - s->q1_start) / s->N_q1;
    P.inv_dq = 1.0 / P.dq1;
    P.dp1 = (s->p1_end - s->p1_start) / s->N_p1;
    P.p1_start = s->p1_start;
    P.mass = s->mass;
    P.kB = s->boltzmann_constant;
    P.tau = s->tau;
    P.measure = (s->dp3 * s->dp2) * P.dp1;
    const size_t eb = dtype == BOLT_F64 ? 8 : 4;
    int rc = BOLT_OK;
    auto alloc = [&](void** p, size_t bytes) {
        if (rc == BOLT_OK && cudaMalloc(p, bytes) != cudaSuccess) rc = BOLT_ERR_NOMEM;
    };
    for (int i = 0; i < 4; ++i) alloc(&c->k[i], c->n * eb);
    alloc(&c->a, c->n * eb);
    alloc(&c->gacc, c->n * eb);
    alloc(&c->gs, c->n * eb);
    alloc((void**)&c->dtau_part, 4 * (size_t)s->N_q1 * sizeof(double));
    alloc((void**)&c->dens, s->N_q1 * sizeof(double));
    alloc((void**)&c->reim, 3 * sizeof(double));
    if (rc != BOLT_OK) {
        adj_free(c);
        return rc;
    }
    // whole steps as cooperative launches unless BOLT_ADJ_SEPARATE is set
    if (!getenv("BOLT_ADJ_SEPARATE")) {
        if (dtype == BOLT_F64)
            c->coop_grid = c->recon == kAdjMinmod ? coop_grid_for<double, kAdjMinmod>(P.Nq1)
                                                  : coop_grid_for<double, kAdjWeno5>(P.Nq1);
        else
            c->coop_grid = c->recon == kAdjMinmod ? coop_grid_for<float, kAdjMinmod>(P.Nq1)
                                                  : coop_grid_for<float, kAdjWeno5>(P.Nq1);
    }
    *out = c;
    return BOLT_OK;
}

void bolt_adj1d_destroy(BoltAdj1D* c) { adj_free(c); }

int bolt_adj1d_set_tau(BoltAdj1D* c, double tau) {
    if (!c || tau < 0) return BOLT_ERR_ARG;
    c->P.tau = tau;
    return BOLT_OK;
}

int bolt_adj1d_step(BoltAdj1D* c, void* f, double* J_dev, void* stream) {
    if (!c || !f) return BOLT_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (c->recon == kAdjMinmod)
        return c->dtype == BOLT_F64 ? step_impl<double, kAdjMinmod>(c, (double*)f, J_dev, st)
                                    : step_impl<float, kAdjMinmod>(c, (float*)f, J_dev, st);
    return c->dtype == BOLT_F64 ? step_impl<double, kAdjWeno5>(c, (double*)f, J_dev, st)
                                : step_impl<float, kAdjWeno5>(c, (float*)f, J_dev, st);
}

int bolt_adj1d_step_adjoint(BoltAdj1D* c, const void* f_n, void* lam, int objective_at_start,
                            double* dtau_dev, void* stream) {
    if (!c || !f_n || !lam) return BOLT_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (c->recon == kAdjMinmod)
        return c->dtype == BOLT_F64
            ? adjoint_impl<double, kAdjMinmod>(c, (const double*)f_n, (double*)lam,
                                               objective_at_start, dtau_dev, st)
            : adjoint_impl<float, kAdjMinmod>(c, (const float*)f_n, (float*)lam,
                                              objective_at_start, dtau_dev, st);
    return c->dtype == BOLT_F64
        ? adjoint_impl<double, kAdjWeno5>(c, (const double*)f_n, (double*)lam,
                                          objective_at_start, dtau_dev, st)
        : adjoint_impl<float, kAdjWeno5>(c, (const float*)f_n, (float*)lam,
                                         objective_at_start, dtau_dev, st);
}

int bolt_adj1d_objective(BoltAdj1D* c, const void* f, double* J_dev, void* lam, void* stream) {
    if (!c || !f || !J_dev) return BOLT_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const Adj1DArgs& P = c->P;
    if (c->dtype == BOLT_F64)
        adj_density_kernel<double><<<P.Nq1, kAdjThreads, 0, st>>>(P, (const double*)f, c->dens);
    else
        adj_density_kernel<float><<<P.Nq1, kAdjThreads, 0, st>>>(P, (const float*)f, c->dens);
    adj_mode_kernel<<<1, kAdjThreads, 0, st>>>(P, c->dens, c->dt, J_dev, c->reim);
    if (lam) {
        const int eb = ew_blocks(c->n);
        if (c->dtype == BOLT_F64)
            adj_mode_adjoint_kernel<double><<<eb, 256, 0, st>>>(P, c->reim, c->dt, (double*)lam);
        else
            adj_mode_adjoint_kernel<float><<<eb, 256, 0, st>>>(P, c->reim, c->dt, (float*)lam);
    }
    return cudaGetLastError() == cudaSuccess ? BOLT_OK : BOLT_ERR_CUDA;
}

}  // extern "C"
