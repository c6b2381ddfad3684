/*
 * bolt_b200.h - C ABI of the B200 (sm_100a) finite-volume kinetic update.
 *
 * One context per device per solver.  All device buffers passed in are owned
 * by the caller (PyTorch tensors in the Python layer); the context owns its
 * scratch (RK stage buffers, moment partial sums, Yee/cell field arrays).
 * Every call is asynchronous on the CUDA stream it is given; nothing here
 * synchronises the host except bolt_status_sync().
 *
 * Distribution-function layout (identical to Bolt's q-expanded array, which is
 * column-major (N_p1*N_p2*N_p3, N_s, N_q1+2Ng, N_q2+2Ng)):
 *     f[q2g][q1g][s][p3][p2][p1]   row-major, p1 fastest, ghost zones included
 * Moments (FP64):  m[q2g][q1g][s]
 * Fields  (FP64):  fld[c][q2g][q1g], c = E1,E2,E3,B1,B2,B3
 *
 * Reference interfaces replaced (paths within the Bolt project):
 *   bolt_ctx_create      nonlinear_solver.__init__   bolt/lib/nonlinear/nonlinear_solver.py:67-413
 *   bolt_fill_ghosts     communicate_f + apply_bcs_f bolt/lib/nonlinear/communicate.py:8-38,
 *                                                    bolt/lib/nonlinear/boundaries.py:415-577
 *   bolt_dfdt            df_dt_fvm                   bolt/lib/nonlinear/finite_volume/df_dt_fvm.py:33-339
 *   bolt_step            op_fvm / timestep_fvm       bolt/lib/nonlinear/finite_volume/fvm_operator.py:6-50
 *                        (RK4 stages: bolt/lib/nonlinear/temporal_evolution/integrators.py:15-28)
 *   bolt_moments         compute_moments             bolt/lib/nonlinear/compute_moments.py:7-59
 *   bolt_fields_set/get  fields_solver state         bolt/lib/nonlinear/fields/fields.py:421-495,649-690
 *   bolt_divergence_flag check_divergence            bolt/lib/nonlinear/timestep.py:28-38
 *   bolt_dfdt_term       df_dt_fvm(term_to_return)   bolt/lib/nonlinear/finite_volume/df_dt_fvm.py:325-339
 *   bolt_set_shear/time  apply_shearing_box_bcs_f    bolt/lib/nonlinear/boundaries.py:6-145
 *   bolt_set_p_space_grid params.p_space_grid        bolt/lib/nonlinear/boundaries.py:313-413,
 *                                                    bolt/lib/nonlinear/compute_moments.py:42-56
 *   bolt_timings         print_table                 bolt/lib/utils/performance_timings.py:9-165
 */
#ifndef BOLT_B200_H
#define BOLT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BOLT_MAX_SPECIES 8

/* status codes */
#define BOLT_OK                 0
#define BOLT_ERR_ARG            1   /* bad argument / unsupported combination */
#define BOLT_ERR_CUDA           2   /* a CUDA runtime/driver call failed        */
#define BOLT_ERR_NONFINITE      3   /* Inf/NaN appeared in f ('Solver Diverging!') */
#define BOLT_ERR_TIMEOUT        4   /* a bounded device-side wait gave up       */
#define BOLT_ERR_UNSUPPORTED    5   /* shape/option outside this build's kernels */
#define BOLT_ERR_NOMEM          6

/* dtype of f */
#define BOLT_F64 0
#define BOLT_F32 1
/* f in FP64; the fused q-stage of 8x8-tiled grids runs the paired kernel with
 * FMA contraction and Newton-refined reciprocals (throughput form, agreeing
 * with BOLT_F64 to rounding), every other kernel as for BOLT_F64 */
#define BOLT_F64_FAST 2

/* reconstruction (reconstruct.py:29-44) */
#define BOLT_RECON_PC     0   /* 'piecewise-constant' */
#define BOLT_RECON_MINMOD 1   /* 'minmod'             */
#define BOLT_RECON_PPM    2   /* 'ppm'                */
#define BOLT_RECON_WENO5  3   /* 'weno5'              */

/* numerical flux (riemann.py:46-49 upwind; LLF, the local Lax-Friedrichs flux, has no
 * counterpart in riemann.py) */
#define BOLT_FLUX_UPWIND 0
#define BOLT_FLUX_LLF    1

/* boundary conditions along q1/q2 (boundaries.py:415-577) */
#define BOLT_BC_PERIODIC  0
#define BOLT_BC_DIRICHLET 1
/* the ghost rows (q2) / columns (q1) are supplied by the caller before every
 * stage (a block of a larger domain whose neighbours own those cells); the
 * library reads them and never writes them. */
#define BOLT_BC_EXTERNAL  2
/* mirror (boundaries.py:226-301, cartesian p-grid): ghost cell i < 0 holds
 * interior cell -1-i (i >= N: 2N-1-i) with the p-index normal to the edge
 * reversed (p1 for q1, p2 for q2); needs N_ghost <= N_q along the axis */
#define BOLT_BC_MIRROR    3
/* mirror, then the Dirichlet inflow values where the velocity normal to the
 * edge points into the domain (apply_bcs_f's 'mirror+dirichlet') */
#define BOLT_BC_MIRROR_DIRICHLET 4
/* shearing box (boundaries.py:6-145): periodic, then each ghost strip
 * resampled along the other q axis at positions shifted by -/+ q omega L t
 * (L the length of the strip's own axis, t the time set by bolt_set_time;
 * q, omega from bolt_set_shear), wrapped into the domain, by the
 * one-dimensional Catmull-Rom cubic.  One axis at most, the other periodic;
 * needs N_ghost >= 2. */
#define BOLT_BC_SHEARING_BOX 5

/* p-space grids (params.p_space_grid).  On BOLT_PGRID_POLAR2D, p1 is the
 * radius and p2 the angle theta over a full turn: every moment -- the BGK
 * Maxwellian's, bolt_moments', the field sources' -- carries the factor
 * initial_mu (compute_moments.py:48-53), and a mirror edge reflects theta
 * (boundaries.py:313-413): theta -> -theta at q2 edges (the p2 index
 * reversed), theta -> pi - theta at q1 edges (each half of the p2 index range
 * reversed on its own; needs an even N_p2). */
#define BOLT_PGRID_CARTESIAN 0
#define BOLT_PGRID_POLAR2D   1

/* field models (fields.py:559-690): electrodynamic fields advanced by FDTD
 * once per step, or electrostatic fields re-solved from the charge density of
 * every df/dt argument by the periodic FFT Poisson solve (fft.py:9-78,
 * df_dt_fvm.py:234-242) */
#define BOLT_FIELDS_ELECTRODYNAMIC 0
#define BOLT_FIELDS_ELECTROSTATIC  1

/* integrators */
#define BOLT_RK2 2   /* fvm_operator.py:6-35 midpoint */
#define BOLT_RK4 4   /* classic RK4 around df_dt_fvm  */

/* moment ids (moments.py:6-58) */
#define BOLT_MOM_DENSITY   0
#define BOLT_MOM_V1        1
#define BOLT_MOM_V2        2
#define BOLT_MOM_V3        3
#define BOLT_MOM_ENERGY    4
#define BOLT_MOM_ENERGY_Q1 5
#define BOLT_MOM_ENERGY_Q2 6
#define BOLT_MOM_ENERGY_Q3 7
#define BOLT_MOM_Q_Q1      8
#define BOLT_MOM_Q_Q2      9
#define BOLT_MOM_Q_Q3     10

typedef struct BoltGrid {
    int    N_q1, N_q2, N_ghost;
    int    N_p1, N_p2, N_p3, N_s;
    double q1_start, q2_start, dq1, dq2;
    double p1_start[BOLT_MAX_SPECIES], p2_start[BOLT_MAX_SPECIES], p3_start[BOLT_MAX_SPECIES];
    double dp1[BOLT_MAX_SPECIES], dp2[BOLT_MAX_SPECIES], dp3[BOLT_MAX_SPECIES];
} BoltGrid;

typedef struct BoltParams {
    int    dtype;                 /* BOLT_F64 / BOLT_F32                       */
    int    recon_q, recon_p;      /* BOLT_RECON_*                              */
    int    flux_q, flux_p;        /* BOLT_FLUX_*                               */
    int    bc_q1, bc_q2;          /* BOLT_BC_*                                 */
    int    integrator;            /* BOLT_RK2 / BOLT_RK4                       */
    int    source_enabled;        /* BGK relaxation on/off                     */
    int    fields_enabled;        /* field coupling on/off                     */
    int    p_dim;                 /* 1, 2 or 3                                 */
    int    fields_type;           /* BOLT_FIELDS_* (when fields_enabled)       */
    double mass[BOLT_MAX_SPECIES], charge[BOLT_MAX_SPECIES];
    double boltzmann_constant;
    double tau;                   /* constant BGK tau (see bolt_set_tau_array) */
    double eps, mu;               /* FDTD permittivity / permeability          */
} BoltParams;

typedef struct BoltCtx BoltCtx;

/* Context lifetime.  Allocates the RK scratch on the current device. */
int  bolt_ctx_create(const BoltGrid* grid, const BoltParams* params, BoltCtx** out);
void bolt_ctx_destroy(BoltCtx* ctx);

/* Optional phase-space-dependent tau: f-shaped device array of the same dtype
 * as f (caller-owned, must outlive the context).  NULL restores the constant. */
int  bolt_set_tau_array(BoltCtx* ctx, const void* tau_dev);

/* Dirichlet boundary values for side 0=left,1=right,2=bottom,3=top: an
 * f-shaped device array of boundary-function values (caller-owned).  Ghost
 * cells take these values where the q-velocity points into the domain and
 * zero elsewhere (boundaries.py:147-225; PETSc ghosted halos stay zero). */
int  bolt_set_dirichlet(BoltCtx* ctx, int side, const void* values_dev);

/* Shearing-box constants (params.q, params.omega of boundaries.py:17-18) and
 * the time the ghost strips are sheared to (the reference's time_elapsed,
 * constant over the stages of a step). */
int  bolt_set_shear(BoltCtx* ctx, double q, double omega);

/* The context's p-space grid (BOLT_PGRID_*; cartesian after create) and, for
 * polar2D, params.initial_mu.  Set it before the first step.  Polar2D with a
 * q1 mirror edge and an odd N_p2 is BOLT_ERR_UNSUPPORTED. */
int  bolt_set_p_space_grid(BoltCtx* ctx, int grid, double initial_mu);
int  bolt_set_time(BoltCtx* ctx, double t);

/* Halo refresh of f in place (periodic wrap + Dirichlet inflow). */
int  bolt_fill_ghosts(BoltCtx* ctx, void* f_dev, void* stream);

/* Advective semi-Lagrangian (ASL) method in q, fields off or electrostatic --
 * the operators that Bolt's timesteps split (asl_operators.py:20-83;
 * timestep.py:39-240 composes them by Strang, Lie, SWSS or Jia splitting,
 * operator_splitting_methods.py).
 * bolt_asl_advect_q is op_advect_q (interpolation_routines.py:9-56): ghost
 * refresh, then every interior cell takes f at the foot of its
 * characteristic q - (p1, p2) dt, by the bicubic interpolation that Bolt gets
 * from ArrayFire's approx2(BICUBIC_SPLINE), restated here as the tensor
 * product of Catmull-Rom cubics over the ghosted grid (neighbours clamped to
 * it, 0 for a foot outside it); N_ghost >= 2, feet up to N_ghost - 1 cells
 * away read real ghost data.  bolt_asl_source is op_solve_src: f <- f_MB of
 * f's own moments when instantaneous != 0, else one RK2 step of the BGK
 * source with the constant tau (needs params->source_enabled; no tau array).
 * Both write f's interior in place (the context's first stage buffer is
 * their scratch) and leave its ghost cells stale (the next refresh, or
 * bolt_asl_advect_q itself, fills them); BOLT_ERR_UNSUPPORTED with
 * electrodynamic fields.  With electrostatic fields the pair is split again
 * with op_fvm, the FVM in p (timestep.py:134-148), whose df/dt then has no
 * q-part and no source (df_dt_fvm.py:56-99): bolt_fvm_p_step is that step
 * (the context's integrator, the FFT field solve of every stage input). */
int  bolt_asl_advect_q(BoltCtx* ctx, void* f_dev, double dt, void* stream);
int  bolt_asl_source(BoltCtx* ctx, void* f_dev, double dt, int instantaneous, void* stream);
int  bolt_fvm_p_step(BoltCtx* ctx, void* f_dev, double dt, void* stream);

/* The same two operators between separate f-shaped buffers, so that a
 * splitting hands f from one operator to the next without copying it back
 * (Strang: f -> w -> w -> f; Lie: f -> w -> f, w the context's work buffer
 * 0).  bolt_asl_advect_q_to refreshes f_in's ghost cells and writes the
 * interpolated interior into out (out != f_in).  bolt_asl_source_to reads
 * f_in and writes out's interior (out may be f_in); scratch (!= f_in, may be
 * out; unused when instantaneous) holds the RK2 half step.  Ghost cells of
 * the written buffers are stale afterwards.  bolt_work_buffer gives the
 * context's f-shaped work buffer i (0 always exists; 1 and 2 with RK4). */
int  bolt_asl_advect_q_to(BoltCtx* ctx, void* f_in, void* out, double dt, void* stream);
int  bolt_asl_source_to(BoltCtx* ctx, const void* f_in, void* out, void* scratch, double dt,
                        int instantaneous, void* stream);
int  bolt_work_buffer(BoltCtx* ctx, int i, void** ptr);

/* Forget cached halo/moment state (call after f was modified outside the
 * library; bolt_step then refreshes halos and moments before stepping). */
int  bolt_invalidate(BoltCtx* ctx);

/* df/dt of f (ghosts must be current) into dfdt (interior cells written).
 * With fields enabled, evolve_fields != 0 first advances the fields with the
 * currents of this f (the reference's at_n == False branch). */
int  bolt_dfdt(BoltCtx* ctx, const void* f_dev, void* dfdt_dev, int evolve_fields,
               double dt, void* stream);

/* One p-flux divergence of f (fields enabled): term = 1, 2 or 3 writes
 * d_flux_pk_dpk = (F_pk(right face) - F_pk(left face)) / dpk into the
 * interior cells of out, after the same field evaluation bolt_dfdt performs
 * (evolve_fields as there).  Replaces df_dt_fvm's term_to_return
 * (df_dt_fvm.py:325-339); BOLT_ERR_UNSUPPORTED without fields, where the
 * reference has no p-fluxes either. */
int  bolt_dfdt_term(BoltCtx* ctx, const void* f_dev, void* out_dev, int term, int evolve_fields,
                    double dt, void* stream);

/* One full RK step of f in place (ghosts refreshed by the call). */
int  bolt_step(BoltCtx* ctx, void* f_dev, double dt, void* stream);

/* n_steps RK steps, ghosts refreshed, launched back to back. */
int  bolt_run(BoltCtx* ctx, void* f_dev, double dt, int n_steps, void* stream);

/* One RK step as separate stages, for callers that must act between stages
 * (a q2 slab exchanging its BOLT_BC_EXTERNAL ghost rows with the neighbouring
 * slabs before each stage; fvm_operator.py:22-33 refreshes halos at the same
 * points).  bolt_stage_count gives 2 (RK2) or 4 (RK4); bolt_stage_input the
 * device buffer that stage k reads (f for k = 0, a context stage buffer
 * otherwise; its ghost rows must be current when stage k is launched);
 * bolt_stage runs stage k of the step of f.  Stages 0..count-1 in order are
 * one bolt_step. */
int   bolt_stage_count(BoltCtx* ctx);
void* bolt_stage_input(BoltCtx* ctx, void* f_dev, int k);
int   bolt_stage(BoltCtx* ctx, void* f_dev, double dt, int k, void* stream);

/* A block with electrodynamic fields (an external axis): the stage that
 * advances the FDTD fields runs in bolt_stage_parts(ctx, k) = 3 parts, and
 * before parts 1 and 2 the caller refreshes the Yee ghosts of the external
 * axes from the neighbouring blocks, q1 columns (all rows) first, then q2
 * rows (all columns) -- the reference's communicate_fields between the
 * halves of the FDTD update (fields.py:169-180, fdtd_explicit.py:141-177,
 * communicate.py:40-77).  The Yee array is bolt_fields_yee(ctx),
 * [6][N_q2+2N_g][N_q1+2N_g] FP64 on the device.  Every other stage has one
 * part; parts 0..n-1 in order equal bolt_stage. */
int     bolt_stage_parts(BoltCtx* ctx, int k);
int     bolt_stage_part(BoltCtx* ctx, void* f_dev, double dt, int k, int part, void* stream);

/* Stage k of a block in three calls, so that the halo exchange of its input
 * overlaps computation (the reference exchanges, then computes:
 * communicate.py:8-38 before each df/dt, fvm_operator.py:22-33).  region 0
 * updates the q-tiles whose stencils stay inside the block along its external
 * axes (every 8x8 tile but the outermost ring of tiles on those axes) and
 * reads none of their ghost cells, so it may run while they are being filled;
 * region 1, once they are filled, updates the other tiles (it may run on
 * another stream beside region 0: the two write different tiles); region 2,
 * after both, finishes the stage (ghost pass of non-periodic axes, the step's
 * bookkeeping).  Regions 0, 1, 2 equal bolt_stage.  Each returns
 * BOLT_ERR_UNSUPPORTED, having launched nothing, for a stage that cannot be
 * split: fields enabled, a stage outside the paired kernel, peer halos on, or
 * stage 0 while the ghosts or moments of f are stale (bolt_fill_ghosts /
 * a previous step make them current); the caller then runs bolt_stage after
 * the exchange. */
int     bolt_stage_region(BoltCtx* ctx, void* f_dev, double dt, int k, int region, void* stream);
double* bolt_fields_yee(BoltCtx* ctx);

/* Peer halos of a q2 slab (bc_q2 = BOLT_BC_EXTERNAL, fields off): below[] and
 * above[] are the lower and upper neighbours' device copies of
 * (f, bolt_stage_buffer(0), bolt_stage_buffer(1)) -- on another GPU, its
 * memory mapped into this process (CUDA IPC or symmetric memory).  Every stage
 * then also stores its bottom / top N_g interior rows into the matching
 * buffer's top / bottom ghost rows at the neighbours, from the stage kernel
 * itself, so no exchange precedes the next stage.  The caller must order the
 * slabs' stages: every slab's stage k completes before any slab's stage k+1
 * (one bolt_stage per slab, then a barrier between the ranks).  Null arrays
 * switch it off.  RK2 needs the first two entries. */
int   bolt_set_peer_halos(BoltCtx* ctx, const void* const* below, const void* const* above);
/* The same along q1 for a block of a P1 x P2 grid (bc_q1 = BOLT_BC_EXTERNAL):
 * left[] and right[] are the q1 neighbours' copies; every stage also stores
 * its left / right N_g interior columns into their right / left ghost
 * columns.  Corner ghost cells are written by neither call: no interior
 * update reads them.  Replaces the q1 part of the DMDA halo refresh
 * (communicate.py:8-38, nonlinear_solver.py:251-280).  Null arrays switch
 * it off. */
int   bolt_set_peer_halos_q1(BoltCtx* ctx, const void* const* left, const void* const* right);
/* The context's RK stage buffers 0 and 1 (their neighbours' peer pointers). */
void* bolt_stage_buffer(BoltCtx* ctx, int i);
/* CUDA IPC of a whole device allocation (the stage buffers are): a 64-byte
 * handle another process maps with bolt_ipc_open and releases with
 * bolt_ipc_close. */
int   bolt_ipc_get(const void* dev_ptr, unsigned char* handle64);
int   bolt_ipc_open(const unsigned char* handle64, void** dev_ptr);
int   bolt_ipc_close(void* dev_ptr);

/* One moment (BOLT_MOM_*) of f over the whole ghosted grid, FP64, written to
 * out_dev[q2g][q1g][s] (moments.py definitions times dp1*dp2*dp3). */
int  bolt_moments(BoltCtx* ctx, const void* f_dev, int moment_id, double* out_dev, void* stream);

/* Fields state (FP64 device arrays of 6*Nq2g*Nq1g doubles). */
int  bolt_fields_set(BoltCtx* ctx, const double* cell_dev, const double* yee_dev, void* stream);
int  bolt_fields_get(BoltCtx* ctx, double* cell_dev, double* yee_dev, void* stream);
/* One FDTD update of the context's fields with the caller's currents:
 * J_dev = [3][N_q2+2N_g][N_q1+2N_g] FP64 (J1, J2, J3 summed over species, on
 * the E components' Yee positions), as fields_solver.evolve_electrodynamic_fields
 * (fields.py:568-647): E += dt curl B / (mu eps) - J dt / eps, then
 * B -= dt curl E, then the cell-centred fields.  Electrodynamic contexts only. */
int  bolt_fields_evolve(BoltCtx* ctx, const double* J_dev, double dt, void* stream);

/* FDTD time-level flag of the reference's fields solver (fields.py:271-273,
 * 685-688): each df/dt evaluation flips it; a stage evolves the fields when it
 * is 0 on entry (RK2).  RK4 evolves in stage 2 and leaves it unchanged. */
int  bolt_get_at_n(BoltCtx* ctx);
int  bolt_set_at_n(BoltCtx* ctx, int at_n);

/* Divergence flag: device-side Inf/NaN detection on every step's output,
 * written to pinned host memory.  Returns 1 once any step produced a
 * non-finite value (no synchronisation), 0 otherwise. */
int  bolt_divergence_flag(BoltCtx* ctx);
int  bolt_clear_divergence_flag(BoltCtx* ctx);

/* Allocation-free df/dt, for callers that cannot allocate device memory when
 * they need an evaluation (fixed-budget memory pools, code that must not
 * trigger the implicit synchronisation of cudaMalloc/cudaFree, embedders
 * that own all device memory).  No reference counterpart: Bolt's df_dt_fvm
 * always allocates its temporaries.  Same result as bolt_dfdt for
 * fields-disabled problems with a constant tau (params->tau; a phase-space
 * tau array is not available here): writes df/dt of f (ghost cells current)
 * into the interior cells of dfdt.  Its only scratch (FP64 moment sums, an
 * error word and a non-finite flag) is a fixed device array of this library
 * holding BOLT_NOALLOC_MAX_QCELLS (N_s*N_q1*N_q2) q-cells; larger grids and
 * fields return BOLT_ERR_UNSUPPORTED, and grids or parameters bolt_ctx_create
 * would refuse are refused alike.  The first call on a device looks up that
 * array's address (make it before any stream capture); calls that overlap on
 * the GPU share the array and race. */
#define BOLT_NOALLOC_MAX_QCELLS 65536
int  bolt_dfdt_noalloc(const BoltGrid* grid, const BoltParams* params, const void* f_dev,
                       void* dfdt_dev, void* stream);
/* Status of the last bolt_dfdt_noalloc on the current device, read after the
 * stream has synchronised and then cleared: *status = BOLT_OK,
 * BOLT_ERR_TIMEOUT (a bounded tile wait ran out and part of dfdt is
 * unwritten) or BOLT_ERR_NONFINITE (df/dt holds Inf/NaN).  Allocates nothing;
 * returns BOLT_ERR_CUDA if the copy or the synchronisation failed. */
int  bolt_noalloc_status(void* stream, int* status);

/* Synchronise the stream and return the first sticky error of the context:
 * the device error word (BOLT_ERR_TIMEOUT once a stage kernel's bounded wait
 * ran out), else the first failed CUDA call. */
int  bolt_status_sync(BoltCtx* ctx, void* stream);

/* The device error word without synchronising (it lives in pinned host
 * memory): BOLT_OK, or BOLT_ERR_TIMEOUT once a stage kernel whose bounded
 * tile wait ran out has finished; that stage left part of its output
 * unwritten.  Like bolt_divergence_flag it reports kernels that have
 * completed; bolt_clear_error resets it.  Extends check_divergence
 * (timestep.py:28-38), which has no timeout to report. */
int  bolt_error_flag(BoltCtx* ctx);
int  bolt_clear_error(BoltCtx* ctx);

/* Budget of the stage kernels' bounded tile waits, in SM clock cycles; the
 * default (<= 0 restores it) is 4e9, about 2 s at the boost clock. */
int  bolt_set_wait_budget(BoltCtx* ctx, long long cycles);

/* Test hook: with on != 0 the TMA stage kernels issue no tile copies, so the
 * first bounded tile wait of every CTA runs out (after the budget above) with
 * nothing in flight; the CTAs record BOLT_ERR_TIMEOUT and return without
 * writing their outputs.  It makes the timeout path testable without a fault
 * or a hang.  No reference counterpart. */
int  bolt_test_stall_waits(BoltCtx* ctx, int on);
const char* bolt_strerror(int code);

/* Per-component device time (performance_timings.py:9-165 reports the same
 * split of a step for the reference's ArrayFire path).  With bolt_set_timing
 * on, every launch group is bracketed by CUDA events on its stream;
 * bolt_timings synchronises on them, writes the accumulated milliseconds per
 * component since the last call to ms_out[BOLT_TIMING_COUNT] and resets
 * them.  Each launch group is also an NVTX range ("bolt: q-stage", ...),
 * inside one range per RK stage ("bolt: RK stage k"), whether or not timing
 * is on. */
#define BOLT_TIMING_GHOSTS  0   /* communicate_f + apply_bcs_f: the ghost pass     */
#define BOLT_TIMING_MOMENTS 1   /* velocity moments of a stage input (BGK)        */
#define BOLT_TIMING_QSTAGE  2   /* q-advection + BGK + RK combine (+ moments out) */
#define BOLT_TIMING_PSTAGE  3   /* p-advection from the cell-centred fields       */
#define BOLT_TIMING_FIELDS  4   /* FDTD update or electrostatic FFT solve          */
#define BOLT_TIMING_COUNT   5
int  bolt_set_timing(BoltCtx* ctx, int on);
int  bolt_timings(BoltCtx* ctx, double* ms_out);

/* Number of kernels launched through this context so far, and how many of
 * them were the paired stage kernel (the fused q-stage taken for FP32 and
 * BOLT_F64_FAST 8x8-tiled grids; every other stage runs the
 * one-cell-per-thread kernel).
 * Diagnostics: the reference has no counterpart. */
long long bolt_launch_count(BoltCtx* ctx);
long long bolt_paired_launch_count(BoltCtx* ctx);

/* The context's p-split of the q-stage grid: nsplit CTAs per q-tile and
 * species, each over chunks_per_split chunks of 32 p-cells (chosen to fill
 * the GPU's SMs; $BOLT_CHUNKS_PER_SPLIT at context creation fixes it). */
int  bolt_split_info(BoltCtx* ctx, int* nsplit, int* chunks_per_split);

/* Bytes of device scratch held by the context. */
size_t bolt_scratch_bytes(BoltCtx* ctx);

/* ------------------------------------------------------------------------
 * Ragged batch of independent 1D1V runs.  No reference counterpart: Bolt
 * advances one system per nonlinear_solver (nonlinear_solver.py:67,
 * timestep.py:101-160); a sweep is a loop of such runs.  Here every run keeps
 * Bolt's 1D1V setup (q1 periodic, N_q2 = N_p2 = N_p3 = 1, p_dim = 1, one
 * species, fields off, WENO5 + upwind/LLF in q1, BGK with a constant tau,
 * RK4 as in bolt_step) with its own N_q1, N_p1, ranges, tau and dt, and all
 * runs advance together: FP32 f with FP64 moments, one launch per RK stage
 * over the packed runs, nsteps steps replayed as one CUDA graph.
 * Layout: run r's ghosted f is N_q1 + 6 rows (q1, N_ghost = 3) of N_p1 FP32
 * values (p1 fastest) at element bolt_batch_f_offset(r) of bolt_batch_f();
 * moment sums are 5 doubles (n, mom_v1..3, energy, raw sums over p without
 * the p-cell measure) per q-cell at q-cell bolt_batch_q_offset(r).
 * ------------------------------------------------------------------------ */
typedef struct BoltBatchRun {
    int N_q1, N_p1;               /* N_q1 % 4 == 0 and >= 6; N_p1 % 32 == 0 */
    double q1_start, q1_end;      /* periodic q1 domain (domain.q1_start/_end) */
    double p1_start, p1_end;      /* domain.p1_start/_end */
    double p2_center, p3_center;  /* centre of the single p2 / p3 cell */
    double dp2, dp3;              /* width of that cell (the p-cell measure) */
    double mass, boltzmann_constant, tau, dt;
} BoltBatchRun;

typedef struct BoltBatch BoltBatch;

/* Allocate the packed buffers and the work queue.  BOLT_ERR_UNSUPPORTED for
 * shapes outside the batch kernel (N_q1 % 4, N_p1 % 32), BOLT_ERR_ARG for
 * invalid ranges or constants. */
int  bolt_batch_create(const BoltBatchRun* runs, int nruns, int source_enabled,
                       BoltBatch** out);
void bolt_batch_destroy(BoltBatch* b);
void* bolt_batch_f(BoltBatch* b);                          /* packed f, device */
long long bolt_batch_f_count(const BoltBatch* b);          /* elements of packed f */
long long bolt_batch_f_offset(const BoltBatch* b, int run);
int  bolt_batch_q_offset(const BoltBatch* b, int run);
int  bolt_batch_q_count(const BoltBatch* b);
/* After f is written: periodic ghosts of every run (communicate_f +
 * apply_bcs_f) and the moments of f. */
int  bolt_batch_prepare(BoltBatch* b, void* stream);
/* nsteps RK4 steps of every run on the stream (a CUDA graph of 4 stage
 * launches per step, captured on first use for this nsteps). */
int  bolt_batch_run(BoltBatch* b, int nsteps, void* stream);
/* Copy the moment sums of the current f ([q-cell][5] doubles) to out_dev. */
int  bolt_batch_moments(BoltBatch* b, double* out_dev, void* stream);
/* 1 once a stage produced a non-finite value (cleared by the call). */
int  bolt_batch_divergence_flag(BoltBatch* b);
/* The launch schedule: q-cells per work item (8, 16, 32 or 64: CTAs of 2, 4,
 * 8 or 16 warps), persistent CTAs per SM (clamped to what fits), and the queue
 * order (1: items by decreasing cells x p-chunks, 0: run by run).  Every
 * schedule gives bit-identical results; it changes only the speed.  The
 * default is (32, all that fit, 1).  Setting it synchronises the device and
 * drops the captured graph.  bolt_batch_get_schedule reports the CTA count
 * actually launched. */
int  bolt_batch_set_schedule(BoltBatch* b, int tile_cells, int ctas_per_sm, int lpt_order);
int  bolt_batch_get_schedule(const BoltBatch* b, int* tile_cells, int* ctas, int* lpt_order);

/* ------------------------------------------------------------------------
 * Adjoint of the 1D1V update.  No reference counterpart: Bolt has no
 * differentiation.  The forward step is the same scheme as bolt_step for a
 * 1D1V system (df_dt_fvm.py:56-97 with the WENO5 of weno5.py:4-98 including
 * its eps (1 + |a| + |b| + |c|) or the minmod of minmod.py:4-71, upwind/LLF
 * faces, BGK with p_dim = 1, RK4 of integrators.py:15-28), on f[N_q1][N_p1]
 * (p1 fastest) with periodic q1 and no ghost storage.  The adjoint step is
 * hand-written: exact derivatives of the WENO5 nonlinear weights (a
 * subgradient of the minmod limiter: the passed argument gets derivative 1),
 * of the Maxwellian through the velocity moments and of tau (see
 * bolt_adj1d_step_adjoint).  Objective:
 * J = sum over steps n >= 1 of dt |nhat_1(f_n)|^2, nhat_1 the k = 1 Fourier
 * coefficient (1/N_q1) sum_i n_i exp(-2 pi i x_i / L) of the density.
 * ------------------------------------------------------------------------ */
typedef struct BoltAdj1DSpec {
    int N_q1, N_p1;                /* N_q1 >= 6, N_p1 <= 2048 */
    double q1_start, q1_end;       /* periodic q1 */
    double p1_start, p1_end;
    double dp2, dp3;               /* the single p2 / p3 cell (centred at 0) */
    double mass, boltzmann_constant;
    double tau;                    /* BGK collision time; 0 = collisionless */
    double dt;
    int recon;                     /* BOLT_RECON_WENO5, or BOLT_RECON_MINMOD
                                      (differentiated by a subgradient)   */
} BoltAdj1DSpec;

typedef struct BoltAdj1D BoltAdj1D;

int  bolt_adj1d_create(const BoltAdj1DSpec* spec, int dtype, BoltAdj1D** out);
void bolt_adj1d_destroy(BoltAdj1D* c);
int  bolt_adj1d_set_tau(BoltAdj1D* c, double tau);
/* One RK4 step of f (device, in place); J_dev (device double, may be null)
 * += dt |nhat_1(f_new)|^2. */
int  bolt_adj1d_step(BoltAdj1D* c, void* f, double* J_dev, void* stream);
/* Adjoint of the step that starts from f_n: lam holds the adjoint of
 * f_{n+1} on entry and of f_n on return; with objective_at_start != 0 the
 * objective's term of f_n is added; dtau_dev (device double, may be null)
 * += this step's contribution to dJ/dtau. */
int  bolt_adj1d_step_adjoint(BoltAdj1D* c, const void* f_n, void* lam, int objective_at_start,
                             double* dtau_dev, void* stream);
/* J_dev += dt |nhat_1(f)|^2; lam (may be null) += its gradient. */
int  bolt_adj1d_objective(BoltAdj1D* c, const void* f, double* J_dev, void* lam, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BOLT_B200_H */
