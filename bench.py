"""Benchmark of the FVM kinetic update on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp32|fp64|fp64-fast] [--small]
                    [--parallelism replicas|slabs] [--workload ...]

Workload (one step = one classic RK4 step over the whole phase space):
  2D3V, N_q1 = N_q2 = 128 on [0,1]^2 periodic, N_p1 = N_p2 = N_p3 = 24 on
  [-6,6]^3 (226,492,416 cells), f0 = Maxwellian (T = 1) with
  n = 1 + 0.05 cos(2 pi q1) cos(2 pi q2), BGK tau = 0.05, fields off,
  WENO5 + LLF, dt = 1e-3; f in FP32 with FP64 moments (both FP64 forms are
  measured as well).  Synthetic data; f (0.99 GB FP32) is larger than L2, so
  no L2 flush is needed between steps.  On one GPU the line also holds the
  benchmark set's other targets (ragged batch, adjoint, 2D2V FDTD).

--impl reference times the FP64 C/OpenMP restatement of the same path
(oracle/bolt_oracle_c.c) on all host cores, on a sample of the workload (the
reference itself is Python over ArrayFire/PETSc and cannot run on the GPU box).

Multi-GPU (torchrun): every rank advances an independent replica of the
workload (no data-path collective); value = cell-updates of all ranks / the
slowest rank's time.  The line's "decomposed" entry times the same workload
as one run cut into q2 slabs over the ranks (strong scaling, peer halos);
--parallelism slabs makes that the line's value.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time
import types

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'cell-updates/s WENO5+LLF RK4: FP64 plain vs FP32/batched/adjoint; % HBM roofline'
UNIT = 'cell-updates/s'
HBM_FALLBACK_GBS = 6650.0
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per stage launch of
# the FP32 workload, averaged over the four RK4 stage kernels of one step:
# measured by ncu on the 64x64 x 24^3 case (959.0 MB per launch) and scaled by
# the 4x cells of 128x128 x 24^3
TRAFFIC_FP32_PER_LAUNCH = 3.836e9


def workload_spec(small=False):
    n = 64 if small else 128
    return dict(
        N_q1=n, N_q2=n, q1_start=0.0, q1_end=1.0, q2_start=0.0, q2_end=1.0, N_ghost=3,
        N_p1=24, N_p2=24, N_p3=24, p1_start=[-6.0], p1_end=[6.0], p2_start=[-6.0],
        p2_end=[6.0], p3_start=[-6.0], p3_end=[6.0], mass=[1.0], charge=[0.0], p_dim=3,
        boltzmann_constant=1.0, tau=0.05, dt=1e-3, recon_q='weno5', recon_p='weno5',
        riemann_q='lax-friedrichs', riemann_p='lax-friedrichs', source_enabled=True,
        fields_enabled=False, fields_type='electrodynamic', fields_initialize='fft',
        fields_solver='fdtd', integrator='RK4', bc_q1='periodic', bc_q2='periodic',
        eps=1.0, mu=1.0, amp=0.05)


def config_modules(spec, precision):
    import torch
    dom = types.ModuleType('domain')
    for k in ('q1_start', 'q1_end', 'q2_start', 'q2_end', 'N_q1', 'N_q2', 'N_p1', 'N_p2',
              'N_p3', 'N_ghost', 'p1_start', 'p1_end', 'p2_start', 'p2_end', 'p3_start',
              'p3_end'):
        setattr(dom, k, spec[k])
    bc = types.ModuleType('boundary_conditions')
    bc.in_q1_left = bc.in_q1_right = 'periodic'
    bc.in_q2_bottom = bc.in_q2_top = 'periodic'
    params = types.ModuleType('params')
    for k, v in dict(fields_type='electrodynamic', fields_initialize='fft', fields_solver='fdtd',
                     solver_method_in_q='FVM', solver_method_in_p='FVM',
                     reconstruction_method_in_q='weno5', reconstruction_method_in_p='weno5',
                     riemann_solver_in_q='lax-friedrichs', riemann_solver_in_p='lax-friedrichs',
                     p_dim=3, num_devices=1, mass=[1.0], charge=[0.0], boltzmann_constant=1.0,
                     fields_enabled=False, source_enabled=True, instantaneous_collisions=False,
                     hybrid_model_enabled=False, eps=1.0, mu=1.0, p_space_grid='cartesian',
                     time_integrator='RK4', precision=precision).items():
        setattr(params, k, v)
    params.tau = lambda q1, q2, p1, p2, p3: spec['tau'] * p1 ** 0 * q1 ** 0
    ini = types.ModuleType('initialize')
    amp = spec['amp']

    def initialize_f(q1, q2, p1, p2, p3, params):
        n = 1 + amp * torch.cos(2 * np.pi * q1) * torch.cos(2 * np.pi * q2)
        m, k = params.mass, params.boltzmann_constant
        T = 1.0
        return n * (m / (2 * np.pi * k * T)) ** 1.5 * torch.exp(-m * p1 ** 2 / (2 * k * T)) \
            * torch.exp(-m * p2 ** 2 / (2 * k * T)) * torch.exp(-m * p3 ** 2 / (2 * k * T))
    ini.initialize_f = initialize_f
    return dom, bc, params, ini


def make_solver(spec, precision):
    from bolt_b200.physical_system import physical_system
    from bolt_b200.nonlinear_solver import nonlinear_solver
    import bolt_b200.src.nonrelativistic_boltzmann.advection_terms as adv
    import bolt_b200.src.nonrelativistic_boltzmann.collision_operator as col
    import bolt_b200.src.nonrelativistic_boltzmann.moments as mom
    dom, bc, params, ini = config_modules(spec, precision)
    return nonlinear_solver(physical_system(dom, bc, params, ini, adv, col.BGK, mom))


def ragged_sweep(nruns=256, seed=0):
    """The ragged 1D1V sweep (seed 0, numpy PCG64): N_q1 uniform over
    {32, 48, ..., 256}, N_p1 over {64, 96, ..., 512}, p1 in [-10, 10],
    tau and the density amplitude log-uniform in [1e-3, 1e-1], wavenumber
    k in {1, 2, 3, 4}; dt = 0.5 dq1 / 10 (CFL 0.5 at |p1| = 10)."""
    rng = np.random.default_rng(seed)
    runs = []
    for _ in range(nruns):
        nq = int(rng.choice(np.arange(32, 257, 16)))
        npp = int(rng.choice(np.arange(64, 513, 32)))
        tau = float(10 ** rng.uniform(-3, -1))
        amp = float(10 ** rng.uniform(-3, -1))
        k = int(rng.integers(1, 5))
        runs.append(dict(N_q1=nq, N_p1=npp, tau=tau, amp=amp, k=k, dt=0.5 * (1.0 / nq) / 10.0))
    return runs


def ragged_system(run, precision='fp32', source=True):
    """Bolt physical_system of one ragged-sweep run: 1D1V, q1 in [0, 1]
    periodic, p1 in [-10, 10], p2 = p3 = [-0.5, 0.5] with one cell, BGK with
    the run's tau, f0 = Maxwellian(T = 1) (1 + A cos(2 pi k q1)), WENO5 + LLF,
    RK4."""
    import torch
    from bolt_b200.physical_system import physical_system
    import bolt_b200.src.nonrelativistic_boltzmann.advection_terms as adv
    import bolt_b200.src.nonrelativistic_boltzmann.collision_operator as col
    import bolt_b200.src.nonrelativistic_boltzmann.moments as mom
    spec = dict(q1_start=0.0, q1_end=1.0, q2_start=0.0, q2_end=1.0, N_q1=run['N_q1'], N_q2=1,
                N_p1=run['N_p1'], N_p2=1, N_p3=1, N_ghost=3, p1_start=[-10.0], p1_end=[10.0],
                p2_start=[-0.5], p2_end=[0.5], p3_start=[-0.5], p3_end=[0.5], tau=run['tau'],
                amp=0.0)
    dom, bc, params, ini = config_modules(spec, precision)
    params.p_dim = 1
    params.source_enabled = source
    amp, k = run['amp'], run['k']

    def initialize_f(q1, q2, p1, p2, p3, params):
        m, kB = params.mass, params.boltzmann_constant
        m = m[0] if isinstance(m, list) else m
        n = 1 + amp * torch.cos(2 * np.pi * k * q1)
        return n * (m / (2 * np.pi * kB)) ** 0.5 * torch.exp(-m * p1 ** 2 / (2 * kB))
    ini.initialize_f = initialize_f
    return physical_system(dom, bc, params, ini, adv, col.BGK, mom)


def interior_cells(spec):
    return spec['N_q1'] * spec['N_q2'] * spec['N_p1'] * spec['N_p2'] * spec['N_p3'] * len(spec['mass'])


def measured_peak():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as fh:
            return float(json.load(fh)['hbm_gbs']), 'measured'
    except Exception:
        return HBM_FALLBACK_GBS, 'fallback'


class ClockSampler(object):
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.index),
                 '--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
                 'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
                 'clocks_event_reasons.sw_power_cap', '--format=csv,noheader,nounits', '-lms', '100'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(',')]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == 'active':
                    reasons.add(nm)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': [], 'samples': 0}
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': max(mx),
                'reasons': sorted(reasons), 'samples': len(sm)}


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), or the platform's."""
    try:
        with open('/proc/cpuinfo') as fh:
            for ln in fh:
                if ln.lower().startswith('model name'):
                    return ln.split(':', 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or platform.machine()


def cpu_sample_spec(spec):
    s = dict(spec)
    s['N_q1'] = s['N_q2'] = 32
    return s


def time_cpu_reference(spec, steps, warmup, threads):
    """FP64 C/OpenMP restatement on a 32x32 x 24^3 sample (periodic)."""
    sys.path.insert(0, os.path.join(ROOT, 'tests', 'golden'))
    from oracle import c_oracle
    c_oracle.build()
    s = cpu_sample_spec(spec)
    Ng = s['N_ghost']
    q1 = (np.arange(-Ng, s['N_q1'] + Ng) + 0.5) / s['N_q1']
    q2 = (np.arange(-Ng, s['N_q2'] + Ng) + 0.5) / s['N_q2']
    p = -6.0 + (0.5 + np.arange(24)) * 0.5
    n = 1 + spec['amp'] * np.cos(2 * np.pi * q1)[None, :] * np.cos(2 * np.pi * q2)[:, None]
    maxw = (2 * np.pi) ** -1.5 * np.exp(-(p[:, None, None] ** 2 + p[None, :, None] ** 2
                                          + p[None, None, :] ** 2) / 2)
    f = np.ascontiguousarray(n[:, :, None, None, None, None] * maxw[None, None, None])
    for _ in range(warmup):
        c_oracle.rk_step(f, s, s['dt'], 4, threads)
    t0 = time.perf_counter()
    for _ in range(steps):
        c_oracle.rk_step(f, s, s['dt'], 4, threads)
    el = time.perf_counter() - t0
    cells = interior_cells(s)
    return cells * steps / el, el / steps, s


def run_reference(args, rank, world):
    spec = workload_spec(args.small)
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    value, sec_per_step, s = time_cpu_reference(spec, args.steps, args.warmup, threads)
    sample = '%dx%d x 24^3 of the workload (periodic), FP64, %d RK4 steps' % (
        s['N_q1'], s['N_q2'], args.steps)
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': UNIT,
        'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': sec_per_step * 1e3, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': 'Bolt FVM 2D3V 128^2 x 24^3 WENO5+LLF RK4 BGK (sampled)',
                   'parallelism': 'cpu-openmp'},
        'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': threads, 'kind': 'port',
                         'cpu_model': cpu_model(), 'sample': sample},
        'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


def max_over_ranks(x, world):
    """The maximum of a per-rank float over all ranks (every rank gets it).
    NCCL reduces on the device, gloo (CPU tests of the multi-rank path) on the
    host."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = 'cuda' if dist.get_backend() == 'nccl' else 'cpu'
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(cells_per_rank, world, ms_max):
    """Whole-job cell-updates/s: every rank advances its own replica of the
    workload, the slowest rank's time per step bounds the job."""
    return cells_per_rank * world / (ms_max * 1e-3)


def slab_result(args, rank, world, local_rank, spec):
    """The same run cut into ``world`` q2 slabs, one per rank (SlabSolver: the
    reference's DMDA split, nonlinear_solver.py:251-280), strong scaling:
    with a process group the stage kernels store their boundary rows straight
    into the neighbouring GPUs' buffers (peer halos over NVLink, CUDA IPC) and
    the ranks order their stages with a one-element all-reduce; a single
    process steps one slab whose halo wraps onto itself.  Time per step is
    the slowest rank's (CUDA events), value = the whole run's cells / time."""
    import torch
    import torch.distributed as dist
    from bolt_b200.distributed import SlabSolver
    from bolt_b200.physical_system import physical_system
    import bolt_b200.src.nonrelativistic_boltzmann.advection_terms as adv
    import bolt_b200.src.nonrelativistic_boltzmann.collision_operator as col
    import bolt_b200.src.nonrelativistic_boltzmann.moments as mom
    dom, bc, params, ini = config_modules(spec, args.precision)
    slab = SlabSolver(physical_system(dom, bc, params, ini, adv, col.BGK, mom))
    peer = world > 1 and dist.is_initialized()
    peer_error = None
    if peer:
        # every rank takes the same halo path: if mapping a neighbour's
        # buffers fails on any rank, all fall back to the send/recv exchange
        ok = 1
        try:
            slab.enable_peer_halos()
        except Exception as exc:                       # noqa: BLE001
            ok, peer_error = 0, '%s: %s' % (type(exc).__name__, str(exc)[:200])
        flag = torch.tensor([ok], dtype=torch.int32, device='cuda')
        dist.all_reduce(flag, op=dist.ReduceOp.MIN)
        if int(flag.item()) == 0:
            slab.disable_peer_halos()
            peer = False
    dt = spec['dt']
    for _ in range(args.warmup):
        slab.strang_timestep(dt)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = slab.local.launch_count()
    paired0 = slab.local.paired_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        slab.strang_timestep(dt)
    e1.record()
    e1.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    launches = slab.local.launch_count() - launches0
    paired = slab.local.paired_launch_count() - paired0
    slab.local.synchronize()
    if peer:
        dist.barrier()
        slab.disable_peer_halos()
    cells = interior_cells(spec)
    return {'value': cells / (ms * 1e-3), 'ms_per_step': ms, 'scaling': 'strong',
            'slabs': world, 'rows_per_slab': spec['N_q2'] // world,
            'halos': 'peer stores over NVLink' if peer else
                     ('send/recv exchange, overlapped with the inner tiles' if world > 1 else
                      'single slab (wraps onto itself), exchange overlapped with the inner tiles'),
            'peer_halo_error': peer_error,
            'gpu_launches_per_rank': launches,
            'paired_launches_per_rank': paired}


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    spec = workload_spec(args.small)
    cells = interior_cells(spec)
    dt = spec['dt']
    if args.parallelism == 'slabs':
        res = slab_result(args, rank, world, local_rank, spec)
        if rank == 0:
            print(json.dumps({
                'metric': METRIC, 'value': res['value'], 'unit': UNIT, 'n_gpus': world,
                'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': res['ms_per_step'],
                'higher_is_better': True, 'scaling': 'strong', 'vs_baseline': None,
                'dtype': 'f32' if args.precision == 'fp32' else 'f64', 'data': 'synthetic',
                'config': {'workload': '2D3V %dx%d x 24^3, one run in %d q2 slabs'
                                       % (spec['N_q1'], spec['N_q2'], world),
                           'parallelism': 'q2-slabs'},
                'decomposed': res, 'gpu_launches': res['gpu_launches_per_rank']}), flush=True)
        return
    nls = make_solver(spec, args.precision)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        nls.strang_timestep(dt)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = nls.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        time.sleep(0.3)
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(args.steps):
            nls.strang_timestep(dt)
        ev1.record()
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    launches = nls.launch_count() - launches0
    torch.cuda.synchronize()
    # density and energy after warmup + steps, for the FP32-vs-FP64 check
    g = spec['N_ghost']
    mom32 = {k: nls.compute_moments(k)[..., g:-g, g:-g].clone() for k in ('density', 'energy')}
    ms = max_over_ranks(ms, world)
    if world > 1:
        dist.barrier()
    value = job_value(cells, world, ms)

    # end-to-end through the public API with host buffers: every step copies
    # its input f from pinned host memory and its result f back.  The copies
    # are pipelined over two streams and two staging buffers per direction:
    # the input goes host -> device staging on one stream, the public setter
    # (nls.f = ...) moves it into the solver, the step runs, the result is
    # copied device -> device staging and then -> host on the other stream.
    # With two buffers each way the uploads run back to back, the downloads
    # run back to back (PCIe is full duplex), and the solver never waits on a
    # host copy except for its own input.
    host_in = torch.empty_like(nls._fstore, device='cpu').pin_memory()
    host_in.copy_(nls._fstore)
    host_out = torch.empty_like(host_in).pin_memory()
    stage_in = [torch.empty_like(nls._fstore) for _ in range(2)]
    stage_out = [torch.empty_like(nls._fstore) for _ in range(2)]
    main = torch.cuda.current_stream()
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in, ev_used, ev_ready, ev_freed = ([torch.cuda.Event() for _ in range(2)]
                                          for _ in range(4))
    e2e_steps = max(1, min(args.steps, 30))   # amortises the pipeline fill and drain
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for ev in ev_used + ev_freed:
        ev.record(main)
    e0.record(main)
    s_in.wait_stream(main)
    s_out.wait_stream(main)
    for k in range(e2e_steps):
        b = k % 2
        s_in.wait_event(ev_used[b])                  # the input two steps back was consumed
        with torch.cuda.stream(s_in):
            stage_in[b].copy_(host_in, non_blocking=True)
            ev_in[b].record(s_in)
        main.wait_event(ev_in[b])
        nls.f = stage_in[b].permute(3, 2, 1, 0)      # the public setter
        ev_used[b].record(main)
        nls.strang_timestep(dt)
        main.wait_event(ev_freed[b])                 # the download two steps back is done
        stage_out[b].copy_(nls._fstore)
        ev_ready[b].record(main)
        s_out.wait_event(ev_ready[b])
        with torch.cuda.stream(s_out):
            host_out.copy_(stage_out[b], non_blocking=True)
            ev_freed[b].record(s_out)
    main.wait_stream(s_out)
    e1.record(main)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    # the copies alone, both directions at once on the same pinned buffers:
    # the PCIe floor of one end-to-end step
    torch.cuda.synchronize()
    e0.record(main)
    s_in.wait_stream(main)
    s_out.wait_stream(main)
    for k in range(e2e_steps):
        with torch.cuda.stream(s_in):
            stage_in[k % 2].copy_(host_in, non_blocking=True)
        with torch.cuda.stream(s_out):
            host_out.copy_(stage_out[k % 2], non_blocking=True)
    main.wait_stream(s_in)
    main.wait_stream(s_out)
    e1.record(main)
    e1.synchronize()
    copy_ms = e0.elapsed_time(e1) / e2e_steps
    e2e_ms = max_over_ranks(e2e_ms, world)
    copy_ms = max_over_ranks(copy_ms, world)
    fbytes = host_in.numel() * host_in.element_size()
    e2e = {'value': job_value(cells, world, e2e_ms), 'unit': UNIT,
           'h2d_bytes_per_step': fbytes, 'd2h_bytes_per_step': fbytes,
           'ms_per_step': e2e_ms,
           # floor: the same host<->device bytes copied with nothing else running
           'copy_floor_ms_per_step': copy_ms,
           'frac_of_copy_floor': copy_ms / e2e_ms,
           'pcie_gbs_per_direction': fbytes / (copy_ms * 1e-3) / 1e9}

    # the FP64 forms of the same workload, reported beside the FP32 number:
    # 'fp64' keeps the reference's operation order (-fmad=false, IEEE
    # divisions; the 1e-12 parity path), 'fp64-fast' runs the paired kernel's
    # FP64 form (one q-row per thread) with FMA and Newton-refined reciprocals
    fp64 = fp64f = None
    if args.precision == 'fp32' and not args.no_fp64:
        del host_in, host_out, stage_in, stage_out
        res = {}
        for form in ('fp64', 'fp64-fast'):
            nls64 = make_solver(spec, form)
            for _ in range(args.warmup):
                nls64.strang_timestep(dt)
            torch.cuda.synchronize()
            a0 = torch.cuda.Event(enable_timing=True)
            a1 = torch.cuda.Event(enable_timing=True)
            n64 = max(1, args.steps // 2)
            a0.record()
            for _ in range(n64):
                nls64.strang_timestep(dt)
            a1.record()
            a1.synchronize()
            ms64 = max_over_ranks(a0.elapsed_time(a1) / n64, world)
            # untimed steps up to the FP32 run's count, for the error checks
            for _ in range(args.steps - n64):
                nls64.strang_timestep(dt)
            mom = {k: nls64.compute_moments(k)[..., g:-g, g:-g].clone() for k in mom32}
            res[form] = (ms64, mom, nls64.paired_launch_count())
            del nls64
            torch.cuda.empty_cache()
        ms64, mom64, _ = res['fp64']
        msf, momf, pairf = res['fp64-fast']
        err = lambda got: {k: float((got[k] - v64).norm() / v64.norm()) for k, v64 in mom64.items()}
        peak, _ = measured_peak()
        fp64 = {'value': job_value(cells, world, ms64), 'ms_per_step': ms64,
                'bytes_per_cell_update': 136,
                'hbm_frac': 136 * cells / (ms64 * 1e-3) / (peak * 1e9),
                'kernel': 'qstage_kernel<double> (reference operation order, -fmad=false)',
                'fp32_rel_l2_error_vs_fp64': err(mom32),
                'fp32_over_fp64': ms64 / ms,
                'error_after_steps': args.warmup + args.steps}
        fp64f = {'value': job_value(cells, world, msf), 'ms_per_step': msf,
                 'bytes_per_cell_update': 136,
                 'hbm_frac': 136 * cells / (msf * 1e-3) / (peak * 1e9),
                 'kernel': 'qpair_kernel<double> (one q-row per thread, FMA, Newton-refined reciprocals)',
                 'paired_launches': pairf,
                 'rel_l2_error_vs_fp64': err(momf),
                 'fp32_over_fp64_fast': msf / ms,
                 'speedup_vs_fp64': ms64 / msf,
                 'error_after_steps': args.warmup + args.steps}

    # with several ranks: the same workload as one run cut into q2 slabs
    # (strong scaling), beside the replicas of the headline
    decomposed = None
    if world > 1 and not args.no_decompose:
        # the headline above stands whatever happens here: a failure of the
        # slab split (e.g. peer mappings refused between the GPUs) is recorded
        # in the line instead of ending the run
        try:
            decomposed = slab_result(args, rank, world, local_rank, spec)
        except Exception as exc:                       # noqa: BLE001
            decomposed = {'error': '%s: %s' % (type(exc).__name__, str(exc)[:300])}
            torch.cuda.synchronize()

    # the benchmark set's other targets, on one GPU (kept out of the scaling runs)
    targets = None
    if world == 1 and not args.no_extras:
        f_gb = nls._fstore.numel() * (4 if args.precision == 'fp32' else 8) / 1e9
        del nls
        torch.cuda.empty_cache()
        targets = other_targets(args, local_rank)
    else:
        f_gb = nls._fstore.numel() * (4 if args.precision == 'fp32' else 8) / 1e9

    if rank != 0:
        return
    word = 4 if args.precision == 'fp32' else 8
    # algorithmic bytes per cell-update of classic RK4 with the combine and the
    # moments fused: 3 + 5 + 5 + 4 = 17 words (the stages read/write f, k-stage
    # inputs and the accumulator); this implementation moves 16 (the last stage
    # reads the accumulator as its only base)
    alg_bytes_per_update = 17 * word
    peak, peak_kind = measured_peak()
    launches_per_step = launches / args.steps
    qstage_per_step = 4.0                      # one fused stage kernel per RK4 stage
    achieved = alg_bytes_per_update * cells / (ms * 1e-3) / 1e9
    traffic = args.traffic
    if traffic is None and args.precision == 'fp32' and not args.small:
        traffic = TRAFFIC_FP32_PER_LAUNCH
    roofline = {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                'frac': achieved / peak, 'traffic': traffic,
                'peak_kind': peak_kind,
                'kernel': 'qpair_kernel (paired FP32 WENO5 RK stage, 8x8 q-tile)'
                if args.precision == 'fp32' else 'qstage_kernel (WENO5, 8x8 q-tile)',
                'alg_bytes_per_update': alg_bytes_per_update,
                'alg_bytes_per_launch': alg_bytes_per_update * cells / qstage_per_step,
                'avg_launch_ms': ms / qstage_per_step}
    cpu = None
    if world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        v, sps, s = time_cpu_reference(spec, 2, 1, threads)
        cpu = {'value': v, 'unit': UNIT, 'cores': threads, 'kind': 'port',
               'cpu_model': cpu_model(),
               'sample': '%dx%d x 24^3 of the workload, FP64 C/OpenMP restatement, 2 RK4 steps'
                         % (s['N_q1'], s['N_q2'])}
    line = {
        'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f32' if args.precision == 'fp32' else 'f64',
        'data': 'synthetic',
        'config': {'workload': '2D3V %dx%d x 24^3 (%d cells) Maxwellian n=1+0.05cos(2pi q1)cos(2pi q2),'
                               ' BGK tau=0.05, WENO5+LLF, RK4, dt=1e-3, %s f + FP64 moments'
                               % (spec['N_q1'], spec['N_q2'], cells, args.precision.upper()),
                   'cells': cells, 'l2': 'inputs larger than L2 (f %.2f GB), no flush' % f_gb,
                   'parallelism': 'replicas' if world > 1 else 'single'},
        'roofline': roofline,
        'cpu_baseline': cpu,
        'e2e': e2e,
        'gpu_launches': launches,
        'launches_per_step': launches_per_step,
        'clocks': clk.summary(),
        'fp64_plain': fp64,
        'fp64_fast': fp64f,
        'decomposed': decomposed,
        'targets': targets,
    }
    print(json.dumps(line), flush=True)


def other_targets(args, local_rank):
    """The benchmark set's other targets, measured after the headline so the
    default run records them: the ragged 256-run batch against sequential
    plain runs (target >= 5x), the adjoint's gradient time and its checks
    against central differences and FP64 autograd (target 1e-4), and the
    FDTD-coupled 2D2V run's FP32 / FP64 throughput ratio, and the
    semi-Lagrangian q-step on the headline grid.  Each entry is
    measured as its own --workload measures it (see batch_result,
    adjoint_result, c2_result); sequential runs time --seq-steps steps each,
    scaled to the batch's step count."""
    import torch
    out = {}
    t0 = time.perf_counter()
    b = batch_result(args, 1, local_rank, seq_steps=args.seq_steps)
    out['ragged_batch'] = {k: b[k] for k in ('value', 'sequential_value', 'speedup_vs_sequential',
                                             'batch_s', 'sequential_s', 'sequential_steps_timed',
                                             'schedule', 'steps')}
    out['ragged_batch']['runs'] = b['config']['runs']
    out['ragged_batch']['cells'] = b['config']['cells']
    out['ragged_batch']['stage_kernel_hbm_frac'] = b['roofline']['frac']
    torch.cuda.empty_cache()
    t1 = time.perf_counter()
    a = adjoint_result(args, local_rank, autograd_steps=args.autograd_steps)
    c = a['check']
    out['adjoint'] = {'gradient_s': a['value'], 'forward_s': a['forward_s'],
                      'forward_to_gradient': a['forward_to_gradient'], 'steps': a['steps'],
                      'recomputed_steps': a['recomputed_steps'],
                      'fp64_gradient_s': a['fp64']['gradient_s'],
                      'rel_fp64_vs_fd': c['rel_fp64_vs_fd'],
                      'autograd_steps': c['autograd_steps'],
                      'rel_fp64_vs_autograd': c['rel_fp64_vs_autograd'],
                      'rel_fp32_vs_fp64': c['rel_fp32_vs_fp64']}
    torch.cuda.empty_cache()
    t2 = time.perf_counter()
    c2 = c2_result(args, local_rank)
    out['c2_fdtd'] = {'fp32_over_fp64': c2['fp32_over_fp64'], 'fp32_value': c2['fp32']['value'],
                      'fp64_value': c2['fp64']['value'], 'steps': c2['steps'],
                      'fp32_vs_fp64_after_steps': c2['fp32_vs_fp64_after_steps']}
    t3 = time.perf_counter()
    out['asl_q'] = asl_result(args, local_rank)
    t4 = time.perf_counter()
    out['wall_s'] = {'ragged_batch': t1 - t0, 'adjoint': t2 - t1, 'c2_fdtd': t3 - t2,
                     'asl_q': t4 - t3}
    return out


def batch_result(args, world, local_rank, seq_steps=None):
    """The ragged 1D1V sweep: all runs advanced by BatchSolver (one launch per
    RK stage over the packed runs, the steps replayed as one CUDA graph)
    against the same runs advanced one after another by nonlinear_solver
    (sequential plain runs, same FP32 f + FP64 moments), both timed with CUDA
    events; value = total cell-updates/s of the batch.  With seq_steps, each
    sequential run times seq_steps steps and its time is scaled to the
    batch's step count (a plain run's step time does not change from step to
    step: every step launches the same kernels)."""
    import torch
    from bolt_b200.batch import BatchSolver
    from bolt_b200.nonlinear_solver import nonlinear_solver
    torch.cuda.set_device(local_rank)
    runs = ragged_sweep(args.batch_runs)
    nsteps = args.batch_steps
    cells = sum(r['N_q1'] * r['N_p1'] for r in runs)
    fixed = [int(x) for x in args.batch_schedule.split(',')] if args.batch_schedule else None
    bs = BatchSolver([ragged_system(r) for r in runs], [r['dt'] for r in runs],
                     autotune=fixed is None)
    if fixed:
        bs.set_schedule(*fixed)
    bs.run(nsteps)                       # warm-up: autotunes, captures the graph
    bs.synchronize()
    tuning = bs.tuning
    eff = bs.schedule()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    bs.run(nsteps)
    e1.record()
    e1.synchronize()
    t_batch = e0.elapsed_time(e1) * 1e-3
    bs.synchronize()
    del bs
    # sequential plain runs: each run constructed, then its steps timed
    ns = nsteps if seq_steps is None else min(seq_steps, nsteps)
    t_seq = 0.0
    for r in runs:
        nls = nonlinear_solver(ragged_system(r))
        for _ in range(2):
            nls.strang_timestep(r['dt'])
        torch.cuda.synchronize()
        e0.record()
        for _ in range(ns):
            nls.strang_timestep(r['dt'])
        e1.record()
        e1.synchronize()
        t_seq += e0.elapsed_time(e1) * 1e-3 * nsteps / ns
        del nls
    t_batch = max_over_ranks(t_batch, world)
    t_seq = max_over_ranks(t_seq, world)
    value = job_value(cells * nsteps, world, t_batch * 1e3)
    seq = job_value(cells * nsteps, world, t_seq * 1e3)
    line = {
        'metric': 'cell-updates/s ragged 1D1V batch (one launch per RK stage, CUDA graph) '
                  'vs sequential plain runs', 'value': value, 'unit': UNIT,
        'n_gpus': world, 'steps': nsteps, 'higher_is_better': True, 'scaling': 'weak',
        'dtype': 'f32', 'data': 'synthetic',
        'config': {'workload': '%d ragged 1D1V runs (seed 0): N_q1 in {32..256}, N_p1 in '
                               '{64..512}, tau, amplitude log-uniform [1e-3, 1e-1], k in 1..4, '
                               'WENO5+LLF, RK4, dt = 0.5 dq1/10, FP32 f + FP64 moments'
                               % len(runs), 'cells': cells, 'runs': len(runs)},
        'batch_s': t_batch, 'sequential_s': t_seq, 'sequential_value': seq,
        'sequential_steps_timed': ns,
        'speedup_vs_sequential': t_seq / t_batch,
        # launch schedule picked by the batch's autotuner before the timed run
        'schedule': tuning['chosen'] if tuning else
        {'tile_cells': eff[0], 'ctas': eff[1], 'lpt_order': eff[2], 'fixed': True},
        'schedules_timed': len(tuning['candidates']) if tuning else 0,
        # four batch_stage_kernel launches per step (the graph's only kernels)
        'gpu_launches': 4 * nsteps,
    }
    # the stage kernel against HBM at the RK4 FP32 figure of 68 B per update
    # (17 B per cell per stage launch); the packed f and its three stage
    # buffers (~4 x 44 MB) are largely L2-resident, so this fraction
    # understates the kernel's memory-side headroom
    peak, kind = measured_peak()
    launch_s = t_batch / (4 * nsteps)
    achieved = cells * (17 * 4 / 4.0) / launch_s / 1e9
    line['roofline'] = {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                        'frac': achieved / peak, 'traffic': None, 'peak_kind': kind,
                        'kernel': 'batch_stage_kernel', 'avg_launch_ms': launch_s * 1e3,
                        'note': 'working set comparable to L2 (126 MB)'}
    return line


def run_batch(args, rank, world, local_rank):
    line = batch_result(args, world, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)


def adjoint_result(args, local_rank, autograd_steps=None):
    """Adjoint workload: gradients of J = sum_n dt |nhat_1(n)|^2 for 1D1V 128 x 256,
    p1 in [-10, 10], n = 1 + a cos(2 pi q1) (a = 0.01), Maxwellian T = 1,
    tau = 0.02, RK4, dt = 2e-4, 2000 steps, binomial checkpointing with 20
    snapshots; FP32 f with FP64 moments.  Reports the forward and gradient
    wall times (CUDA events), and checks dJ/dtau and dJ/da against central
    differences (h = 1e-4, FP64 forward) and dJ/d(f0, tau, a) against FP64
    autograd of the PyTorch transcription of the reference scheme."""
    import math
    import torch
    from bolt_b200.adjoint import Rollout1D1V, rollout
    torch.cuda.set_device(local_rank)
    NQ, NP, P0, P1, TAU, DT, STEPS, AMP = 128, 256, -10.0, 10.0, 0.02, 2e-4, args.adj_steps, 0.01
    dev = torch.device('cuda', local_rank)
    x = ((0.5 + torch.arange(NQ, dtype=torch.float64, device=dev)) / NQ)[:, None]
    v = (P0 + (0.5 + torch.arange(NP, dtype=torch.float64, device=dev)) * (P1 - P0) / NP)[None, :]
    maxw = torch.exp(-v ** 2 / 2) / math.sqrt(2 * math.pi)
    f_of = lambda a: (1 + a * torch.cos(2 * math.pi * x)) * maxw
    ev = lambda: torch.cuda.Event(enable_timing=True)
    out = {}
    for prec in ('fp32', 'fp64'):
        r = Rollout1D1V(NQ, NP, P0, P1, DT, TAU, STEPS, snapshots=20, precision=prec)
        a = torch.tensor(AMP, dtype=torch.float64, device=dev, requires_grad=True)
        tau = torch.tensor(TAU, dtype=torch.float64, device=dev, requires_grad=True)
        r.forward(f_of(AMP))                             # warm-up
        e0, e1, e2 = ev(), ev(), ev()
        e0.record()
        J = rollout(f_of(a), tau, r)
        e1.record()
        J.backward()
        e2.record()
        e2.synchronize()
        gf, _ = r.gradient(f_of(AMP))
        out[prec] = dict(J=float(J), da=float(a.grad), dtau=float(tau.grad), gf=gf.double(),
                         fwd_s=e0.elapsed_time(e1) * 1e-3, grad_s=e1.elapsed_time(e2) * 1e-3,
                         recomputed_steps=r.forward_steps)
        if prec == 'fp64':
            h = 1e-4
            Jf = lambda aa, tt: float(r.forward(f_of(aa), tt)[0])
            out['fd_da'] = (Jf(AMP * (1 + h), TAU) - Jf(AMP * (1 - h), TAU)) / (2 * AMP * h)
            out['fd_dtau'] = (Jf(AMP, TAU * (1 + h)) - Jf(AMP, TAU * (1 - h))) / (2 * TAU * h)
    # FP64 autograd of the transcription (checkpointed every 50 steps), over
    # the whole horizon or, with autograd_steps, a shorter one (the FP64
    # adjoint is then evaluated over that horizon as well)
    sys.path.insert(0, ROOT)
    from oracle.bolt_torch import Problem1D1V
    AG = STEPS if not autograd_steps else min(autograd_steps, STEPS)
    o64ag = out['fp64']
    if AG != STEPS:
        r = Rollout1D1V(NQ, NP, P0, P1, DT, TAU, AG, snapshots=20, precision='fp64')
        a = torch.tensor(AMP, dtype=torch.float64, device=dev, requires_grad=True)
        tau = torch.tensor(TAU, dtype=torch.float64, device=dev, requires_grad=True)
        rollout(f_of(a), tau, r).backward()
        o64ag = dict(da=float(a.grad), dtau=float(tau.grad), gf=r.gradient(f_of(AMP))[0].double())
    pr = Problem1D1V(NQ, NP, P0, P1, DT, TAU, device=dev)
    a = torch.tensor(AMP, dtype=torch.float64, device=dev, requires_grad=True)
    tau = torch.tensor(TAU, dtype=torch.float64, device=dev, requires_grad=True)
    f0 = f_of(a)
    f0.retain_grad()
    Jt, _ = pr.objective(f0, tau, AG, checkpoint_every=50)
    Jt.backward()
    rel = lambda x, y: abs(x - y) / abs(y)
    o32, o64 = out['fp32'], out['fp64']
    line = {
        'metric': 'adjoint of the 1D1V WENO5+LLF RK4 BGK update: gradient wall time',
        'value': o32['grad_s'], 'unit': 's', 'higher_is_better': False, 'n_gpus': 1,
        'steps': STEPS, 'dtype': 'f32', 'data': 'synthetic',
        'config': {'workload': '1D1V 128 x 256, p1 in [-10, 10], n = 1 + 0.01 cos(2 pi q1), '
                               'tau = 0.02, dt = 2e-4, %d RK4 steps, J = sum dt |nhat_1|^2, '
                               '20 snapshots (binomial checkpointing)' % STEPS},
        'J': o32['J'], 'forward_s': o32['fwd_s'], 'forward_to_gradient': o32['grad_s'] / o32['fwd_s'],
        'recomputed_steps': o32['recomputed_steps'],
        'fp64': {'J': o64['J'], 'forward_s': o64['fwd_s'], 'gradient_s': o64['grad_s']},
        'check': {
            'dJ_da': {'fp64_adjoint': o64['da'], 'central_difference': out['fd_da'],
                      'fp32_adjoint': o32['da']},
            'dJ_dtau': {'fp64_adjoint': o64['dtau'], 'central_difference': out['fd_dtau'],
                        'fp32_adjoint': o32['dtau']},
            'autograd_steps': AG,
            'autograd_fp64': {'dJ_da': float(a.grad), 'dJ_dtau': float(tau.grad),
                              'fp64_adjoint_da': o64ag['da'], 'fp64_adjoint_dtau': o64ag['dtau']},
            'rel_fp64_vs_fd': {'a': rel(o64['da'], out['fd_da']), 'tau': rel(o64['dtau'], out['fd_dtau'])},
            'rel_fp64_vs_autograd': {'a': rel(o64ag['da'], float(a.grad)),
                                     'tau': rel(o64ag['dtau'], float(tau.grad)),
                                     'f0': float((o64ag['gf'] - f0.grad).norm() / f0.grad.norm())},
            'rel_fp32_vs_fp64': {'a': rel(o32['da'], o64['da']), 'tau': rel(o32['dtau'], o64['dtau']),
                                 'f0': float((o32['gf'] - o64['gf']).norm() / o64['gf'].norm())},
        },
    }
    return line


def run_adjoint(args, rank, world, local_rank):
    line = adjoint_result(args, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)


def c2_spec():
    """2D2V FDTD-coupled workload: [0,1]^2 periodic, 64 x 64 q, p1, p2 in [-8, 8] with
    32 x 32, p3 one cell in [-0.5, 0.5], p_dim 2; f0 = n_q exp(-p1^2/4 - p2^2/2)
    / (2 pi sqrt 2), n_q = 1 + 1e-3 xi_q with xi ~ N(0, 1) per q-cell from
    numpy.random.default_rng(0); collisionless, electrodynamic FDTD with the
    fields of the FFT solve of the noise density, charge -1, m = eps = mu =
    k = 1, WENO5 + LLF, RK4, dt = 5e-4."""
    sys.path.insert(0, os.path.join(ROOT, 'tests'))
    sys.path.insert(0, os.path.join(ROOT, 'tests', 'golden'))
    import cases as C
    return C.make(N_q1=64, N_q2=64, N_p1=32, N_p2=32, N_p3=1,
                  p1_start=[-8.0], p1_end=[8.0], p2_start=[-8.0], p2_end=[8.0],
                  p3_start=[-0.5], p3_end=[0.5], mass=[1.0], charge=[-1.0], p_dim=2,
                  source_enabled=False, fields_enabled=True, dt=5e-4, integrator='RK4',
                  riemann_q='lax-friedrichs', riemann_p='lax-friedrichs',
                  init=dict(amp=0.0, noise=1e-3, seed=0, T=[2.0, 1.0, 1.0]))


def run_c1(args, rank, world, local_rank):
    """1D1V BGK relaxation (64 x 128, WENO5, RK2, dt = 1e-4, 100 steps, FP64): 8,192
    cells, so a step is launch-latency bound.  Times 100 steps three ways:
    Python strang_timestep calls, nls.run(dt, 100) (the C loop of bolt_run),
    and one replay of a CUDA graph captured around nls.run."""
    import torch
    c2_spec()                            # puts the case builders on sys.path
    import cases as C
    from _modules import make_solver as make_case_solver
    torch.cuda.set_device(local_rank)
    spec = C.CASES['c1_1d1v_weno5_rk2']
    cells = spec['N_q1'] * spec['N_p1']
    n, dt = spec['steps'], spec['dt']
    nls = make_case_solver(spec, 'fp64')
    ev = lambda: torch.cuda.Event(enable_timing=True)
    res = {}
    for _ in range(3):
        nls.strang_timestep(dt)
    e0, e1 = ev(), ev()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(n):
        nls.strang_timestep(dt)
    e1.record()
    e1.synchronize()
    res['python_loop_ms_per_step'] = e0.elapsed_time(e1) / n
    nls.run(dt, n)
    torch.cuda.synchronize()
    e0.record()
    nls.run(dt, n)
    e1.record()
    e1.synchronize()
    res['bolt_run_ms_per_step'] = e0.elapsed_time(e1) / n
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        nls.run(dt, n)                    # warm-up on the capture stream
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    with torch.cuda.graph(g):
        nls.run(dt, n)
    g.replay()
    torch.cuda.synchronize()
    e0.record()
    g.replay()
    e1.record()
    e1.synchronize()
    res['cuda_graph_ms_per_step'] = e0.elapsed_time(e1) / n
    del g
    if rank != 0:
        return
    line = {'metric': 'cell-updates/s 1D1V 64x128 WENO5 RK2 FP64, launch-bound',
            'value': cells / (res['cuda_graph_ms_per_step'] * 1e-3), 'unit': UNIT, 'n_gpus': 1,
            'steps': n, 'higher_is_better': True, 'dtype': 'f64', 'data': 'synthetic',
            'config': {'workload': '1D1V 64 x 128, n = 1 + 0.01 cos(2 pi q1), tau = '
                                   '0.01, WENO5, RK2, dt = 1e-4', 'cells': cells},
            }
    line.update({k: v for k, v in res.items()})
    line['python_loop_value'] = cells / (res['python_loop_ms_per_step'] * 1e-3)
    line['bolt_run_value'] = cells / (res['bolt_run_ms_per_step'] * 1e-3)
    print(json.dumps(line), flush=True)


def asl_result(args, local_rank, steps=10):
    """The semi-Lagrangian q-step (solver_method_in_q = 'ASL', Strang
    splitting of the bicubic q-advection and the RK2 BGK source) on the
    headline grid, 2D3V 128^2 x 24^3 (Maxwellian, n = 1 + 0.05 cos cos, BGK
    tau = 0.05, dt = 1e-3), FP32 and FP64 f: cell-updates/s over ``steps``
    timed steps (CUDA events) after 3 warm-up steps.  --small: 64^2 x 24^3
    (for profiler captures)."""
    import torch
    c2_spec()                            # puts the case builders on sys.path
    import cases as C
    from _modules import make_solver as make_case_solver
    torch.cuda.set_device(local_rank)
    n = 64 if getattr(args, 'small', False) else 128
    spec = C.make(N_q1=n, N_q2=n, N_p1=24, N_p2=24, N_p3=24,
                  p1_start=[-6.0], p1_end=[6.0], p2_start=[-6.0], p2_end=[6.0],
                  p3_start=[-6.0], p3_end=[6.0], mass=[1.0], charge=[0.0], p_dim=3,
                  solver_q='ASL', splitting='strang', tau=0.05, dt=1e-3,
                  init=dict(amp=0.05, k1=1, k2=1))
    cells = n * n * 24 ** 3
    out = {'steps': steps, 'splitting': 'strang', 'cells': cells}
    for prec in ('fp32', 'fp64'):
        nls = make_case_solver(spec, prec)
        for _ in range(3):
            nls.strang_timestep(spec['dt'])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            nls.strang_timestep(spec['dt'])
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[prec] = {'value': cells / (ms * 1e-3), 'ms_per_step': ms}
        nls.synchronize()
        del nls
        torch.cuda.empty_cache()
    return out


def c2_result(args, local_rank):
    """2D2V FDTD-coupled workload, FP64 and FP32 f (FP64 moments): cell-updates/s over the timed
    steps (CUDA events) and, after all steps, the FP32 error in density,
    energy and the cell-centred fields against the FP64 run."""
    import torch
    spec = c2_spec()                     # also puts the case builders on sys.path
    from _modules import make_solver as make_case_solver, moments_layout
    torch.cuda.set_device(local_rank)
    cells = spec['N_q1'] * spec['N_q2'] * spec['N_p1'] * spec['N_p2']
    res, state = {}, {}
    for prec in ('fp64', 'fp32'):
        nls = make_case_solver(spec, prec)
        for _ in range(args.warmup):
            nls.strang_timestep(spec['dt'])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.c2_steps - args.warmup):
            nls.strang_timestep(spec['dt'])
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / (args.c2_steps - args.warmup)
        res[prec] = {'value': cells / (ms * 1e-3), 'ms_per_step': ms,
                     'launches_per_step': None}
        g = spec['N_ghost']
        state[prec] = {k: moments_layout(nls.compute_moments(k))[g:-g, g:-g]
                       for k in ('density', 'energy')}
        state[prec]['fields'] = nls.fields_solver.cell_centered_EM_fields[:, 0, g:-g, g:-g] \
            .detach().cpu().numpy()
        del nls
        torch.cuda.empty_cache()
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    line = {
        'metric': 'cell-updates/s 2D2V FDTD-coupled WENO5+LLF RK4, FP32 vs FP64',
        'value': res['fp32']['value'], 'unit': UNIT, 'n_gpus': 1, 'steps': args.c2_steps,
        'higher_is_better': True, 'dtype': 'f32', 'data': 'synthetic (seed 0 noise)',
        'config': {'workload': '2D2V 64^2 x 32^2, FDTD fields, collisionless, dt = 5e-4',
                   'cells': cells},
        'fp32': res['fp32'], 'fp64': res['fp64'],
        'fp32_over_fp64': res['fp32']['value'] / res['fp64']['value'],
        'fp32_vs_fp64_after_steps': {
            'density': rel(state['fp32']['density'], state['fp64']['density']),
            'energy': rel(state['fp32']['energy'], state['fp64']['energy']),
            'fields': rel(state['fp32']['fields'], state['fp64']['fields'])},
    }
    return line


def run_asl(args, rank, world, local_rank):
    line = {'metric': 'cell-updates/s, semi-Lagrangian q-step (Strang split with the BGK '
                      'source)', 'unit': 'cell-updates/s', 'higher_is_better': True,
            'data': 'synthetic', 'n_gpus': 1}
    line.update(asl_result(args, local_rank, steps=args.steps))
    line['value'] = line['fp32']['value']
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_c2(args, rank, world, local_rank):
    line = c2_result(args, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=30)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--precision', default='fp32', choices=['fp32', 'fp64', 'fp64-fast'])
    ap.add_argument('--small', action='store_true', help='64x64 x 24^3 (profiling size)')
    ap.add_argument('--no-cpu', action='store_true')
    ap.add_argument('--no-fp64', action='store_true')
    ap.add_argument('--workload', default='2d3v',
                    choices=['2d3v', '1d1v-relax', '2d2v-fdtd', 'ragged-batch', 'adjoint',
                             'asl-q', 'c3', 'c1', 'c2'],
                    help='2d3v: the 128^2 x 24^3 BGK throughput headline; 1d1v-relax: the '
                         '64 x 128 FP64 relaxation (launch-bound); 2d2v-fdtd: the 64^2 x 32^2 '
                         'FDTD-coupled run, FP32 vs FP64; ragged-batch: the 1D1V sweep; adjoint: '
                         'gradients of the 1D1V density-mode functional; asl-q: the '
                         'semi-Lagrangian q-step on the 128^2 x 24^3 grid (c3, c1, c2: short names '
                         'of the first three)')
    ap.add_argument('--adj-steps', type=int, default=2000)
    ap.add_argument('--c2-steps', type=int, default=500, help='steps of the 2d2v-fdtd workload')
    ap.add_argument('--batch-runs', type=int, default=256)
    ap.add_argument('--batch-steps', type=int, default=200)
    ap.add_argument('--batch-schedule', default=None, metavar='TILE,CTAS,LPT',
                    help='fix the batch launch schedule (e.g. 16,4,1) instead of autotuning; '
                         'the warm-up run then launches exactly 4 x batch-steps stage kernels')
    ap.add_argument('--parallelism', default='replicas', choices=['replicas', 'slabs'],
                    help='replicas: every rank advances its own copy of the workload (the line\'s '
                         'value; with several ranks the line also holds the slab split as '
                         '"decomposed"); slabs: one run cut into q2 slabs over the ranks')
    ap.add_argument('--no-decompose', action='store_true',
                    help='with several ranks, skip the slab-split measurement')
    ap.add_argument('--no-extras', action='store_true',
                    help='skip the other targets (batch, adjoint, 2D2V) after the headline')
    ap.add_argument('--autograd-steps', type=int, default=200,
                    help='horizon of the FP64 autograd check in the default line\'s adjoint target '
                         '(--workload adjoint checks the whole horizon)')
    ap.add_argument('--seq-steps', type=int, default=20,
                    help='steps timed per sequential run in the default line\'s batch target')
    ap.add_argument('--traffic', type=float, default=None,
                    help='ncu dram bytes per launch of the dominant kernel (recorded in roofline)')
    args = ap.parse_args()
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local_rank = int(os.environ.get('LOCAL_RANK', '0'))
    if args.impl == 'reference':
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    try:
        if args.workload == 'ragged-batch':
            run_batch(args, rank, world, local_rank)
        elif args.workload == 'adjoint':
            run_adjoint(args, rank, world, local_rank)
        elif args.workload in ('2d2v-fdtd', 'c2'):
            run_c2(args, rank, world, local_rank)
        elif args.workload == 'asl-q':
            run_asl(args, rank, world, local_rank)
        elif args.workload in ('1d1v-relax', 'c1'):
            run_c1(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == '__main__':
    main()
