"""Benchmark of the 3+1D envelope ERK4(3)-IP UPPE step (one JSON line on rank 0).

Workload: 256 x 256 x 512 grid (6 mm x 6 mm x 400 fs), collimated Gaussian beam
(w0 = 1 mm, 800 nm, 40 fs FWHM, 2 mJ) with seeded 1 % amplitude speckle, argon at
1 bar (n2 = 1e-23 m^2/W, GVD 20 fs^2/m, ADK ionisation, plasma defocusing and
loss, self-steepening), L = 2 m, tol = 1e-5; mixed precision by default.

A "step" is one ERK4(3) attempt of that adaptive propagation, with acceptance and
step-size control on the device (one CUDA-graph launch per attempt).  The timed
attempts start at z = 1 m, where the beam collapses into a filament: the step
size falls, attempts are rejected and the first lines ionise.  value = grid
points x attempts x ranks / (max over ranks of the CUDA-event time of the timed
attempts).  Every field (268 MB in complex64) is larger than the 126 MB L2, so
no L2 flush is inserted.  The whole 2 m run is timed as well (config1_full), and
e2e runs it through the public propagate() call with host buffers.

--impl reference times the CPU oracle port of the reference's algorithm on the
host cores (rank 0 only), one ERK attempt of the same 256 x 256 x 512 workload
per step.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "3+1D UPPE pt-steps/s & batched-1D sims/s vs plain GPU at relL2<=1e-4; % HBM"
NX = NY = 256
NT = 512
LAM = 800e-9
FWHM = 40e-15
ENERGY = 2e-3
W0 = 1e-3
L_PROP = 2.0
TOL = 1e-5
LAM_1D = 800e-9
Z_TIMED = 1.0        # the timed attempts start here: onset of the collapse
Z_ION_TIMED = 1.0    # with the multiphoton table: start of the ionising filament
H_FIRST = 2e-3       # first step of the 2 m run: min(max_step, L/1000) (solver_3d.py:173)


CONFIG_WORKLOAD = ('3+1D UPPE envelope ERK4(3)-IP, argon 1 bar, ADK + plasma, self-steepening, '
                   '256x256x512, 6 mm x 400 fs, 2 mJ 40 fs, w0 1 mm, 1% speckle, L 2 m, tol 1e-5')


def grids(n=NX, nt=NT):
    x = np.linspace(-3e-3, 3e-3, n)
    t = np.linspace(-200e-15, 200e-15, nt)
    return x, x.copy(), t


def argon_medium(precision, oracle=False):
    """Argon 1 bar, Taylor GVD 20 fs^2/m about the Cauchy index at 800 nm."""
    if oracle:
        from oracle import uppe3d
        m0 = uppe3d.argon(LAM, 1.0, precision, True)
        n0 = float(m0.refractive_index(np.array([m0.omega0]))[0])
        return uppe3d.argon(LAM, 1.0, precision, True, dispersion=('taylor', n0, 20e-30, 0.0))
    from project_b200.media import Argon
    m0 = Argon(LAM, 1.0, precision, True)
    n0 = float(m0.refractive_index(np.array([m0.omega0]))[0])
    return Argon(LAM, 1.0, precision, True, dispersion=('taylor', n0, 20e-30, 0.0))


def make_input(x, y, t, dtype=np.complex64):
    from project_b200.pulses import gaussian_beam, speckle
    A = gaussian_beam(x, y, t, W0, ENERGY, FWHM, dtype=np.complex128)
    A *= speckle(x, y, 50e-6, 0.01, seed=1)[:, :, None]
    return A.astype(dtype)


def peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            return float(json.load(f)['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join('/tmp', f'uppe_clocks_{os.getpid()}.csv')

    def start(self):
        try:
            self.f = open(self.path, 'w')
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.gpu), f'--query-gpu={self.Q}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in open(self.path):
            p = [v.strip() for v in line.split(',')]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == 'active':
                    reasons.add(n)
        os.unlink(self.path)
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': smax,
                'reasons': sorted(reasons), 'samples': len(sm)}


def _oracle_attempt_setup(precision='single'):
    """The oracle port's solver and normalised input at the full 256 x 256 x 512 grid."""
    from oracle import uppe3d
    x, y, t = grids()
    med = argon_medium(precision, oracle=True)
    sol = uppe3d.Solver3D(x, y, t, med, precision)
    A0 = make_input(x, y, t, np.complex64 if precision == 'single' else np.complex128)
    sol.A_scale = float(np.max(np.abs(A0)))
    return sol, (A0 / sol.A_scale).astype(sol.complex_dtype)


def cpu_baseline(precision='single'):
    """Oracle port (the reference algorithm on numpy/scipy) on the host: one ERK
    attempt of the full 256 x 256 x 512 workload with scipy.fft using every host
    core, and one with a single FFT worker (the reference's default)."""
    import scipy.fft
    cores = len(os.sched_getaffinity(0))
    sol, A = _oracle_attempt_setup(precision)
    pts = NX * NY * NT
    out = {}
    for workers in (cores, 1):
        with scipy.fft.set_workers(workers):
            t0 = time.perf_counter()
            sol.erk43_step(A, H_FIRST)
            out[workers] = time.perf_counter() - t0
    return {'value': pts / out[cores], 'unit': 'pt-steps/s', 'cores': cores, 'kind': 'port',
            'sample': f'one ERK attempt of the full {NX}x{NY}x{NT} workload (c64, numpy/scipy oracle '
                      f'port, {cores} FFT workers): {out[cores]:.2f} s',
            'single_worker': {'value': pts / out[1], 'unit': 'pt-steps/s', 'cores': 1,
                              'sample': f'the same attempt with 1 FFT worker: {out[1]:.2f} s'}}


def run_reference(args, rank):
    """The reference's algorithm (oracle port of solver_3d.py:100-160 with
    media_physics.py:156-205, numpy/scipy) on the host cores, rank 0 only: each step
    is one ERK attempt of the same 256 x 256 x 512 c64 workload the GPU arm runs.
    One untimed warm-up attempt (FFT planning); the CPU path has no other warm-up."""
    if rank != 0:
        return 0
    import scipy.fft
    cores = len(os.sched_getaffinity(0))
    sol, A = _oracle_attempt_setup('single')
    pts = NX * NY * NT
    with scipy.fft.set_workers(cores):
        sol.erk43_step(A, H_FIRST)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            sol.erk43_step(A, H_FIRST)
        dt = time.perf_counter() - t0
    v = pts * args.steps / dt
    sample = (f'{args.steps} ERK attempts of the full {NX}x{NY}x{NT} workload from z = 0 (c64, oracle '
              f'port of solver_3d.py:100-160 + media_physics.py, {cores} FFT workers), 1 warm-up attempt')
    print(json.dumps({
        'impl': 'reference', 'metric': METRIC, 'value': v, 'unit': 'pt-steps/s',
        'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup, 'warmup_attempts_run': 1,
        'ms_per_step': 1e3 * dt / args.steps, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'c64', 'data': 'synthetic',
        'config': {'workload': CONFIG_WORKLOAD, 'grid': [NX, NY, NT], 'same_config': True},
        'cpu_baseline': {'value': v, 'unit': 'pt-steps/s', 'cores': cores, 'kind': 'port',
                         'sample': sample},
        'e2e': {'value': v, 'unit': 'pt-steps/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }), flush=True)
    return 0


def batched1d_instances(n=256, seed=2, L=1.0):
    """Batched 1D sweep (seeded): Nt in {2048..16384} with dt = 1 ps/4095, E log-uniform in
    10 uJ..1 mJ, pressure U(0.2, 3) bar (n2, beta2, beta3, plasma scale with it), GDD
    U(-500, 500) fs^2; argon capillary a = 125 um, A_eff = pi (0.65 a)^2, loss 0.5 dB/m,
    beta2 15 fs^2/m, beta3 15 fs^3/m per bar, ADK plasma, one-photon-per-mode noise."""
    from project_b200.distributed import instance_cost
    from project_b200.pulses import dispersed_pulse, photon_noise
    from project_b200.solver1d import ERK43IP_UPPE, GasPlasma1D
    rng = np.random.Generator(np.random.PCG64(seed))
    Aeff = np.pi * (0.65 * 125e-6) ** 2
    insts, fields = [], []
    for k in range(n):
        Nt = int(rng.choice([2048, 4096, 8192, 16384]))
        E = float(np.exp(rng.uniform(np.log(10e-6), np.log(1e-3))))
        P = float(rng.uniform(0.2, 3.0))
        GDD = float(rng.uniform(-500e-30, 500e-30))
        t = (np.arange(Nt) - (Nt - 1) / 2) * (1e-12 / 4095)
        s = ERK43IP_UPPE(material='argon_gas', n2=1e-23 * P, beam_radius=0.65 * 125e-6,
                         center_wavelength=LAM_1D, alpha=0.5 * np.log(10) / 10, use_raman=False,
                         taylor=(15e-30 * P, 15e-45 * P), plasma=GasPlasma1D(Aeff, pressure_atm=P),
                         precision='single')
        inst = s.instance(t, L, tol=1e-6)
        inst['desc'].cost = instance_cost(Nt, L, energy=E, pressure=P)   # longest expected first
        inst['energy'], inst['pressure'] = E, P
        insts.append(inst)
        fields.append(dispersed_pulse(t, E, 30e-15, GDD=GDD) + photon_noise(t, LAM_1D, 1000 + k))
    return insts, fields


def run_batched1d(dev, rank=0, world=1, accuracy=False):
    """Whole sweep in one persistent launch per GPU; sims/s over CUDA events.  With
    several ranks the instances are sharded (longest-processing-time balance on
    Nt log Nt), the time is the max over ranks and the per-instance results are
    gathered (no data-path collective)."""
    import torch
    from project_b200.distributed import gather_results, instance_cost, partition_instances
    from project_b200.solver1d import BatchedPropagator
    insts, fields = batched1d_instances()
    n_all = len(insts)
    mine = list(range(n_all))
    if world > 1:
        costs = [i['desc'].cost for i in insts]
        mine = partition_instances(costs, world)[rank]
        insts, fields = [insts[i] for i in mine], [fields[i] for i in mine]
    bp = BatchedPropagator(insts, precision='single', device=dev)
    packed0 = bp.pack(fields)
    work = packed0.clone()
    bp.run_packed(work)                      # warm-up (first launch)
    work.copy_(packed0)
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    res = bp.run_packed(work)
    e1.record()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    att = [r.attempts for r in res]
    busy, span = ctypes.c_double(), ctypes.c_double()
    from project_b200 import _lib
    _lib.check(bp._lib.uppe1d_last_activity(bp._plan, ctypes.byref(busy), ctypes.byref(span), _lib.stream_ptr()),
               'uppe1d_last_activity')
    # FLOP model of one attempt of an N-point line: 4 nonlinear evaluations (the
    # first stage is carried over), each with 3 line FFTs (5 N log2 N) and ~80 N
    # pointwise operations (stage algebra, Kerr, steepening, plasma scan)
    nts = [int(i['desc'].Nt) for i in insts]
    flops = sum(a * 4 * (3 * 5 * n * np.log2(n) + 80 * n) for a, n in zip(att, nts))
    fp32_nominal = 148 * 128 * 2 * 1.965e9
    occupancy = {'sm_busy': busy.value, 'span_ms': span.value,
                 'how': 'persistent CTAs record the global timer at start and when the queue runs dry; '
                        'sum(exit - start) / (148 SMs x span)',
                 'flop_model': '4 evaluations x (3 x 5 N log2 N + 80 N) per attempt',
                 'tflops': flops / sec / 1e12, 'fp32_frac_nominal': flops / sec / fp32_nominal,
                 'fp32_peak_nominal_tflops': fp32_nominal / 1e12}
    acc = None
    if accuracy and world == 1:
        try:
            acc = batched1d_accuracy(bp, insts, packed0, work, dev)
        except Exception as e:   # reported, never fatal
            acc = {'error': str(e)[:300]}
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([sec], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sec = float(t.item())
        merged = gather_results([(i, {'attempts': r.attempts, 'status': r.status}) for i, r in zip(mine, res)])
        att = [merged[i]['attempts'] for i in range(n_all)]
        res = [type('R', (), merged[i]) for i in range(n_all)]
    return {'value': n_all / sec, 'unit': 'sims/s', 'n_instances': n_all, 'seconds': sec, 'ranks': world,
            'kernel': ('thread-block clusters per line: eight CTAs for the costliest lines, four for the rest'
                       if bp._lib.uppe1d_uses_clusters(bp._plan) else 'one CTA per line'),
            'attempts_total': int(sum(att)), 'attempts_max': int(max(att)),
            'status_nonzero': int(sum(1 for r in res if r.status)), 'dtype': 'c64',
            'workload': 'batched 1D sweep, 256 argon-capillary instances, L = 1 m, tol 1e-6, '
                        'one persistent launch', 'occupancy': occupancy, 'accuracy': acc}


def batched1d_accuracy(bp, insts, packed0, final64, dev):
    """Each instance's mixed-precision final field against the complex128 run of the
    same instance (each with its own adaptive steps at the sweep's tol 1e-6); every
    instance the complex128 kernel supports.  A frozen-step replay is not used
    here: the stiffest instances (1 mJ at 3 bar) are ill-conditioned, and a step
    sequence accepted in one precision can be unstable in the other."""
    import torch
    from project_b200.solver1d import BatchedPropagator
    n = len(insts)
    sub = [k for k in range(n) if insts[k]['desc'].Nt <= 8192]
    bd = BatchedPropagator([insts[k] for k in sub], precision='double', device=dev)
    off = bp.offsets
    f128 = torch.cat([packed0[off[k]:off[k + 1]] for k in sub]).to(torch.complex128).contiguous()
    r2 = bd.run_packed(f128)
    res64 = getattr(bp, 'last_results', None)
    rels, dE = [], []
    for j, k in enumerate(sub):
        a = final64[off[k]:off[k + 1]]
        b = f128[bd.offsets[j]:bd.offsets[j + 1]]
        rels.append(_rel(a, b))
        e64 = float((a.abs().double() ** 2).sum()) * insts[k]['desc'].dt
        dE.append(abs(e64 - r2[j].energy) / r2[j].energy)
    rels = np.array(rels)
    worst = [{'Nt': int(insts[sub[j]]['desc'].Nt), 'attempts_c128': int(r2[j].attempts),
              'relL2': float(rels[j])} for j in np.argsort(rels)[::-1][:3]]
    # conditioning of those instances: complex128 runs from the same input and from
    # the input times (1 + 1e-7 xi), xi complex unit-variance noise (seeded)
    wk = [sub[j] for j in np.argsort(rels)[::-1][:3]]
    bw = BatchedPropagator([insts[k] for k in wk], precision='double', device=dev)
    fa = torch.cat([packed0[off[k]:off[k + 1]] for k in wk]).to(torch.complex128).contiguous()
    g = torch.Generator(device='cpu').manual_seed(7)
    xi = torch.complex(torch.randn(fa.shape, generator=g, dtype=torch.float64),
                       torch.randn(fa.shape, generator=g, dtype=torch.float64)).to(dev) / np.sqrt(2.0)
    fb = (fa * (1 + 1e-7 * xi)).contiguous()
    bw.run_packed(fa)
    bw.run_packed(fb)
    for j in range(len(wk)):
        worst[j]['c128_input_1e-7_perturbed_relL2'] = _rel(fb[bw.offsets[j]:bw.offsets[j + 1]],
                                                          fa[bw.offsets[j]:bw.offsets[j + 1]])
    # the same comparison on the same steps: complex128 replays of each instance's
    # complex64 step log; a replay whose energy leaves the complex64 run's by more
    # than 1 % (a step accepted in one precision is unstable in the other) is counted
    # apart, since its difference measures that instability, not the precision
    import ctypes
    from project_b200 import _lib
    lib = _lib.load()
    cap = 8192
    hlog = torch.zeros(n * cap, dtype=torch.float64, device=dev)
    w64 = packed0.clone()
    r64 = (_lib.Result1D * n)()
    _lib.check(lib.uppe1d_propagate_logged(bp._plan, ctypes.c_void_p(w64.data_ptr()),
                                           ctypes.c_void_p(hlog.data_ptr()), cap, r64, _lib.stream_ptr()), 'log')
    nsched = max(int(r64[k].accepted) for k in sub)
    sched = torch.zeros(len(sub), nsched, dtype=torch.float64, device=dev)
    hv = hlog.view(n, cap)
    for j, k in enumerate(sub):         # zero-length steps leave a state unchanged
        sched[j, :int(r64[k].accepted)] = hv[k, :int(r64[k].accepted)]
    f2 = torch.cat([packed0[off[k]:off[k + 1]] for k in sub]).to(torch.complex128).contiguous()
    r3 = (_lib.Result1D * len(sub))()
    _lib.check(lib.uppe1d_propagate_schedule(bd._plan, ctypes.c_void_p(f2.data_ptr()),
                                             ctypes.c_void_p(sched.data_ptr()), nsched, r3, _lib.stream_ptr()),
               'uppe1d_propagate_schedule')
    rr, unstable = [], 0
    for j, k in enumerate(sub):
        e64, e128 = r64[k].energy, r3[j].energy
        if not np.isfinite(e128) or abs(e128 - e64) > 0.01 * e64:
            unstable += 1
            continue
        rr.append(_rel(w64[off[k]:off[k + 1]], f2[bd.offsets[j]:bd.offsets[j + 1]]))
    rr = np.array(rr)
    same_steps = {'relL2_median': float(np.median(rr)), 'relL2_p90': float(np.percentile(rr, 90)),
                  'relL2_max': float(rr.max()), 'within_1e-4': int(np.sum(rr <= 1e-4)),
                  'replays_unstable': unstable}
    return {'instances_compared': len(sub), 'instances_not_compared': n - len(sub), 'worst': worst,
            'why_not': 'Nt = 16384 in complex128 needs the cluster line kernel',
            'relL2_median': float(np.median(rels)), 'relL2_p90': float(np.percentile(rels, 90)),
            'relL2_max': float(rels.max()), 'within_1e-4': int(np.sum(rels <= 1e-4)),
            'energy_rel_diff_max': float(max(dE)), 'tolerance': 1e-4,
            'note': 'free-running in both precisions at tol 1e-6: differences include the adaptive '
                    'steps\' own O(tol) discretisation differences', 'same_steps': same_steps}


def run_gradients(dev, accuracy=False):
    """Gradient evaluations through the device adjoints (forward with step log +
    reverse pass, checkpoint every 32 steps), wall time with the device synchronised:
    (1) 1D capillary compression, Nt 8192 over 2 ps, 2 GW 30 fs + one-photon noise,
    argon 1 bar with ADK plasma, 1 m, tol 1e-6, gradients w.r.t. 64 spline knots,
    pressure and length; (2) 3+1D filament, 128 x 128 x 1024 over 4 mm x 500 fs, 1.5 mJ
    50 fs, w0 1 mm, 15 Zernike coefficients (sigma 0.1 rad, seed 4, aperture 2 mm) +
    input GDD, argon 1.5 bar with ADK plasma, 1.5 m, tol 1e-4, mixed precision.
    Peak memory = plan allocations + torch's peak (workspace, checkpoints, tensors).
    Beside the adjoint values: the loss, central differences of the frozen-step map
    (the map the adjoint differentiates) for one Zernike coefficient and the GDD,
    and (accuracy) the mixed-precision exit field against complex128 on the same steps."""
    import torch
    from project_b200.adjoint import CapillaryCompression, FilamentZernike, Propagate1D, Propagate3D
    from project_b200.media import Argon
    from project_b200.pulses import gaussian_pulse, photon_noise
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    out = {}
    Nt = 8192
    t = np.linspace(-1e-12, 1e-12, Nt)
    fw = 30e-15
    A0 = gaussian_pulse(t, 2e9 * fw * np.sqrt(np.pi / (4 * np.log(2))), fw) + photon_noise(t, LAM_1D, 0)
    cc = CapillaryCompression(t, A0, n_knots=64, plasma=True, device=dev)
    knots = torch.zeros(64, dtype=torch.float64, device=dev, requires_grad=True)
    P = torch.tensor(1.0, dtype=torch.float64, device=dev, requires_grad=True)
    L = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    cc.loss(knots, P, L)          # warm-up
    torch.cuda.synchronize(dev)
    torch.cuda.reset_peak_memory_stats(dev)
    t0 = time.perf_counter()
    loss = cc.loss(knots, P, L, tol=1e-6, K=32)
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    gk, gP, gL = torch.autograd.grad(loss, [knots, P, L])
    torch.cuda.synchronize(dev)
    t2 = time.perf_counter()
    out['capillary_1d'] = {'forward_s': t1 - t0, 'adjoint_s': t2 - t1, 'steps': len(Propagate1D.last_steps),
                           'checkpoint_every': 32, 'params': 66, 'dtype': 'c128',
                           'loss_W': float(loss.detach()),
                           'torch_peak_gb': torch.cuda.max_memory_allocated(dev) / 1e9,
                           'grad_norm_knots': float(gk.norm()), 'dL_dP': float(gP), 'dL_dL': float(gL)}
    N, Nt3 = 128, 1024
    x = np.linspace(-2e-3, 2e-3, N)
    t3 = np.linspace(-250e-15, 250e-15, Nt3)
    free0 = torch.cuda.mem_get_info(dev)[0]
    sol = ERK43IP_UPPE_3D_Optimized(x, x, t3, Argon(LAM_1D, 1.5, 'single', True), precision='single',
                                    device=dev)
    torch.cuda.synchronize(dev)
    plan_bytes = free0 - torch.cuda.mem_get_info(dev)[0]
    obj = FilamentZernike(sol, w0=1e-3, energy=1.5e-3, fwhm=50e-15, aperture_radius=2e-3)
    rng = np.random.Generator(np.random.PCG64(4))
    c = torch.tensor(rng.normal(0, 0.1, 15), dtype=torch.float64, device=dev, requires_grad=True)
    gdd = torch.tensor(0.0, dtype=torch.float64, device=dev, requires_grad=True)
    torch.cuda.synchronize(dev)
    torch.cuda.reset_peak_memory_stats(dev)
    base = torch.cuda.memory_allocated(dev)
    t0 = time.perf_counter()
    loss = obj.loss(c, gdd, 1.5, tol=1e-4, K=32)
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    gc, gg = torch.autograd.grad(loss, [c, gdd])
    torch.cuda.synchronize(dev)
    t2 = time.perf_counter()
    r = sol.last_result
    steps = np.array(Propagate3D.last_steps)
    f3 = {'forward_s': t1 - t0, 'adjoint_s': t2 - t1, 'steps': int(r.accepted),
          'attempts': int(r.attempts), 'checkpoint_every': 32, 'params': 16,
          'dtype': 'c64 bulk, FP64 phase/error/controller',
          'workspace_gb': Propagate3D.workspace_bytes / 1e9,
          'peak_memory_gb': (plan_bytes + torch.cuda.max_memory_allocated(dev) - base) / 1e9,
          'plan_gb': plan_bytes / 1e9,
          'peak_ionization': sol.diagnostics()['peak_ionization'],
          'loss_J_per_m2': float(loss.detach()), 'grad_norm_zernike': float(gc.norm()),
          'dL_dGDD_per_fs2': float(gg) * 1e-30}

    def frozen_loss(cv, gv, solver):
        with torch.no_grad():
            A = solver.replay(obj.input_field(cv, gv).to(solver.complex_dtype), steps)   # obj, steps: current
            a = A[obj.ix, obj.iy, :].to(torch.complex128)
            return float(-(a.real ** 2 + a.imag ** 2).sum() * solver.dt)

    # central differences and the c64/c128 comparison on a shorter cell (0.25 m, well
    # before the collapse near 0.5 m): at 1.5 m the beam has collapsed, the exit fluence
    # is ill-conditioned (|grad| ~ 1e11-1e15 per rad) and a perturbed input can make
    # a frozen step unstable, so differences there measure the collapse, not the adjoint
    Lfd = 0.25
    loss_fd = obj.loss(c, gdd, Lfd, tol=1e-4, K=32)
    gc, gg = torch.autograd.grad(loss_fd, [c, gdd])
    steps = np.array(Propagate3D.last_steps)
    f3['check_L_m'] = Lfd
    f3['check_loss_J_per_m2'] = float(loss_fd.detach())
    j = int(torch.argmax(gc.abs()))
    dc, dg = 1e-3, 10e-30
    e = torch.zeros_like(c)
    e[j] = dc
    cd = c.detach()
    fd_c = (frozen_loss(cd + e, gdd.detach(), sol) - frozen_loss(cd - e, gdd.detach(), sol)) / (2 * dc)
    fd_g = (frozen_loss(cd, gdd.detach() + dg, sol) - frozen_loss(cd, gdd.detach() - dg, sol)) / (2 * dg)
    f3['central_difference'] = {
        'map': 'frozen accepted steps (the map the adjoint differentiates), mixed precision',
        'zernike_index': j, 'step_rad': dc, 'adjoint': float(gc[j]), 'fd': fd_c,
        'gdd_step_fs2': dg * 1e30, 'adjoint_gdd_per_fs2': float(gg) * 1e-30, 'fd_gdd_per_fs2': fd_g * 1e-30}
    if accuracy:
        s128 = ERK43IP_UPPE_3D_Optimized(x, x, t3, Argon(LAM_1D, 1.5, 'double', True), precision='double',
                                         device=dev)
        with torch.no_grad():
            Ain = obj.input_field(cd, gdd.detach())
            o64 = sol.replay(Ain.to(torch.complex64), steps)
            o128 = s128.replay(Ain.to(torch.complex128), steps)
            f3['accuracy'] = {'L_m': Lfd, 'relL2_exit_c64_vs_c128_same_steps': _rel(o64, o128), 'tolerance': 1e-4,
                              'loss_c64': frozen_loss(cd, gdd.detach(), sol),
                              'loss_c128': frozen_loss(cd, gdd.detach(), s128)}
        # the same check with the complex128 plan: its adjoint against central
        # differences of its own frozen-step map (separates the adjoint from the
        # rounding of the mixed map)
        obj128 = FilamentZernike(s128, w0=1e-3, energy=1.5e-3, fwhm=50e-15, aperture_radius=2e-3)
        c2 = cd.clone().requires_grad_(True)
        g2 = gdd.detach().clone().requires_grad_(True)
        l128 = obj128.loss(c2, g2, Lfd, tol=1e-4, K=32)
        gc2, gg2 = torch.autograd.grad(l128, [c2, g2])
        steps_saved = steps
        steps = np.array(Propagate3D.last_steps)
        obj_saved, obj = obj, obj128
        fd2_c = (frozen_loss(cd + e, gdd.detach(), s128) - frozen_loss(cd - e, gdd.detach(), s128)) / (2 * dc)
        fd2_g = (frozen_loss(cd, gdd.detach() + dg, s128) - frozen_loss(cd, gdd.detach() - dg, s128)) / (2 * dg)
        obj, steps = obj_saved, steps_saved
        f3['central_difference_complex128'] = {
            'zernike_index': j, 'adjoint': float(gc2[j]), 'fd': fd2_c,
            'adjoint_gdd_per_fs2': float(gg2) * 1e-30, 'fd_gdd_per_fs2': fd2_g * 1e-30,
            'grad_relL2_mixed_vs_c128': float(torch.linalg.vector_norm(gc - gc2) / torch.linalg.vector_norm(gc2))}
        del s128, obj128
        torch.cuda.empty_cache()
    out['filament_3d'] = f3
    return out


def run_realfield(dev, cpu=True):
    """Real-field 3+1D solver (src/3+1D-UPPE-ERK4(3)IP-real-field): argon 1 atm,
    128 x 128 x 1024 real samples over 0.8 mm x 200 fs, 800 nm 20 fs pulse at
    4e10 V/m, single precision (the reference's); time per ERK attempt over CUDA
    events, bytes per attempt from the pass list, and the oracle's step on a
    32 x 32 x 1024 sample on the host.  Bytes: spectral fields F of Nx Ny (Nt/2 + 16)
    complex64 and real fields R of Nx Ny Nt float32: rfft (R + F), x and y forward
    transforms (4 F), inverse y of E_kw (2 F), per stage inverse x (2 F), the
    nonlinear t-line pass (2 F) and forward x (2 F), then the fused y pass with the
    stage algebra (5, 6, 5, 5 F), and the output (inverse x 2 F, irfft F + R):
    55 F + 2 R."""
    import torch
    from project_b200.realfield import Argon, ERK43_RealField_UPPE_3D
    N, Nt = 128, 1024
    x = np.linspace(-0.4e-3, 0.4e-3, N)
    t = np.linspace(-100e-15, 100e-15, Nt)
    X, Y = np.meshgrid(x, x, indexing='ij')
    w = 2 * np.pi * 299792458.0 / 800e-9
    env = np.exp(-2 * np.log(2) * t ** 2 / (20e-15) ** 2) * np.cos(w * t)
    E0 = (4e10 * np.exp(-(X ** 2 + Y ** 2) / (0.2e-3) ** 2)[:, :, None] * env[None, None, :]).astype(np.float32)
    sol = ERK43_RealField_UPPE_3D(x, x, t, Argon(800e-9, 1.0), precision='single', device=dev)
    sol.set_field(torch.from_numpy(E0).to(dev))
    h = 1e-6
    for _ in range(3):
        sol.attempt(h)
    n = 10
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record()
    for _ in range(n):
        sol.attempt(h)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / n
    Nw = Nt // 2 + 16
    Fs = N * N * Nw * 8
    Fr = N * N * Nt * 4
    byts = 55 * Fs + 2 * Fr
    out = {'workload': 'real-field 3+1D ERK4(3)-IP attempt, argon 1 atm, 128x128x1024, 0.8 mm x 200 fs, '
                       '20 fs 800 nm at 4e10 V/m, PPT + Drude current, single precision',
           'ms_per_attempt': ms, 'value': N * N * Nt / (ms / 1e3), 'unit': 'pt-steps/s',
           'achieved_gbs': byts / (ms / 1e3) / 1e9, 'bytes_model': '55 spectral + 2 real field passes per attempt'}
    if cpu:
        from oracle import realfield as orf
        xs = np.linspace(-0.4e-3, 0.4e-3, 32)
        Xs, Ys = np.meshgrid(xs, xs, indexing='ij')
        Es = (4e10 * np.exp(-(Xs ** 2 + Ys ** 2) / (0.2e-3) ** 2)[:, :, None] * env[None, None, :]).astype(np.float32)
        os_ = orf.Solver(xs, xs, t, orf.argon(800e-9, 1.0), 'single')
        os_.E_scale = float(np.abs(Es).max())
        t0 = time.perf_counter()
        os_.step(Es / np.float32(os_.E_scale), h)
        dt_ = time.perf_counter() - t0
        out['cpu_baseline'] = {'value': 32 * 32 * Nt / dt_, 'unit': 'pt-steps/s', 'cores': 1, 'kind': 'port',
                               'sample': f'one attempt on 32x32x1024 (numpy/scipy oracle): {dt_:.2f} s'}
    return out


def cpu_baseline_1d():
    """Oracle port of the reference 1D solver on one argon-capillary instance (Nt 4096, 2 GW 30 fs,
    argon 1 bar, 1 m, tol 1e-6, with the plasma term) on the host."""
    from oracle import uppe1d as o1
    from oracle.inputs import gaussian_pulse
    Aeff = np.pi * (0.65 * 125e-6) ** 2
    t = np.linspace(-0.5e-12, 0.5e-12, 4096)
    fw = 30e-15
    s = o1.Solver1D(material='argon_gas', n2=1e-23, beam_radius=0.65 * 125e-6, center_wavelength=LAM_1D,
                    alpha=0.5 * np.log(10) / 10, use_raman=False, taylor=(15e-30, 15e-45),
                    plasma=o1.Plasma1D(Aeff, center_wavelength=LAM_1D))
    t0 = time.perf_counter()
    _, _, _, log = s.propagate(gaussian_pulse(t, 2e9 * fw * np.sqrt(np.pi / (4 * np.log(2))), fw), t, 1.0, tol=1e-6)
    dt = time.perf_counter() - t0
    return {'value': 1.0 / dt, 'unit': 'sims/s', 'cores': 1, 'kind': 'port',
            'sample': f'one argon-capillary instance (Nt 4096, 2 GW 30 fs, 1 m, {len(log)} attempts) on numpy/scipy: {dt:.2f} s'}


def profile_kernels(sol, lib, n_attempts=3):
    """Per-launch CUDA-event times of whole attempts -> per-kernel totals."""
    import torch
    from project_b200 import _lib
    cap = 64
    ms = (ctypes.c_float * cap)()
    kind = (ctypes.c_int * cap)()
    byts = (ctypes.c_double * cap)()
    n = ctypes.c_int()
    agg = {}
    for _ in range(n_attempts):
        _lib.check(lib.uppe3d_profile_attempt(sol._plan, cap, ms, kind, byts, ctypes.byref(n),
                                              _lib.stream_ptr()), 'uppe3d_profile_attempt')
        for i in range(n.value):
            if byts[i] == 0:
                continue
            name = {0: 'k_tpass_w', 1: 'k_xpass_sq', 2: 'k_space', 4: 'k_ypass_tma',
                    5: 'k_ypass_rq', 6: 'k_ypass_tq'}.get(kind[i], 'scalar')
            a = agg.setdefault(name, [0.0, 0.0, 0])
            a[0] += ms[i]
            a[1] += byts[i]
            a[2] += 1
    torch.cuda.synchronize()
    return agg


def pattern_ceilings(dev, reps=20):
    """Copy bandwidth of the passes' access patterns alone (uppe_pattern_probe: one
    read + one write of a 256 x 256 x 512 complex64 field, sequential, as x-pass
    tiles or as y-pass tiles of 8, 16 or 32 omega columns), CUDA events over
    `reps` launches after three warm-up launches; GB/s."""
    import torch
    from project_b200 import _lib
    lib = _lib.load()
    a = torch.zeros((NX, NY, NT), dtype=torch.complex64, device=dev)
    b = torch.zeros_like(a)
    s = _lib.stream_ptr()
    out = {}
    for name, pat, kw in (('sequential', 0, 16), ('x tiles kw8', 1, 8), ('x tiles kw16', 1, 16),
                          ('x tiles kw32', 1, 32), ('y tiles kw8', 2, 8), ('y tiles kw16', 2, 16),
                          ('y tiles kw32', 2, 32)):
        def run():
            _lib.check(lib.uppe_pattern_probe(pat, kw, ctypes.c_void_p(a.data_ptr()),
                                              ctypes.c_void_p(b.data_ptr()), NT, s), 'uppe_pattern_probe')
        for _ in range(3):
            run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run()
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / reps
        out[name] = 2.0 * a.numel() * 8 / (ms / 1e3) / 1e9
    del a, b
    return out


# the access pattern of each pass kernel in pattern_ceilings
PASS_PATTERN = {'k_ypass_rq': 'y tiles kw16', 'k_ypass_tma': 'y tiles kw16', 'k_ypass_ring': 'y tiles kw16',
                'k_space': 'y tiles kw16', 'k_xpass_sq': 'x tiles kw16', 'k_tpass_w': 'sequential',
                'k_tpass': 'sequential'}


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run_chunks(sol, nmax, chunk, stop=None):
    """Graph launches (one attempt each) in chunks, CUDA events around each chunk;
    stops when the run is over (the attempt count no longer moves), after nmax
    launches, or when stop(result) holds.  Returns (device ms, result)."""
    import torch
    from project_b200 import _lib
    lib, s = sol._lib, _lib.stream_ptr()
    ms, done = 0.0, 0
    r = sol.result()
    while done < nmax:
        n = min(chunk, nmax - done)
        e0, e1 = _events()
        e0.record()
        _lib.check(lib.uppe3d_run_steps(sol._plan, n, s), 'uppe3d_run_steps')
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        done += n
        r1 = sol.result()
        finished = r1.attempts == r.attempts
        r = r1
        if finished or (stop is not None and stop(r)):
            break
    return ms, r


def line_stats(sol, med):
    """From the current field: the fraction of (x, y) lines on which the t-line kernel
    runs the plasma terms (peak intensity above the last zero of the float32 rate
    table) and the fraction on which the density scan leaves its affine form (rate
    x dt above exp(-dt/tau_rec) at the peak: one sample can saturate the density)."""
    A = sol.field()
    Ipk = (A.real.float() ** 2 + A.imag.float() ** 2).amax(dim=2).double().cpu().numpy().ravel()
    lx = np.asarray(med.lut_log10I, dtype=np.float64)
    lw = np.asarray(med.lut_W, dtype=np.float32).astype(np.float64)
    nz = np.nonzero(lw)[0]
    I_on = 10.0 ** lx[nz[0] - 1] if len(nz) and nz[0] > 0 else (0.0 if len(nz) else np.inf)
    W = np.interp(np.clip(np.log10(Ipk + 1e-30), lx[0], lx[-1]), lx, lw)
    dt = float(sol.dt)
    return {'plasma_lines': float(np.mean(Ipk > I_on)),
            'saturating_lines': float(np.mean(W * dt > np.exp(-dt / med.tau_rec))),
            'peak_intensity_Wm2': float(Ipk.max())}


def full_run(sol, A_dev, hlog=None):
    """The whole adaptive 2 m propagation from A_dev on the device, CUDA-event timed."""
    import ctypes
    from project_b200 import _lib
    lib, s = sol._lib, _lib.stream_ptr()
    sol.set_field(A_dev)
    if hlog is not None:
        _lib.check(lib.uppe3d_set_step_log(sol._plan, ctypes.c_void_p(hlog.data_ptr()), hlog.numel(), s), 'log')
    _lib.check(lib.uppe3d_begin(sol._plan, L_PROP, TOL, 1e-2, 1e-9, 0, s), 'uppe3d_begin')
    ms, r = run_chunks(sol, 10 ** 7, 16)
    if hlog is not None:
        _lib.check(lib.uppe3d_set_step_log(sol._plan, None, 0, s), 'log')
    d = sol.diagnostics()
    npts = sol.Nx * sol.Ny * sol.Nt
    return {'device_s': ms / 1e3, 'attempts': int(r.attempts), 'accepted': int(r.accepted),
            'rejected': int(r.attempts - r.accepted), 'z_m': r.z, 'status': int(r.status),
            'value': npts * r.attempts / (ms / 1e3), 'unit': 'pt-steps/s',
            'energy_J': d['energy'], 'photons': d['photons'], 'peak_ionization': d['peak_ionization']}


def _rel(a, b):
    import torch
    a = a.to(torch.complex128)
    b = b.to(torch.complex128)
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def accuracy_config1(sol64, x, y, t, A0, steps, a_T, state_T, final64, dev, early=None):
    """Mixed precision against the complex128 device path (pinned to the oracle and
    the reference's own runs at small grids) on the same accepted step sequence:
    rel-L2 of the field at the end of the timed attempts and at z = 2 m, energy,
    photon number and peak ionisation of both; one attempt from the same state in
    both precisions; and the complex128 run from the complex64-rounded input, which
    shows how far the dynamics alone amplify an input difference of that size."""
    import torch
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    s128 = ERK43IP_UPPE_3D_Optimized(x, y, t, argon_medium('double'), precision='double', device=dev)
    marks = {a_T, len(steps)} | ({k for k in early} if early else set())

    def replay(Ain):
        s128.set_field(Ain)
        snaps = {}
        for k, h in enumerate(steps):
            s128.attempt(float(h))
            s128.commit(True)
            if k + 1 in marks:
                snaps[k + 1] = s128.field()
        return snaps

    A128 = torch.from_numpy(make_input(x, y, t, np.complex128)).to(dev)   # exact input
    base = replay(A128)
    d128 = s128.diagnostics()
    d64 = sol64.diagnostics()
    rounded = replay(A128.to(torch.complex64).to(torch.complex128))
    out = {'grid': [NX, NY, NT], 'steps_replayed': len(steps), 'tolerance': 1e-4,
           'relL2_after_timed': _rel(state_T, base[a_T]), 'z_after_timed_m': float(np.sum(steps[:a_T])),
           'relL2_end': _rel(final64, base[len(steps)]),
           'relL2_earlier': [{'accepted_steps': k, 'z_m': float(np.sum(steps[:k])),
                              'relL2': _rel(early[k], base[k])} for k in sorted(early)] if early else None,
           'c128_from_c64_rounded_input_relL2_after_timed': _rel(rounded[a_T], base[a_T]),
           'c128_from_c64_rounded_input_relL2_end': _rel(rounded[len(steps)], base[len(steps)]),
           'energy_J': {'c64': d64['energy'], 'c128': d128['energy']},
           'photons': {'c64': d64['photons'], 'c128': d128['photons']},
           'peak_ionization': {'c64': d64['peak_ionization'], 'c128': d128['peak_ionization']}}
    # one attempt from the complex128 state at the timed window's end, in both precisions
    snap = base[a_T]
    h = float(steps[a_T]) if a_T < len(steps) else float(steps[-1])
    s128.set_field(snap)
    s128.attempt(h)
    s128.commit(True)
    o128 = s128.field()
    sol64.set_field(snap.to(torch.complex64))
    sol64.attempt(h)
    sol64.commit(True)
    o64 = sol64.field()
    out['one_attempt_relL2'] = _rel(o64, o128)
    out['one_attempt_input_rounding_relL2'] = _rel(snap.to(torch.complex64), snap)
    del s128
    torch.cuda.empty_cache()
    return out


def mpi_argon(precision, P=1.0):
    """Argon with the reference's own multiphoton rate as the ionisation table:
    W = sigma_K I^K, K = 11, sigma_K = 1e-188 P (media_physics.py:139-142, 410-417),
    on the reference's grid (:121-126), without the tunnel term whose +1e-20
    denominator makes it 1e15 1/s at every intensity.  Taylor GVD as argon_medium."""
    from project_b200.media import Argon
    m0 = Argon(LAM, P, precision, True)
    lx = m0._lut_grid()
    W = 1.0e-188 * P * (10.0 ** lx) ** 11
    n0 = float(m0.refractive_index(np.array([m0.omega0]))[0])
    return Argon(LAM, P, precision, True, dispersion=('taylor', n0, 20e-30, 0.0), lut=(lx, W))


def run_ionising(args, x, y, t, A_dev, dev):
    """The same 2 m run with the multiphoton table: the filament ionises (the
    intensity clamps), so the density scan, plasma loss and defocusing and the
    plasma transform run on the lines of the filament.  Timed: K attempts from
    z = Z_ION_TIMED and the whole run (CUDA events)."""
    import torch
    from project_b200 import _lib
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    med = mpi_argon('single')
    sol = ERK43IP_UPPE_3D_Optimized(x, y, t, med, precision='single', device=dev)
    lib, s = sol._lib, _lib.stream_ptr()
    npts = NX * NY * NT
    sol.set_field(A_dev)
    _lib.check(lib.uppe3d_begin(sol._plan, L_PROP, TOL, 1e-2, 1e-9, 0, s), 'begin')
    ms_pos, _ = run_chunks(sol, 10 ** 6, 4, stop=lambda r: r.z >= Z_ION_TIMED)
    ms_w, _ = run_chunks(sol, args.warmup, args.warmup)
    r0 = sol.result()
    lines0 = line_stats(sol, med)
    ms_t, r1 = run_chunks(sol, args.steps, args.steps)
    lines1 = line_stats(sol, med)
    agg = profile_kernels(sol, lib)
    ms_rest, r2 = run_chunks(sol, 10 ** 7, 16)
    d = sol.diagnostics()
    prof = {k: v[0] / 3 for k, v in agg.items()}
    total_ms = ms_pos + ms_w + ms_t + ms_rest + sum(v[0] for v in agg.values())
    del sol
    torch.cuda.empty_cache()
    return {'table': 'multiphoton sigma_K I^K, K = 11, sigma_K = 1e-188 m^22/W^11/s (reference media_physics.py)',
            'timed': {'attempts': int(r1.attempts - r0.attempts), 'accepted': int(r1.accepted - r0.accepted),
                      'z_m': [r0.z, r1.z], 'ms_per_attempt': ms_t / max(r1.attempts - r0.attempts, 1),
                      'value': npts * (r1.attempts - r0.attempts) / (ms_t / 1e3), 'unit': 'pt-steps/s',
                      'lines_at_start': lines0, 'lines_at_end': lines1},
            'kernel_ms_per_attempt': prof,
            'full_run': {'device_s': total_ms / 1e3, 'attempts': int(r2.attempts), 'accepted': int(r2.accepted),
                         'z_m': r2.z, 'status': int(r2.status), 'value': npts * r2.attempts / (total_ms / 1e3),
                         'unit': 'pt-steps/s', 'energy_J': d['energy'], 'photons': d['photons'],
                         'peak_ionization': d['peak_ionization'],
                         'note': 'includes 3 attempts run launch by launch for the kernel split'}}


def plan_tuning(sol):
    """The launch configuration the plan's tuner picked, with the candidates' times."""
    import ctypes
    from project_b200 import _lib
    cfg = (ctypes.c_int * 6)()
    ms = (ctypes.c_float * _lib.UPPE3D_TUNE_SLOTS)()
    _lib.check(sol._lib.uppe3d_tuning(sol._plan, cfg, ms), 'uppe3d_tuning')
    names = ['tma16 2/SM', 'tma16 1/SM', 'tma16 late 3/SM', 'tma16 late 2/SM', 'tma8 4/SM', 'tma8 late 6/SM',
             'reg4step 2/SM', 'reg4step late 3/SM', 'reg4step tma ring 1/SM', 'reg4step8 4/SM',
             'reg4step8 late 6/SM']
    kind = {0: 'plain', 1: f'tma{cfg[3]}', 2: 'reg4step' if cfg[3] == 16 else 'reg4step8',
            3: 'reg4step tma ring'}[cfg[0]]
    y = kind if not cfg[0] else f"{kind}{' late' if cfg[2] else ''} {cfg[1]}/SM"
    return {'y_pass': y, 't_lines_per_block': cfg[4], 'source': {0: 'defaults', 1: 'timed', 2: 'cache'}[cfg[5]],
            'y_candidates_ms': {n: round(float(v), 4) for n, v in zip(names, ms[:11]) if v > 0},
            't_candidates_ms': {w: round(float(v), 4) for w, v in zip((8, 4), ms[11:13]) if v > 0}}


def run_b200(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from project_b200 import _lib
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    dev = torch.device('cuda', local_rank)
    torch.cuda.set_device(dev)
    x, y, t = grids()
    prec = args.precision
    cdt = np.complex64 if prec == 'single' else np.complex128
    A0 = make_input(x, y, t, cdt)
    med = argon_medium(prec)
    sol = ERK43IP_UPPE_3D_Optimized(x, y, t, med, precision=prec, device=dev)
    lib = sol._lib
    A_dev = torch.from_numpy(A0).to(dev)
    s = _lib.stream_ptr()
    npts = NX * NY * NT
    tuning = plan_tuning(sol)

    # (1) the timed attempts: position the run at the collapse (untimed), warm up, time K
    want_acc = rank == 0 and prec == 'single' and not args.no_accuracy
    sol.set_field(A_dev)
    _lib.check(lib.uppe3d_begin(sol._plan, L_PROP, TOL, 1e-2, 1e-9, 0, s), 'begin')
    early = {}
    r20 = run_chunks(sol, 10 ** 6, 1, stop=lambda r: r.accepted >= 20)[1]
    if want_acc:
        early[int(r20.accepted)] = sol.field().clone()       # the first 20 steps from z = 0
    rpre = run_chunks(sol, 10 ** 6, 4, stop=lambda r: r.z >= Z_TIMED)[1]
    if want_acc:
        early[int(rpre.accepted)] = sol.field().clone()      # the onset of the collapse
    _lib.check(lib.uppe3d_run_steps(sol._plan, args.warmup, s), 'warmup')
    torch.cuda.synchronize()
    r0 = sol.result()
    lines0 = line_stats(sol, med)
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    ev0, ev1 = _events()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0.record()
    _lib.check(lib.uppe3d_run_steps(sol._plan, args.steps, s), 'run_steps')
    ev1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    r1 = sol.result()
    attempts = r1.attempts - r0.attempts
    accepted = r1.accepted - r0.accepted
    if attempts != args.steps:
        raise RuntimeError(f'the run ended inside the timed window ({attempts} of {args.steps} attempts)')
    state_T = sol.field().clone() if want_acc else None
    a_T = int(r1.accepted)
    lines1 = line_stats(sol, med)
    ms_t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = npts * args.steps * world / (ms_max / 1e3)

    # per-kernel roofline (CUDA events around each launch of 3 attempts at this state)
    agg = profile_kernels(sol, lib)
    peak, peak_kind = peaks()
    dom = max((k for k in agg if k != 'scalar'), key=lambda k: agg[k][0])
    d_ms, d_bytes, d_n = agg[dom]
    achieved = d_bytes / (d_ms / 1e3) / 1e9
    traffic = None
    try:   # DRAM bytes from the committed ncu capture of the same kernel, per launch
        with open(os.path.join(ROOT, 'profiles', 'ncu_traffic.json')) as f:
            traffic = json.load(f)[dom]['measured_over_algorithmic'] * d_bytes / d_n
    except Exception:
        traffic = None
    try:
        patterns = pattern_ceilings(dev)
    except Exception as e:   # reported, never fatal
        patterns = {'error': str(e)[:200]}
    pat_key = PASS_PATTERN.get(dom)
    pat_gbs = patterns.get(pat_key) if pat_key else None
    step_bytes = 64.0 * (8 if prec == 'single' else 16) * npts     # 64 s N per attempt
    step_achieved = step_bytes / (ms_max / args.steps / 1e3) / 1e9

    # (2) the whole 2 m propagation on the device, with the accepted steps logged
    hlog = torch.zeros(1 << 16, dtype=torch.float64, device=dev)
    full = full_run(sol, A_dev, hlog)
    steps = hlog[:full['accepted']].cpu().numpy()
    final64 = sol.field().clone() if want_acc else None
    full['lines_at_timed_start'] = lines0
    full['lines_at_timed_end'] = lines1

    # (3) e2e: the public propagate() call with pinned host buffers, the whole 2 m run;
    # one host->device copy of A0 and one device->host copy of the spectrum per call
    A_host = torch.from_numpy(A0).pin_memory()
    out_host = torch.empty(A_host.shape, dtype=A_host.dtype).pin_memory()
    sol.propagate(A_host, L_PROP, tol=TOL, out=out_host)      # warm
    torch.cuda.synchronize()
    reps = 2
    t0 = time.perf_counter()
    done = 0
    for _ in range(reps):
        sol.propagate(A_host, L_PROP, tol=TOL, out=out_host)
        done += sol.last_result.attempts
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_v = npts * done * world / float(e2e_t.item())
    per_call = done / reps
    fbytes = A0.nbytes

    accuracy = None
    if want_acc:
        try:
            accuracy = accuracy_config1(sol, x, y, t, A0, steps, a_T, state_T, final64, dev, early)
        except Exception as e:   # reported, never fatal
            accuracy = {'error': str(e)[:300]}
        del state_T, final64
        early.clear()
        torch.cuda.empty_cache()

    ionising = None
    if rank == 0 and not args.no_ionising:
        try:
            ionising = run_ionising(args, x, y, t, A_dev, dev)
        except Exception as e:   # reported, never fatal
            ionising = {'error': str(e)[:300]}

    plain = None
    if rank == 0 and not args.no_plain_gpu:
        try:
            from baseline import plain_gpu
            plain = plain_gpu.time_step(x, y, t, A0.astype(np.complex128), argon_medium('double'),
                                        dev)
        except Exception as e:   # reported, never fatal
            plain = {'error': str(e)[:200]}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(prec)
    b1d = None
    if not args.no_batched_1d:
        b1d = run_batched1d(dev, rank, world, accuracy=want_acc)
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            b1d['cpu_baseline'] = cpu_baseline_1d()

    rfield = None
    if rank == 0 and not args.no_realfield:
        try:
            rfield = run_realfield(dev, cpu=(world == 1 and not args.no_cpu_baseline))
        except Exception as e:   # reported, never fatal
            rfield = {'error': str(e)[:300]}
    grads = None
    if rank == 0 and not args.no_gradients:
        try:
            grads = run_gradients(dev, accuracy=want_acc)
        except Exception as e:   # reported, never fatal
            grads = {'error': str(e)[:300]}

    if rank == 0:
        line = {
            'metric': METRIC, 'value': value, 'unit': 'pt-steps/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms_max / args.steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'c64' if prec == 'single' else 'c128', 'data': 'synthetic',
            'config': {'workload': CONFIG_WORKLOAD,
                       'grid': [NX, NY, NT], 'precision': prec,
                       'mixed_precision': 'complex64 bulk; FP64 phase (mod 2pi), density scan, '
                                          'error norm, controller' if prec == 'single' else None,
                       'timed_window': f'attempts {int(r0.attempts)}..{int(r1.attempts)} of the 2 m run, '
                                       f'z = {r0.z:.4f} -> {r1.z:.4f} m (collapse onset)',
                       'attempts_timed': attempts, 'accepted_timed': accepted,
                       'parallelism': f'replicas x{world}',
                       'l2': 'every field (268 MB c64) exceeds the 126 MB L2; no flush'},
            'roofline': {'bound': 'hbm', 'kernel': dom, 'achieved': achieved, 'peak': peak,
                         'peak_source': peak_kind, 'unit': 'GB/s', 'frac': achieved / peak,
                         'traffic': traffic, 'traffic_unit': 'bytes per launch',
                         'launches_profiled': d_n,
                         'bytes_model': 'per launch: fields read + written x field bytes',
                         'access_pattern': pat_key, 'pattern_copy_gbs': pat_gbs,
                         'frac_of_pattern_copy': (achieved / pat_gbs) if pat_gbs else None},
            'access_pattern_copy_gbs': patterns,
            'roofline_step': {'model': '64*s*N bytes per attempt', 'achieved': step_achieved,
                              'peak': peak, 'unit': 'GB/s', 'frac': step_achieved / peak},
            'kernel_ms_per_attempt': {k: v[0] / 3 for k, v in agg.items()},
            'tuning': tuning,
            'config1_full': full,
            'accuracy': accuracy,
            'ionising': ionising,
            'cpu_baseline': cpu,
            'e2e': {'value': e2e_v, 'unit': 'pt-steps/s',
                    'h2d_bytes_per_step': fbytes / per_call, 'd2h_bytes_per_step': fbytes / per_call,
                    'h2d_bytes_per_call': fbytes, 'd2h_bytes_per_call': fbytes,
                    'attempts_per_call': per_call, 'seconds_per_call': e2e_s / reps,
                    'how': 'propagate(host pinned A0, L = 2 m) -> spectrum in pinned host memory: one '
                           'call is the whole configured run; bytes per step = bytes per call / attempts'},
            'plain_gpu': plain,
            'batched_1d': b1d,
            'gradients': grads,
            'realfield_3d': rfield,
            'gpu_launches': args.steps * lib.uppe3d_launches_per_step(sol._plan),
            'clocks': clk,
        }
        print(json.dumps(line), flush=True)
    return 0


def run_profile_case(args):
    """Only the propagator, for profiler commands: position the 2 m run at z =
    --profile-z (untimed), warm up, then run the timed attempts inside an NVTX
    range named "timed" (ncu --nvtx --nvtx-include "timed/" captures only those).
    --profile-table mpi uses the multiphoton table (ionising filament); --profile-grid
    N runs an N x N x 512 grid over the same 6 mm (a smaller case for full captures);
    --profile-tuning Y,C,L,K,W forces the launch configuration (uppe3d_set_tuning:
    y kernel, CTAs per SM, late loads, omega columns, t-lines per block), since the
    tuner's own timings shift under a profiler."""
    import torch
    from project_b200 import _lib
    from project_b200.solver3d import ERK43IP_UPPE_3D_Optimized
    n = args.profile_grid
    x, y, t = grids(n)
    cdt = np.complex64 if args.precision == 'single' else np.complex128
    med = mpi_argon(args.precision) if args.profile_table == 'mpi' else argon_medium(args.precision)
    sol = ERK43IP_UPPE_3D_Optimized(x, y, t, med, precision=args.precision)
    if args.profile_tuning:
        cfg = [int(v) for v in args.profile_tuning.split(',')]
        _lib.check(sol._lib.uppe3d_set_tuning(sol._plan, *cfg), 'uppe3d_set_tuning')
    sol.set_field(torch.from_numpy(make_input(x, y, t, cdt)).cuda())
    lib, s = sol._lib, _lib.stream_ptr()
    _lib.check(lib.uppe3d_begin(sol._plan, L_PROP, TOL, 1e-2, 1e-9, 0, s), 'begin')
    if args.profile_z > 0:
        run_chunks(sol, 10 ** 6, 4, stop=lambda r: r.z >= args.profile_z)
    _lib.check(lib.uppe3d_run_steps(sol._plan, args.warmup, s), 'warmup')
    torch.cuda.synchronize()
    lines = line_stats(sol, med)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push('timed')
    e0.record()
    _lib.check(lib.uppe3d_run_steps(sol._plan, args.steps, s), 'run')
    e1.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    r = sol.result()
    print(json.dumps({'ms_per_attempt': e0.elapsed_time(e1) / args.steps, 'attempts': r.attempts,
                      'accepted': r.accepted, 'z': r.z, 'status': r.status, 'grid': [n, n, NT],
                      'table': args.profile_table, 'lines': lines}), flush=True)
    return 0


def run_profile_batched(args):
    """The batched 1D sweep's longest instance alone, for profiler commands: one
    sweep (untimed) finds the instance with the most attempts; the same instance
    over --profile-l metres runs --warmup times untimed, then once inside an NVTX
    range named "timed" (one launch of the cluster kernel)."""
    import torch
    from project_b200.solver1d import BatchedPropagator
    dev = torch.device('cuda')
    insts, fields = batched1d_instances()
    bp = BatchedPropagator(insts, precision='single', device=dev)
    _, _, res = bp.run(fields)
    k = int(np.argmax([r.attempts for r in res]))
    del bp
    insts_l, fields_l = batched1d_instances(L=args.profile_l)
    one = BatchedPropagator([insts_l[k]], precision='single', device=dev)
    packed0 = one.pack([fields_l[k]])
    work = packed0.clone()
    for _ in range(max(args.warmup, 1)):
        work.copy_(packed0)
        one.run_packed(work)
    work.copy_(packed0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push('timed')
    e0.record()
    r = one.run_packed(work)[0]
    e1.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    print(json.dumps({'instance': k, 'Nt': int(insts_l[k]['desc'].Nt), 'energy_J': insts_l[k]['energy'],
                      'pressure_bar': insts_l[k]['pressure'], 'L_m': args.profile_l,
                      'attempts_full_sweep': int(res[k].attempts), 'attempts': int(r.attempts),
                      'ms': ms, 'ms_per_attempt': ms / max(int(r.attempts), 1),
                      'clusters': int(one._lib.uppe1d_uses_clusters(one._plan))}), flush=True)
    return 0


def run_profile_realfield(args):
    """Only the real-field propagator (the realfield_3d workload), for profiler
    commands: --warmup untimed attempts, then --steps attempts inside an NVTX range
    named "timed"."""
    import torch
    from project_b200.realfield import Argon, ERK43_RealField_UPPE_3D
    N, Nt = 128, 1024
    x = np.linspace(-0.4e-3, 0.4e-3, N)
    t = np.linspace(-100e-15, 100e-15, Nt)
    X, Y = np.meshgrid(x, x, indexing='ij')
    w = 2 * np.pi * 299792458.0 / 800e-9
    env = np.exp(-2 * np.log(2) * t ** 2 / (20e-15) ** 2) * np.cos(w * t)
    E0 = (4e10 * np.exp(-(X ** 2 + Y ** 2) / (0.2e-3) ** 2)[:, :, None] * env[None, None, :]).astype(np.float32)
    sol = ERK43_RealField_UPPE_3D(x, x, t, Argon(800e-9, 1.0), precision='single')
    sol.set_field(torch.from_numpy(E0).cuda())
    for _ in range(args.warmup):
        sol.attempt(1e-6)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push('timed')
    e0.record()
    for _ in range(args.steps):
        sol.attempt(1e-6)
    e1.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    print(json.dumps({'ms_per_attempt': e0.elapsed_time(e1) / max(args.steps, 1), 'grid': [N, N, Nt]}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=4)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--precision', default='single', choices=['single', 'double'])
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-plain-gpu', action='store_true')
    ap.add_argument('--no-batched-1d', action='store_true')
    ap.add_argument('--no-gradients', action='store_true')
    ap.add_argument('--no-realfield', action='store_true')
    ap.add_argument('--no-accuracy', action='store_true')
    ap.add_argument('--no-ionising', action='store_true')
    ap.add_argument('--profile-realfield', action='store_true',
                    help='only the real-field attempts (for profilers): --warmup untimed, --steps in an NVTX range')
    ap.add_argument('--profile-case', action='store_true',
                    help='only the solver: warm-up + timed attempts (a short command for ncu)')
    ap.add_argument('--profile-z', type=float, default=0.0, help='profile case: start the timed attempts at z')
    ap.add_argument('--profile-table', default='adk', choices=['adk', 'mpi'])
    ap.add_argument('--profile-grid', type=int, default=NX)
    ap.add_argument('--profile-tuning', default='', help='profile case: y_tma,y_ctas,y_late,y_kw,t_wpb')
    ap.add_argument('--profile-batched', action='store_true',
                    help='only the batched sweep\'s longest instance over --profile-l m, one timed launch')
    ap.add_argument('--profile-l', type=float, default=0.1)
    ap.add_argument('--pattern-probe', action='store_true',
                    help='only the access-pattern copy bandwidths of the 3D passes (uppe_pattern_probe)')
    args = ap.parse_args()
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local_rank = int(os.environ.get('LOCAL_RANK', '0'))
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == 'reference':
        return run_reference(args, rank)
    if args.profile_realfield:
        return run_profile_realfield(args)
    if args.profile_case:
        return run_profile_case(args)
    if args.profile_batched:
        return run_profile_batched(args)
    if args.pattern_probe:
        import torch
        print(json.dumps({'access_pattern_copy_gbs': pattern_ceilings(torch.device('cuda', local_rank)),
                          'field': [NX, NY, NT], 'dtype': 'c64'}), flush=True)
        return 0
    import datetime
    import torch.distributed as dist
    if world > 1:
        import torch
        torch.cuda.set_device(local_rank)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    try:
        return run_b200(args, rank, world, local_rank)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == '__main__':
    sys.exit(main())
