"""Benchmark: batched mesolve solves/s on one B200 (or N, weak scaling).

Workload (one "step"): the batched driven-Kerr problem -- n=64, 4096 instances, each
H_b = Delta a^+a + (K/2) a^+2 a^2 + eps (a + a^+) with Delta~U(-1,1), K~U(0,0.5),
eps~U(0,2) from a seed, jumps sqrt(0.1) a and sqrt(0.01) a^+a, rho0 = vacuum,
t in [0, 10] with 51 saves, Tsit5 rtol 1e-6 atol 1e-8, complex64 state -- solved to
completion by one launch of the persistent kernel.

Arms:
  default (b200)      value: C-ABI call on device-resident inputs, CUDA events.
                      e2e: the public dq.mesolve from host numpy inputs, including the
                      host->device copies of the inputs and the device->host read of the
                      expectation values and infos (states stay on the device, as the
                      reference returns device arrays).
  --impl reference    the oracle's CPU restatement (numpy) of the reference's loop on
                      the host cores (a process pool), a bounded sample of instances
                      per step.  The reference itself (JAX + diffrax) is not installed.

Multi-GPU (torchrun, --gpus N): every rank solves its own 4096 instances (seed + rank);
no collective on the data path; time = max over ranks; scaling "weak".
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

# The oracle legs run numpy; its OpenBLAS is built with MAX_THREADS=64, whose threaded
# complex GEMM has misbehaved on hosts with more cores.  The CPU legs use one thread per
# process anyway.
for _v in ('OPENBLAS_NUM_THREADS', 'OMP_NUM_THREADS', 'MKL_NUM_THREADS'):
    os.environ.setdefault(_v, '1')
# Streams share CUDA_DEVICE_MAX_CONNECTIONS hardware queues (8 by default); the serving
# configuration runs up to 16 streams whose waves must not queue behind each other.
os.environ.setdefault('CUDA_DEVICE_MAX_CONNECTIONS', '32')

import numpy as np  # noqa: E402

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'mesolve solves/sec vs plain GPU path at equal 1e-5 error; p50/p99 latency'


def _flops_per_rhs(n: int, K: int) -> float:
    # hermitian form: Hnh X, L_k X, (L_k X) L_k^+ -> (1 + 2K) complex n^3 products, 8 flop each
    return (1 + 2 * K) * 8.0 * n ** 3


def _clock_sampler(path):
    q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')
    try:
        return subprocess.Popen(['nvidia-smi', f'--query-gpu={q}', '--format=csv,noheader,nounits',
                                 '-lms', '200', '-i', str(int(os.environ.get('LOCAL_RANK', 0)))],
                                stdout=open(path, 'w'), stderr=subprocess.DEVNULL)
    except OSError:
        return None


def _clock_summary(path):
    try:
        rows = [r.split(',') for r in open(path).read().strip().splitlines() if r.strip()]
    except OSError:
        return None
    sm, smax, reasons = [], None, set()
    names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
    for r in rows:
        try:
            sm.append(float(r[1]))
            smax = float(r[2])
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == 'active':
                    reasons.add(nm)
        except (ValueError, IndexError):
            continue
    if not sm:
        return None
    return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': smax, 'reasons': sorted(reasons),
            'samples': len(sm)}


def _peaks():
    try:
        d = json.load(open(os.path.join(ROOT, 'MEASURED_PEAKS.json')))
        return d, 'measured'
    except OSError:
        return {'hbm_gbs': 6650.0, 'bf16_tflops': 1590.0, 'bf16_tflops_sustained': 1400.0}, 'fallback'


# --------------------------------------------------------------------------------------
# CPU legs (oracle)
# --------------------------------------------------------------------------------------

def _kerr_config(batch):
    return {'workload': CASES['kerr'], 'batch_per_gpu': batch, 'n': 64, 'n_jumps': 2,
            'n_tsave': 51, 'method': 'Tsit5', 'rtol': 1e-6, 'atol': 1e-8}


def _oracle_solve(args):
    """One oracle solve of instance `b` of the workload (complex64 state); returns its
    number of attempted steps."""
    b, seed = args
    from dynamiqs_b200 import workloads
    from oracle.mesolve import mesolve as om

    w = workloads.batched_kerr(batch=b + 1, seed=seed)
    r = om(w['H'][b], w['jump_ops'], w['rho0'], w['tsave'], exp_ops=w['exp_ops'],
           rtol=1e-6, atol=1e-8, dtype=np.complex64)
    return r.nsteps


def cpu_baseline(sample: int = 3, seed: int = 0) -> dict:
    t = time.perf_counter()
    for b in range(sample):
        _oracle_solve((b, seed))
    dt = time.perf_counter() - t
    return {'value': sample / dt, 'unit': 'solves/s', 'cores': 1, 'kind': 'port',
            'sample': f'{sample} instances of the workload through the numpy oracle '
                      f'(complex64 state, 1 thread), {dt:.1f} s'}


def _host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def run_reference(args):
    """The reference's loop restated on the CPU (the oracle: numpy, complex64 state, one
    thread per process) on every host core, through one continuous work queue: each step is
    a sample of 2 x cores distinct instances of the workload's batch, all steps' instances
    are queued at once (imap_unordered, chunksize 1), so no core idles at a step boundary
    and the timed throughput is load-balanced; the only tail is the last few instances."""
    import multiprocessing as mp

    rank = int(os.environ.get('RANK', 0))
    if rank != 0:
        return
    cores = _host_cores()
    per_step = 2 * cores
    ctx = mp.get_context('spawn')
    os.environ.setdefault('OMP_NUM_THREADS', '1')
    os.environ.setdefault('OPENBLAS_NUM_THREADS', '1')
    os.environ.setdefault('MKL_NUM_THREADS', '1')
    B = 4096
    tasks = [(i % B, i // B) for i in range(args.steps * per_step)]
    with ctx.Pool(cores) as pool:
        warm = [(B - 1 - i, 1000 + w) for w in range(args.warmup) for i in range(cores)]
        for _ in pool.imap_unordered(_oracle_solve, warm, chunksize=1):
            pass
        t = time.perf_counter()
        steps_done = sum(pool.imap_unordered(_oracle_solve, tasks, chunksize=1))
        total = time.perf_counter() - t
    value = len(tasks) / total
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': 'solves/s',
        'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': 1e3 * total / args.steps, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'c64', 'data': 'synthetic (seeded numpy generator; no dataset)',
        'config': dict(_kerr_config(B), sample_per_step=per_step,
                       avg_rk_steps_of_sample=steps_done / len(tasks)),
        'cpu_baseline': {'value': value, 'unit': 'solves/s', 'cores': cores, 'kind': 'port',
                         'sample': f'{args.steps} steps x {per_step} distinct instances of the '
                                   'workload (instances 0.. of its seed-0 batch) through the numpy '
                                   'oracle, one process per core, one work queue; the reference '
                                   '(JAX + diffrax) is not installed on this image'},
        'e2e': {'value': value, 'unit': 'solves/s', 'h2d_bytes_per_step': 0,
                'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------------------

CASES = {
    'kerr': 'batched driven Kerr: n=64, B=4096, K=2 jumps, t=[0,10], 51 saves, Tsit5 1e-6/1e-8',
    'oscillator': 'lossy oscillator: n=16, one instance, omega=1, kappa=0.1, alpha0=1, 101 saves, '
                  'Tsit5 1e-6/1e-8',
    'transmon': 'transmon(4) x cavity(64): n=256, B=256, K=2, t=[0,20], 41 saves, Tsit5 1e-6/1e-8',
    'dia': 'coupled Kerr modes 64x64 in sparse DIA: n=4096, B=8, K=2, t=[0,5], 11 saves, '
           'Tsit5 1e-5/1e-7',
    'serving': 'Poisson stream (2000 req/s) of Kerr requests, n in {8..256} weights '
               '(.30,.25,.20,.15,.07,.03), 1-3 jumps, t_end~U(1,20), 11-201 saves, Tsit5 1e-6',
}


def run_serving(args):
    """Replay a seeded Poisson arrival schedule against MESolveServer in real time."""
    import threading

    import torch

    import dynamiqs_b200 as dq
    from dynamiqs_b200 import workloads
    from dynamiqs_b200.server import MESolveServer

    rank = int(os.environ.get('RANK', 0))
    if rank != 0:
        return
    torch.cuda.set_device(0)
    N = args.batch or 2000
    reqs = workloads.serving_requests(N, rate=2000.0, seed=args.seed)
    warm = workloads.serving_requests(24, rate=2000.0, seed=args.seed + 999)
    srv = MESolveServer(n_streams=args.streams)

    def opts_of(r):  # GEMM-path arithmetic for n > 64; the n <= 64 kernel is FP32
        return dq.Options(precision=args.precision if r['n'] > 64 else 'fp32')

    # every large-path graph the stream will use is captured here, before the clock starts
    srv.warmup(method=reqs[0]['method'], options=dq.Options(precision=args.precision))

    for r in warm:
        srv.submit(r['H'], r['jump_ops'], r['rho0'], r['tsave'], exp_ops=r['exp_ops'],
                   method=r['method'], options=opts_of(r))
    while len(srv.finished) < len(warm):
        time.sleep(0.01)
    for t in srv.finished:
        t.release()
    srv.finished.clear()
    clk_path = os.path.join(tempfile.gettempdir(), 'dqb_bench_clocks_rank0.csv')
    os.makedirs(os.path.dirname(clk_path), exist_ok=True)
    sampler = _clock_sampler(clk_path)
    tickets = []

    def feed():
        t0 = time.perf_counter()
        for r in reqs:
            delay = r['arrival'] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            tickets.append(srv.submit(r['H'], r['jump_ops'], r['rho0'], r['tsave'],
                                      exp_ops=r['exp_ops'], method=r['method'],
                                      options=opts_of(r)))

    th = threading.Thread(target=feed)
    th.start()
    th.join()
    for t in tickets:
        t._event.wait()
    srv.close()
    failed = [t for t in tickets if t._error is not None]
    tickets = [t for t in tickets if t._error is None]
    nsteps_of = {t.id: int(t.result().infos.nsteps) for t in tickets}
    for t in tickets:
        t.release()
    if sampler is not None:
        sampler.terminate()
        sampler.wait()
    st = srv.stats()
    flops = 0.0
    for t in tickets:
        flops += (6 * nsteps_of[t.id] + 2) * _flops_per_rhs(t.n, len(t.Ls))
    achieved = flops / st['makespan_s'] / 1e12
    peaks, which = _peaks()
    peak = peaks.get('bf16_tflops_sustained', peaks.get('bf16_tflops'))
    # plain path: the same requests one per launch, in arrival order, no overlap
    plain = None
    if not args.no_plain:
        sample = reqs[: min(len(reqs), args.plain_sample)]
        lat = []
        t0 = time.perf_counter()
        for r in sample:
            a = time.perf_counter()
            res = dq.mesolve(r['H'], r['jump_ops'], r['rho0'], r['tsave'], exp_ops=r['exp_ops'],
                             method=r['method'], options=opts_of(r))
            res.infos.nsteps.cpu()
            lat.append(time.perf_counter() - a)
        tot = time.perf_counter() - t0
        plain = {'value': len(sample) / tot, 'unit': 'solves/s',
                 'what': f'dq.mesolve one request per launch, {len(sample)} requests back to back',
                 'p50_latency_ms': 1e3 * float(np.percentile(lat, 50)),
                 'p99_latency_ms': 1e3 * float(np.percentile(lat, 99)),
                 'served_over_plain': st['solves_per_s'] / (len(sample) / tot)}
    by_n, steps_n = {}, {}
    for t in tickets:
        by_n.setdefault(t.n, []).append(1e3 * t.latency)
        steps_n.setdefault(t.n, []).append(nsteps_of[t.id])
    per_size = {str(n): {'count': len(v), 'p50_ms': float(np.percentile(v, 50)),
                         'p99_ms': float(np.percentile(v, 99)),
                         'mean_rk_steps': float(np.mean(steps_n[n])),
                         'max_rk_steps': int(np.max(steps_n[n]))}
                for n, v in sorted(by_n.items())}
    line = {
        'metric': METRIC, 'value': st['solves_per_s'], 'unit': 'solves/s', 'n_gpus': 1,
        'steps': 1, 'warmup': 1, 'ms_per_step': 1e3 * st['makespan_s'], 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'c64',
        'data': 'synthetic (seeded Poisson arrivals and Kerr problems)',
        'config': {'workload': CASES['serving'], 'requests': N, 'streams': args.streams,
                   'precision_n_gt_64': args.precision,
                   'waves': st['waves'], 'errors': st['errors'],
                   'error_kinds': sorted({f'n={t.n}: {t._error}' for t in failed})[:5],
                   'max_launch_s': max((x[2] for x in srv.launch_seconds), default=0.0),
                   'slow_launches': [(str(k), c, round(sec, 3)) for k, c, sec in srv.launch_seconds
                                     if sec > 0.5][:10],
                   'slow_steps': [(str(k), {a: round(b, 3) for a, b in pr.items() if b > 0.1})
                                  for k, pr in srv.launch_profile if max(pr.values()) > 0.1][:12]},
        'latency_ms': {'p50': st['p50_ms'], 'p99': st['p99_ms'], 'mean': st['mean_ms'],
                       'per_dim': per_size},
        'e2e': {'value': st['solves_per_s'], 'unit': 'solves/s',
                'h2d_bytes_per_step': None, 'd2h_bytes_per_step': None},
        'roofline': {'bound': 'tensor', 'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s',
                     'frac': achieved / peak, 'peak_source': f'bf16_tflops_sustained ({which})',
                     'traffic': None},
        'clocks': _clock_summary(clk_path),
        'plain_path': plain,
    }
    print(json.dumps(line), flush=True)


def _workload(name, args, rank):
    from dynamiqs_b200 import workloads

    seed = args.seed + rank
    if name == 'kerr':
        w = workloads.batched_kerr(batch=args.batch or 4096, n=args.n or 64, seed=seed)
        if args.tend != 10.0:
            w['tsave'] = np.linspace(0.0, args.tend, 51)
    elif name == 'oscillator':
        w = workloads.lossy_oscillator()
    elif name == 'transmon':
        w = workloads.transmon_cavity(batch=args.batch or 256, seed=seed)
        if args.tend != 10.0:
            w['tsave'] = np.linspace(0.0, args.tend, 41)
    else:
        w = workloads.coupled_kerr_dia(batch=args.batch or 8, seed=seed)
        if args.tend != 10.0:
            w['tsave'] = np.linspace(0.0, args.tend, 11)
    return w


def _kernels_per_launch(path: str, K: int, iterations: int, stepper: str = 'auto') -> int:
    """Kernels of this library executed by one solve call."""
    if path == 'dqb_mesolve_dense':
        return 1  # the persistent kernel (plus a 256-byte memset of its work counter)
    if path == 'dqb_mesolve_dia':
        if stepper != 'krylov':
            body = 6 * 2 + 4      # 6 x (combine + stencil) + error, control, save, commit
            init = 10             # set-up, Hnh, rho0, 2 RHS, norms, controls, probe
        else:
            body = 6 + 4          # 6 basis stencils + combination, control, save, commit
            init = 9              # set-up, Hnh, rho0, 2 RHS, 2 norms, 2 controls
        return init + body * iterations + 3
    rhs = (2 if K else 1) + 1 + ((K + 1) // 4 if K > 3 else 0)  # L X, sums, symmetrize
    if stepper != 'krylov':
        body = 6 * (1 + rhs) + 4  # 6 x (combine + RHS) + error, control, save, commit
        init = 3 + 2 * rhs + 5 + (K + 3) // 4
    else:
        body = 6 * rhs + 4        # 6 basis RHS + combination, control, save, commit
        init = 3 + 2 * rhs + 4 + (K + 3) // 4
    return init + body * iterations + 3


def _roofline(config, precision, n, K, nsteps, mean_ms, B, peaks, which, nsave=0, nacc=None,
              stepper='auto'):
    """Roofline record of the dominant kernel of a solve launch: `nsteps` (tensor) is the
    attempted RK steps of every instance, `nacc` the accepted ones, `mean_ms` the launch's
    mean duration."""
    import torch

    if config == 'dia':
        mat = 8.0 * n * n
        # the stage-by-stage step touches at least 34 n x n complex64 matrices per attempt
        # (stages 2-6 read y and k_1..k_{i-1} and write k_i: 25 passes; y1, k7 and the error
        # 9 more) -- the figure of a fully fused stage-form step
        stage_bytes = float((34 * mat * nsteps).sum())
        if stepper != 'krylov':
            nbytes = stage_bytes
            note = ('bytes = 34 n^2 complex64 matrix passes per attempted RK step per '
                    'instance (the fused stage-form minimum of whole-matrix kernels); the '
                    'hermitian-half kernels move 3.60 GB = 27 passes per attempt (measured '
                    'DRAM bytes, see traffic)')
        else:
            # the Krylov form: per accepted step six right-hand sides build the basis (read
            # one matrix, write one: 12 passes); per attempt one pass reads u_0..u_7 and
            # writes y1 and the next first stage (10 passes); per save point the dense
            # output reads the basis and writes the state (9 passes).  (The hermitian-half
            # kernels read about half of each hermitian matrix: the counts are of whole
            # matrices, as the stage form's 34.)
            nbytes = float((mat * (12 * nacc + 10 * nsteps)).sum()) + 9 * mat * nsave * B
            note = ('bytes = the Krylov-form step: 12 n^2 complex64 passes per accepted step '
                    '(basis), 10 per attempt (combination), 9 per save point; the same step '
                    'in the stage form needs at least 34 per attempt')
        achieved = nbytes / (mean_ms / 1e3) / 1e9
        roof = {'bound': 'hbm', 'achieved': achieved, 'peak': peaks['hbm_gbs'], 'unit': 'GB/s',
                'frac': achieved / peaks['hbm_gbs'], 'peak_source': f'hbm_gbs ({which})',
                'traffic': _traffic(config, precision, B, nsteps, nsave, stepper, nacc),
                'algorithmic_bytes_per_launch': nbytes, 'note': note}
        if stepper == 'krylov':
            eff = stage_bytes / (mean_ms / 1e3) / 1e9
            roof['stage_form_equivalent'] = {
                'achieved': eff, 'frac': eff / peaks['hbm_gbs'],
                'note': 'the 34-pass stage-form bytes of the same attempted steps over the '
                        'measured time: the HBM bandwidth a stage-form step would need to '
                        'match this speed'}
        return roof
    rhs_evals = float((6 * nsteps + 2).sum())
    flops = rhs_evals * _flops_per_rhs(n, K)
    achieved = flops / (mean_ms / 1e3) / 1e12
    peak = peaks.get('bf16_tflops_sustained', peaks.get('bf16_tflops'))
    roof = {'bound': 'tensor', 'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s',
            'frac': achieved / peak, 'peak_source': f'bf16_tflops_sustained ({which})',
            'traffic': _traffic(config, precision, B, nsteps), 'algorithmic_flops_per_launch': flops}
    if precision == 'fp32' or (precision in ('tf32x3', 'bf16x3', 'tf32') and n <= 64):
        roof['note'] = ('products run on the FP32 CUDA-core pipe (SIMT), not the tensor '
                        'pipe; see roofline_fp32_simt')
        if n <= 64 and K > 0:
            R = (16 if n <= 16 else (32 if n <= 32 else 64)) // 16
            part = (R + 1) * R / 2 / (R * R)
            roof['note'] += ('. Algorithmic flops count (1+2K) complex products per RHS; '
                             f'the hermitian form computes (L X) L^+ on {part:.3f} of the '
                             'tile pairs, so the kernel executes '
                             f'{(1 + K + K * part) / (1 + 2 * K):.3f} of them')
    elif precision in ('f16x3', 'auto') and n <= 64:
        roof['note'] = ('products run on tcgen05 tensor cores (f16x3: a complex 64^3 product is '
                        'one 128x128x64 real MMA, the same real work, taken three times on the hi '
                        'and lo FP16 parts, so the tensor pipe executes 3x the algorithmic flops)')
    else:
        roof['note'] = (f'products run on tcgen05 tensor cores ({precision}: three products '
                        'per complex MAC term, so the tensor pipe executes 3x the algorithmic '
                        'flops)')
    return roof


# DRAM bytes (read + write) per unit of work of each solve, from one ncu capture of
# dram__bytes_read.sum + dram__bytes_write.sum on a smaller launch of the same workload,
# scaled to the benchmark launch by the units it processes:
#   kerr / fp32: per instance (148 instances, the full t in [0, 10] and 51 saves: 419.9 MB
#     for 148 = 2.837 MB; inputs, states and expectation values, the RK slots stay in L2);
#     profiles/mesolve_small_kernel_n64_kerr.md.
#   dia / fp32, stage form: per attempted RK step of one instance (every kernel of the
#     stepper, host loop: six hermitian-half stage combinations 2.36 GB, six stencils
#     writing the upper tiles of their stage slot 0.64 GB, the hermitian-half error pass
#     0.61 GB: 3.60 GB) plus 0.81 GB per save point (a step that crosses saves reads the
#     upper tiles of y, the seven stages and the expectation operators, 0.68 GB, and each
#     save writes its state, 0.13 GB); profiles/dia_stepper_n4096_coupled_kerr_traffic.md.
#   dia / fp32, Krylov form: 0.917 GB per accepted step (six basis stencils, 69.9 MB read
#     + 82.9 MB written each), 0.774 GB per attempt (the hermitian-half combination pass:
#     541.1 MB read, 233.3 MB written) and 0.81 GB per save point; same profile.
TRAFFIC_PER_UNIT = {
    ('kerr', 'fp32', 'auto'): ('instance', 2.837e6, 0.0, 0.0),
    ('dia', 'fp32', 'stages'): ('instance_step', 3.60e9, 0.0, 0.81e9),
    ('dia', 'fp32', 'krylov'): ('instance_step', 0.774e9, 0.917e9, 0.81e9),
}


def _traffic(config, precision, B, nsteps, nsave=0, stepper='auto', nacc=None):
    key = (config, precision, ('krylov' if stepper == 'krylov' else 'stages') if config == 'dia' else 'auto')
    if key not in TRAFFIC_PER_UNIT:
        return None
    unit, per, per_acc, per_save = TRAFFIC_PER_UNIT[key]
    units = B if unit == 'instance' else float(nsteps.sum())
    acc = 0.0 if nacc is None else float(nacc.sum())
    return float(per * units + per_acc * acc + per_save * nsave * B)


def run_b200(args):
    import torch

    import dynamiqs_b200 as dq
    from dynamiqs_b200.mesolve import MESolveB200Integrator, make_batch_plan

    world = int(os.environ.get('WORLD_SIZE', 1))
    rank = int(os.environ.get('RANK', 0))
    local = int(os.environ.get('LOCAL_RANK', 0))
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group('nccl', timeout=datetime.timedelta(seconds=600))
        dist = dist_mod

    def barrier():
        if dist is not None:
            dist.barrier(device_ids=[local])
        torch.cuda.synchronize()

    w = _workload(args.config, args, rank)
    Es = w.get('exp_ops')
    opts = dq.Options(precision=args.precision, stepper=args.stepper)
    plan = make_batch_plan(w['H'], w['jump_ops'], w['rho0'], True)
    integ = MESolveB200Integrator(ts=w['tsave'], y0=w['rho0'], method=w['method'], gradient=None,
                                  options=opts, H=w['H'], Ls=w['jump_ops'], Es=Es, plan=plan)
    prep = integ.prepare()
    B = plan.batch
    n = w['H'].shape[-1]
    K = len(w['jump_ops'])
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    for _ in range(args.warmup):
        prep.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    status = prep.bufs['status']
    assert int((status != 0).sum()) == 0, 'solver status not OK'

    # ---- timed region: device-resident inputs --------------------------------------
    clk_path = os.path.join(tempfile.gettempdir(), f'dqb_bench_clocks_rank{rank}.csv')
    os.makedirs(os.path.dirname(clk_path), exist_ok=True)
    sampler = _clock_sampler(clk_path)
    time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    barrier()
    for i in range(args.steps):
        flush.zero_()  # L2 flush between iterations (256 MiB > 126 MB L2)
        ev[i][0].record(stream)
        prep.launch(stream.cuda_stream)
        ev[i][1].record(stream)
    barrier()
    if sampler is not None:
        sampler.terminate()
        sampler.wait()
    kernel_ms = [a.elapsed_time(b) for a, b in ev]
    infos = prep.bufs['infos']
    nsteps = infos[:, 0].to(torch.float64)
    nacc = infos[:, 1].to(torch.float64)
    kern = float(np.sum(kernel_ms))
    if dist is not None:
        tt = torch.tensor([kern], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        kern = float(tt[0])
    value = world * B * args.steps / (kern / 1e3)
    mean_ms = kern / args.steps
    peaks, which = _peaks()
    roof = _roofline(args.config, args.precision, n, K, nsteps, mean_ms, B, peaks, which,
                     len(w['tsave']), nacc, args.stepper)

    # ---- e2e: public API from host inputs --------------------------------------------
    e2e = None
    if not args.no_e2e:
        H_host = w['H']
        if isinstance(H_host, np.ndarray):
            H_host = torch.from_numpy(H_host).pin_memory()
        times = []
        for i in range(max(1, args.e2e_steps) + 1):
            barrier()
            t = time.perf_counter()
            res = dq.mesolve(H_host, w['jump_ops'], w['rho0'], w['tsave'], exp_ops=Es,
                             method=w['method'], options=opts)
            ex = res.expects.cpu() if res.expects is not None else torch.zeros(0)
            inf = res.infos.nsteps.cpu()
            torch.cuda.synchronize()
            if i > 0:
                times.append(time.perf_counter() - t)
        e2e_s = float(np.mean(times))
        if dist is not None:
            tt = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_s = float(tt[0])

        def nb(x):
            return x.diags.nbytes if hasattr(x, 'diags') else np.asarray(x).nbytes

        h2d = (nb(w['H']) + sum(nb(L) for L in w['jump_ops']) + np.asarray(w['rho0']).nbytes
               + (sum(np.asarray(E).nbytes for E in Es) if Es else 0) + w['tsave'].nbytes)
        d2h = ex.numel() * ex.element_size() + inf.numel() * inf.element_size()
        e2e = {'value': world * B / e2e_s, 'unit': 'solves/s', 'h2d_bytes_per_step': int(h2d),
               'd2h_bytes_per_step': int(d2h)}

    # ---- plain path: one instance per launch, FP32 ------------------------------------
    plain = None
    if args.config in ('kerr', 'transmon') and not args.no_plain and rank == 0:
        nplain = 16 if args.config == 'kerr' else 4
        lat = []
        for b in range(nplain):
            p1 = make_batch_plan(w['H'][b], w['jump_ops'], w['rho0'], True)
            i1 = MESolveB200Integrator(ts=w['tsave'], y0=w['rho0'], method=w['method'],
                                       gradient=None, options=dq.Options(), H=w['H'][b],
                                       Ls=w['jump_ops'], Es=Es, plan=p1).prepare()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            i1.launch(stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            lat.append(e0.elapsed_time(e1))
        plain_s = float(np.sum(lat)) / 1e3
        plain = {'value': nplain / plain_s, 'unit': 'solves/s',
                 'what': f'{prep.name} with FP32 products, one instance per launch '
                         f'({nplain} instances)',
                 'p50_latency_ms': float(np.percentile(lat, 50)),
                 'p99_latency_ms': float(np.percentile(lat, 99)),
                 'batched_over_plain': value / world / (nplain / plain_s)}

    if dist is not None:
        dist.barrier(device_ids=[local])
        dist.destroy_process_group()
    if rank != 0:
        return

    clocks = _clock_summary(clk_path)
    extra = {}
    if roof['bound'] == 'tensor' and args.precision == 'fp32':
        # the FP32 FMA pipe: 148 SMs x 128 lanes x 2 flop per clock, at the sampled SM clock
        mhz = (clocks or {}).get('sm_mhz') or peaks.get('sm_max_mhz', 1965.0)
        simt = 148 * 128 * 2 * mhz * 1e6 / 1e12
        extra['roofline_fp32_simt'] = {'bound': 'fp32_fma', 'achieved': roof['achieved'],
                                       'peak': simt, 'unit': 'TFLOP/s',
                                       'frac': roof['achieved'] / simt,
                                       'peak_source': f'nominal at the sampled {mhz:.0f} MHz'}
    line = {
        'metric': METRIC, 'value': value, 'unit': 'solves/s', 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': mean_ms,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'c64',
        'data': 'synthetic (seeded numpy generator; no dataset)',
        'config': {'workload': CASES[args.config] if n == 64 or args.config != 'kerr' else
                   CASES['kerr'].replace('n=64', f'n={n}'), 'batch_per_gpu': B, 'n': n, 'n_jumps': K,
                   'n_tsave': len(w['tsave']), 'method': type(w['method']).__name__,
                   'rtol': w['method'].rtol, 'atol': w['method'].atol, 'path': prep.name,
                   'precision': args.precision,
                   **({'stepper': args.stepper} if args.config in ('dia', 'transmon') else {}),
                   'l2': 'flushed between iterations (256 MiB write)',
                   'parallelism': f'instances sharded over {world} GPU(s), no collective',
                   'avg_rk_steps': float(nsteps.mean()), 'max_rk_steps': float(nsteps.max())},
        'e2e': e2e,
        'gpu_launches': args.steps * _kernels_per_launch(prep.name, K, int(nsteps.max()),
                                                         args.stepper),
        'roofline': roof,
        **extra,
        'clocks': clocks,
        'plain_path': plain,
        'latency_ms': {'per_batch': mean_ms},
    }
    if args.config == 'kerr' and not args.no_cpu_baseline:
        line['cpu_baseline'] = cpu_baseline(sample=args.cpu_sample)
    if args.config == 'kerr' and world == 1 and not args.no_extra:
        line['extra_configs'] = _extra_configs(args, dev, stream, flush, peaks, which)
    print(json.dumps(line), flush=True)


def _extra_configs(args, dev, stream, flush, peaks, which):
    """The tensor-core GEMM path (transmon x cavity, n = 256, 3xTF32) and the sparse-DIA
    path (coupled Kerr modes, n = 4096) measured in the same run as the headline, on
    device-resident inputs with the headline's timing rules (CUDA events on the launching
    stream, L2 flushed between launches), 3 warm-up and 2 timed launches each; each with the
    default stage form of the step and with the opt-in Krylov form."""
    import torch

    import dynamiqs_b200 as dq
    from dynamiqs_b200.mesolve import MESolveB200Integrator, make_batch_plan

    out = {}
    for key, cfg, prec, stepper in (('transmon_tf32x3', 'transmon', 'tf32x3', 'auto'),
                                    ('transmon_tf32x3_krylov', 'transmon', 'tf32x3', 'krylov'),
                                    ('coupled_kerr_dia', 'dia', 'fp32', 'auto'),
                                    ('coupled_kerr_dia_krylov', 'dia', 'fp32', 'krylov')):
        sub = argparse.Namespace(**vars(args))
        sub.batch, sub.n, sub.tend = 0, 0, 10.0
        w = _workload(cfg, sub, 0)
        plan = make_batch_plan(w['H'], w['jump_ops'], w['rho0'], True)
        prep = MESolveB200Integrator(ts=w['tsave'], y0=w['rho0'], method=w['method'], gradient=None,
                                     options=dq.Options(precision=prec, stepper=stepper), H=w['H'],
                                     Ls=w['jump_ops'],
                                     Es=w.get('exp_ops'), plan=plan).prepare()
        for _ in range(3):
            prep.launch(stream.cuda_stream)
        torch.cuda.synchronize()
        assert int((prep.bufs['status'] != 0).sum()) == 0, f'{key}: solver status not OK'
        ms = []
        for _ in range(2):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            prep.launch(stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        nsteps = prep.bufs['infos'][:, 0].to(torch.float64)
        nacc = prep.bufs['infos'][:, 1].to(torch.float64)
        B = plan.batch
        n = int(w['H'].shape[-1])
        mean_ms = float(np.mean(ms))
        out[key] = {'workload': CASES[cfg], 'path': prep.name, 'precision': prec,
                    'value': B / (mean_ms / 1e3), 'unit': 'solves/s', 'ms_per_step': mean_ms,
                    'steps': 2, 'warmup': 3, 'batch': B, 'avg_rk_steps': float(nsteps.mean()),
                    'max_rk_steps': float(nsteps.max()),
                    'stepper': stepper,
                    'roofline': _roofline(cfg, prec, n, len(w['jump_ops']), nsteps, mean_ms, B,
                                          peaks, which, len(w['tsave']), nacc, stepper)}
        del prep
        torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--config', default='kerr', choices=sorted(CASES))
    ap.add_argument('--batch', type=int, default=0, help='instances (0: the workload default)')
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--n', type=int, default=0, help='kerr: Hilbert dimension (0: 64, the workload)')
    ap.add_argument('--tend', type=float, default=10.0, help='end time (10 in the workload; '
                    'shorter only for profiling captures)')
    ap.add_argument('--e2e-steps', type=int, default=1)
    ap.add_argument('--cpu-sample', type=int, default=3)
    ap.add_argument('--streams', type=int, default=16, help='serving: CUDA streams')
    ap.add_argument('--plain-sample', type=int, default=100, help='serving: plain-path sample')
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-plain', action='store_true')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-extra', action='store_true',
                    help='skip the GEMM-path and DIA lines the kerr run adds (extra_configs)')
    ap.add_argument('--stepper', default='auto', choices=['auto', 'stages', 'krylov'],
                    help='dia, transmon: form of the RK step (auto = stages)')
    ap.add_argument('--precision', default='fp32',
                    choices=['fp32', 'tf32x3', 'bf16x3', 'tf32', 'f16x3', 'auto'],
                    help='arithmetic of the complex products (tf32x3 / bf16x3 / tf32: GEMM '
                         'path, n > 64; f16x3: the n <= 64 kernel)')
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    elif args.config == 'serving':
        run_serving(args)
    else:
        run_b200(args)


if __name__ == '__main__':
    main()
