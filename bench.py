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
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = 'batched driven Kerr: n=64, B=4096, K=2 jumps, t=[0,10], 51 saves, Tsit5 1e-6/1e-8'
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

def _oracle_solve(args):
    """One oracle solve of instance `b` of the workload (complex64 state)."""
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


def run_reference(args):
    import multiprocessing as mp

    rank = int(os.environ.get('RANK', 0))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    per_step = cores  # one instance per core per step
    ctx = mp.get_context('spawn')
    os.environ.setdefault('OMP_NUM_THREADS', '1')
    os.environ.setdefault('OPENBLAS_NUM_THREADS', '1')
    os.environ.setdefault('MKL_NUM_THREADS', '1')
    with ctx.Pool(cores) as pool:
        for w in range(args.warmup):
            pool.map(_oracle_solve, [(b, 1000 + w) for b in range(per_step)])
        times = []
        for s in range(args.steps):
            t = time.perf_counter()
            pool.map(_oracle_solve, [(b, s) for b in range(per_step)])
            times.append(time.perf_counter() - t)
    total = sum(times)
    value = per_step * args.steps / total
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': 'solves/s',
        'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': 1e3 * total / args.steps, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'c64', 'data': 'synthetic (seeded)',
        'config': {'workload': WORKLOAD, 'sample_per_step': per_step},
        'cpu_baseline': {'value': value, 'unit': 'solves/s', 'cores': cores, 'kind': 'port',
                         'sample': f'{per_step} instances per step (one per core) through '
                                   'the numpy oracle; the reference (JAX + diffrax) is not '
                                   'installed on this image'},
        'e2e': {'value': value, 'unit': 'solves/s', 'h2d_bytes_per_step': 0,
                'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------------------

def run_b200(args):
    import torch

    import dynamiqs_b200 as dq
    from dynamiqs_b200 import _lib, workloads

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

    B = args.batch
    w = workloads.batched_kerr(batch=B, seed=args.seed + rank)
    n, K = 64, 2
    lib = _lib.load()
    c64 = torch.complex64
    H_d = torch.from_numpy(w['H']).to(dev)
    L_d = torch.from_numpy(np.stack(w['jump_ops'])[None].copy()).to(dev)
    r_d = torch.from_numpy(w['rho0'].copy()).to(dev)
    E_d = torch.from_numpy(np.stack(w['exp_ops']).copy()).to(dev)
    ts = w['tsave'] if args.tend == 10.0 else np.linspace(0.0, args.tend, 51)
    ts_d = torch.from_numpy(ts).to(dev)
    zeros = torch.zeros(B, dtype=torch.int32, device=dev)
    H_idx = torch.arange(B, dtype=torch.int32, device=dev)
    nt = len(ts)
    states = torch.empty((B, nt, n, n), dtype=c64, device=dev)
    expects = torch.empty((B, 1, nt), dtype=c64, device=dev)
    infos = torch.empty((B, 3), dtype=torch.int32, device=dev)
    status = torch.empty((B,), dtype=torch.int32, device=dev)
    prob = _lib.DenseProblem(n=n, n_jumps=K, n_exp=1, n_tsave=nt, batch=B, H=H_d.data_ptr(),
                             L=L_d.data_ptr(), rho0=r_d.data_ptr(), rho0_is_ket=1,
                             E=E_d.data_ptr(), tsave=ts_d.data_ptr(), H_index=H_idx.data_ptr(),
                             L_index=zeros.data_ptr(), rho0_index=zeros.data_ptr())
    outs = _lib.Outputs(states=states.data_ptr(), expects=expects.data_ptr(),
                        infos=infos.data_ptr(), status=status.data_ptr())
    opts = _lib.OdeOptions(method=_lib.METHOD_TSIT5, form=_lib.FORM_HERMITIAN, rtol=1e-6,
                           atol=1e-8, safety=0.9, factormin=0.2, factormax=5.0,
                           max_steps=100_000, t0=float(ts[0]), save_states=1, check_hermitian=1)
    ws_bytes = lib.dqb_mesolve_dense_workspace_size(n, K, B)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    def step():
        rc = lib.dqb_mesolve_dense(prob, opts, outs, ws.data_ptr(), ws_bytes, stream.cuda_stream)
        _lib.check(rc, 'dqb_mesolve_dense')

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    assert int((status != 0).sum()) == 0, 'solver status not OK'

    # ---- timed region: device-resident inputs --------------------------------------
    clk_path = os.path.join(ROOT, 'gpurun_out', f'clocks_rank{rank}.csv')
    os.makedirs(os.path.dirname(clk_path), exist_ok=True)
    sampler = _clock_sampler(clk_path)
    time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    barrier()
    t_start = torch.cuda.Event(enable_timing=True)
    t_stop = torch.cuda.Event(enable_timing=True)
    kernel_ms = []
    t_start.record(stream)
    for i in range(args.steps):
        flush.zero_()  # L2 flush between iterations (256 MiB > 126 MB L2)
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
    t_stop.record(stream)
    barrier()
    if sampler is not None:
        sampler.terminate()
        sampler.wait()
    kernel_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = t_start.elapsed_time(t_stop)
    nsteps = infos[:, 0].to(torch.float64)
    rhs_evals = float((6 * nsteps + 2).sum())
    flops_per_solve_batch = rhs_evals * _flops_per_rhs(n, K)
    # max over ranks
    kern = float(np.sum(kernel_ms))
    if dist is not None:
        tt = torch.tensor([kern, total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        kern, total_ms = float(tt[0]), float(tt[1])
    value = world * B * args.steps / (kern / 1e3)
    mean_kernel_ms = kern / args.steps
    achieved_tflops = flops_per_solve_batch / (mean_kernel_ms / 1e3) / 1e12

    # ---- e2e: public API from host inputs --------------------------------------------
    e2e_value = None
    h2d = d2h = 0
    if not args.no_e2e:
        H_host = torch.from_numpy(w['H']).pin_memory()
        Ls = w['jump_ops']
        e2e_times = []
        for i in range(max(1, args.e2e_steps) + 1):
            barrier()
            t = time.perf_counter()
            res = dq.mesolve(H_host, Ls, w['rho0'], ts, exp_ops=w['exp_ops'], method=w['method'])
            ex = res.expects.cpu()
            inf = res.infos.nsteps.cpu()
            torch.cuda.synchronize()
            if i > 0:
                e2e_times.append(time.perf_counter() - t)
        e2e_s = max(e2e_times) if dist is None else e2e_times[-1]
        if dist is not None:
            tt = torch.tensor([float(np.mean(e2e_times))], device=dev, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_s = float(tt[0])
        else:
            e2e_s = float(np.mean(e2e_times))
        e2e_value = world * B / e2e_s
        h2d = (w['H'].nbytes + sum(L.nbytes for L in Ls) + w['rho0'].nbytes
               + sum(E.nbytes for E in w['exp_ops']) + ts.nbytes)
        d2h = ex.numel() * ex.element_size() + inf.numel() * inf.element_size()

    # ---- plain path: one instance per launch -------------------------------------------
    plain = None
    if not args.no_plain and rank == 0:
        nplain = 16
        p1 = _lib.DenseProblem(n=n, n_jumps=K, n_exp=1, n_tsave=nt, batch=1, H=0,
                               L=L_d.data_ptr(), rho0=r_d.data_ptr(), rho0_is_ket=1,
                               E=E_d.data_ptr(), tsave=ts_d.data_ptr(), H_index=None,
                               L_index=zeros.data_ptr(), rho0_index=zeros.data_ptr())
        ws1 = lib.dqb_mesolve_dense_workspace_size(n, K, 1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for b in range(nplain):
            p1.H = H_d[b].data_ptr()
            o1 = _lib.Outputs(states=states[b].data_ptr(), expects=expects[b].data_ptr(),
                              infos=infos[b].data_ptr(), status=status[b].data_ptr())
            _lib.check(lib.dqb_mesolve_dense(p1, opts, o1, ws.data_ptr(), ws1, stream.cuda_stream),
                       'plain')
        e1.record(stream)
        torch.cuda.synchronize()
        plain_s = e0.elapsed_time(e1) / 1e3
        lat = plain_s / nplain
        plain = {'value': nplain / plain_s, 'unit': 'solves/s',
                 'what': 'same kernel, one instance per launch, launches back to back',
                 'p50_latency_ms': 1e3 * lat, 'batched_over_plain': value / (world * nplain / plain_s)}

    if dist is not None:
        dist.barrier(device_ids=[local])
        dist.destroy_process_group()
    if rank != 0:
        return

    peaks, which = _peaks()
    peak = peaks.get('bf16_tflops_sustained', peaks.get('bf16_tflops'))
    clocks = _clock_summary(clk_path)
    per_inst_ms = None
    line = {
        'metric': METRIC, 'value': value, 'unit': 'solves/s', 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': mean_kernel_ms,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'c64',
        'data': 'synthetic (seeded numpy generator; no dataset)',
        'config': {'workload': WORKLOAD, 'batch_per_gpu': B, 'n': n, 'n_jumps': K,
                   'n_tsave': nt, 'method': 'Tsit5', 'rtol': 1e-6, 'atol': 1e-8,
                   'l2': 'flushed between iterations (256 MiB write); inputs+outputs > L2',
                   'parallelism': f'instances sharded over {world} GPU(s), no collective',
                   'avg_rk_steps': float(nsteps.mean())},
        'e2e': ({'value': e2e_value, 'unit': 'solves/s', 'h2d_bytes_per_step': int(h2d),
                 'd2h_bytes_per_step': int(d2h)} if e2e_value else None),
        'gpu_launches': args.steps,
        'roofline': {'bound': 'tensor', 'achieved': achieved_tflops, 'peak': peak,
                     'unit': 'TFLOP/s', 'frac': achieved_tflops / peak,
                     'peak_source': f'bf16_tflops_sustained ({which})',
                     'traffic': None,
                     'algorithmic_flops_per_launch': flops_per_solve_batch,
                     'note': 'mesolve_small_kernel<64> runs its products on the FP32 '
                             'CUDA-core pipe; FP32 SIMT nominal peak is 148 SMs x 128 FMA '
                             'x 2 x clock'},
        'clocks': clocks,
        'plain_path': plain,
        'latency_ms': {'per_batch': mean_kernel_ms, 'p50': per_inst_ms, 'p99': per_inst_ms},
    }
    if not args.no_cpu_baseline:
        line['cpu_baseline'] = cpu_baseline(sample=args.cpu_sample)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--batch', type=int, default=4096)
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--tend', type=float, default=10.0, help='end time (10 in the workload; '
                    'shorter only for profiling captures)')
    ap.add_argument('--e2e-steps', type=int, default=1)
    ap.add_argument('--cpu-sample', type=int, default=3)
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-plain', action='store_true')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    else:
        run_b200(args)


if __name__ == '__main__':
    main()
