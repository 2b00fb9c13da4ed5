"""Continuous-batching server: each result is the same alone (``dq.mesolve`` on that one
request) and in the mix, within the 1e-5 relative bar; requests that arrive while others
are on the GPU are launched before those finish (their work overlaps on the device)."""

import numpy as np
import pytest

import dynamiqs_b200 as dq
from dynamiqs_b200 import workloads
from dynamiqs_b200.server import MESolveServer

pytestmark = pytest.mark.gpu


def _requests(num, seed, dims=(8, 16, 32, 64, 128), weights=(0.3, 0.25, 0.2, 0.15, 0.1)):
    reqs = workloads.serving_requests(num, seed=seed, dims=dims, weights=weights)
    for r in reqs:  # short horizons keep the test quick
        r['tsave'] = np.linspace(0.0, min(r['tsave'][-1], 3.0), len(r['tsave']))
    return reqs


def _rel(x, ref):
    x, ref = np.asarray(x), np.asarray(ref)
    return float((np.linalg.norm(x - ref, axis=(-2, -1)) / np.linalg.norm(ref, axis=(-2, -1))).max())


def test_results_same_alone_and_in_the_mix(cuda_device):
    reqs = _requests(24, seed=11)
    srv = MESolveServer(n_streams=4)
    tickets = [srv.submit(r['H'], r['jump_ops'], r['rho0'], r['tsave'], exp_ops=r['exp_ops'],
                          method=r['method']) for r in reqs]
    results = [t.result(timeout=300) for t in tickets]
    srv.close()
    assert srv.stats()['solves'] == len(reqs)
    for r, res in zip(reqs, results):
        alone = dq.mesolve(r['H'], r['jump_ops'], r['rho0'], r['tsave'], exp_ops=r['exp_ops'],
                           method=r['method'])
        assert _rel(res.states.cpu().numpy(), alone.states.cpu().numpy()) < 1e-5
        e_mix, e_alone = res.expects.cpu().numpy(), alone.expects.cpu().numpy()
        assert np.max(np.abs(e_mix - e_alone) / np.maximum(np.abs(e_alone), 1.0)) < 1e-5
        assert int(res.infos.nsteps) == int(alone.infos.nsteps)


def test_late_arrivals_overlap_running_waves(cuda_device):
    first = _requests(12, seed=3, dims=(64,), weights=(1.0,))
    late = _requests(12, seed=4, dims=(16, 32), weights=(0.5, 0.5))
    srv = MESolveServer(n_streams=8)
    t1 = [srv.submit(r['H'], r['jump_ops'], r['rho0'], r['tsave'], method=r['method']) for r in first]
    t2 = [srv.submit(r['H'], r['jump_ops'], r['rho0'], r['tsave'], method=r['method']) for r in late]
    for t in t1 + t2:
        t.result(timeout=300)
    srv.close()
    # some late request was launched before the last of the first group finished
    assert min(t.t_launch for t in t2) < max(t.t_done for t in t1)
    st = srv.stats()
    assert st['errors'] == 0 and st['p99_ms'] >= st['p50_ms'] > 0


def test_budget_admission_and_errors(cuda_device):
    reqs = _requests(6, seed=5, dims=(16,), weights=(1.0,))
    tiny = MESolveServer(budget_bytes=4096, n_streams=2, staging_bytes=1 << 20)
    t = tiny.submit(reqs[0]['H'], reqs[0]['jump_ops'], reqs[0]['rho0'], reqs[0]['tsave'],
                    method=reqs[0]['method'])
    with pytest.raises(MemoryError, match='budget'):
        t.result(timeout=60)
    tiny.close()
    srv = MESolveServer(budget_bytes=1 << 30, n_streams=2, staging_bytes=1 << 24)
    tickets = [srv.submit(r['H'], r['jump_ops'], r['rho0'], r['tsave'], method=r['method'])
               for r in reqs]
    bad = srv.submit(reqs[0]['H'], reqs[0]['jump_ops'], reqs[0]['rho0'], reqs[0]['tsave'],
                     method=dq.Tsit5(max_steps=2))
    for t in tickets:
        assert t.result(timeout=120).states.shape[-1] == 16
        t.release()
    with pytest.raises(RuntimeError, match='maximum number of method steps'):
        bad.result(timeout=120)
    srv.close()
    assert srv._dev.used() == 0  # every wave and every released result gave its memory back


def test_quick_request_leaves_before_slow_one_of_its_wave(cuda_device):
    """A quick and a slow request launched in the same GEMM-path wave: the quick one is
    handed out when its own status word is written, long before the wave ends, and both
    results equal the request solved alone."""
    from dynamiqs_b200 import operators as ops

    n = 80

    def kerr(kerr_, t_end):
        H = workloads.kerr_hamiltonians(n, [0.3], [kerr_], [1.0])[0]
        a = ops.destroy(n, layout='dense')
        return dict(H=H, jump_ops=[np.float32(np.sqrt(0.1)) * a], rho0=ops.fock(n, 0),
                    tsave=np.linspace(0.0, t_end, 5), method=dq.Tsit5(rtol=1e-6, atol=1e-6))

    quick, slow = kerr(0.1, 0.05), kerr(0.5, 8.0)
    srv = MESolveServer(n_streams=2)  # one stream per class
    with srv.paused():  # submitted while paused: launched together, as one wave
        sub = [srv.submit(r['H'], r['jump_ops'], r['rho0'], r['tsave'], method=r['method'])
               for r in (quick, slow)]
    res = [t.result(timeout=600) for t in sub]
    srv.close()
    t_q, t_s = sub
    assert t_q.t_launch == t_s.t_launch  # the same wave
    assert t_s.t_done - t_q.t_done > 0.05, (t_q.t_done, t_s.t_done)
    for r, got in zip((quick, slow), res):
        alone = dq.mesolve(r['H'], r['jump_ops'], r['rho0'], r['tsave'], method=r['method'])
        assert _rel(got.states.cpu().numpy(), alone.states.cpu().numpy()) < 1e-5
        assert int(got.infos.nsteps) == int(alone.infos.nsteps)


def test_cancel_running_and_waiting_requests(cuda_device):
    """Ticket.cancel(): a waiting request leaves the queue without launching; a running
    request stops at its next check between RK steps (n <= 64 kernel and GEMM path), ends
    with CancelledError soon after, and the other request of its wave is unaffected."""
    import time
    from concurrent.futures import CancelledError

    from dynamiqs_b200 import operators as ops

    def kerr(n, kerr_, t_end):
        H = workloads.kerr_hamiltonians(n, [0.3], [kerr_], [1.0])[0]
        a = ops.destroy(n, layout='dense')
        return dict(H=H, jump_ops=[np.float32(np.sqrt(0.1)) * a], rho0=ops.fock(n, 0),
                    tsave=np.linspace(0.0, t_end, 5), method=dq.Tsit5(rtol=1e-6, atol=1e-6))

    srv = MESolveServer(n_streams=2)  # one stream per class
    for n in (64, 80):
        slow, quick = kerr(n, 0.5, 400.0), kerr(n, 0.1, 0.05)
        with srv.paused():  # slow and quick are launched together, as one wave
            ts = [srv.submit(r['H'], r['jump_ops'], r['rho0'], r['tsave'], method=r['method'])
                  for r in (slow, quick)]
        t0 = time.perf_counter()
        while ts[0].t_launch == 0.0 and time.perf_counter() - t0 < 120:
            time.sleep(0.01)
        assert ts[0].t_launch > 0.0 and ts[1].t_launch == ts[0].t_launch
        # a request that arrives now waits: the class's only stream runs the slow wave
        waiting = srv.submit(quick['H'], quick['jump_ops'], quick['rho0'], quick['tsave'],
                             method=quick['method'])
        assert waiting.cancel()
        with pytest.raises(CancelledError):
            waiting.result(timeout=1)
        assert waiting.t_launch == 0.0
        got_quick = ts[1].result(timeout=600)
        t_cancel = time.perf_counter()
        assert ts[0].cancel()
        with pytest.raises(CancelledError):
            ts[0].result(timeout=60)
        assert ts[0].t_done - t_cancel < 5.0
        assert not ts[0].cancel()  # already finished
        alone = dq.mesolve(quick['H'], quick['jump_ops'], quick['rho0'], quick['tsave'],
                           method=quick['method'])
        assert _rel(got_quick.states.cpu().numpy(), alone.states.cpu().numpy()) < 1e-5
        ts[1].release()  # (carried out when the wave ends)
    srv.close()
