"""GPU parity of the dense persistent kernel (n <= 64) against the oracle, through the
C ABI (``dqb_lindblad_rhs_dense``, ``dqb_mesolve_dense``) and the public ``mesolve``.

Solves are held to the bar of tests/parity.py (1e-5 relative Frobenius error on every
saved state and 1e-5 on expectation values against the oracle's trajectory; on stiff
instances whose step sequences part at a borderline accept/reject decision, the
accuracy bar against a tight FP64 solution).  Single right-hand sides are compared at
2e-6 relative (FP32 products of length <= 64)."""

import numpy as np
import pytest
import torch

import dynamiqs_b200 as dq
from dynamiqs_b200 import _lib
from dynamiqs_b200 import operators as ops
from dynamiqs_b200 import workloads
from oracle import lindblad as lb
from oracle.mesolve import mesolve as oracle_mesolve
from tests.parity import assert_solve_parity
from tests.systems import ocavity, random_problem, readme_oscillator

pytestmark = pytest.mark.gpu

STATE_RTOL = 1e-5
EXPECT_TOL = 1e-5


def rel_frob(x, ref):
    x, ref = np.asarray(x), np.asarray(ref)
    return np.linalg.norm(x - ref, axis=(-2, -1)) / np.maximum(np.linalg.norm(ref, axis=(-2, -1)), 1e-30)


def expect_err(x, ref):
    return np.abs(np.asarray(x) - ref) / np.maximum(np.abs(ref), 1.0)


def _dev(x, dtype=torch.complex64):
    return torch.from_numpy(np.ascontiguousarray(x)).to('cuda', dtype)


@pytest.mark.parametrize('n', [2, 7, 16, 33, 64])
@pytest.mark.parametrize('K', [0, 1, 3])
@pytest.mark.parametrize('form', [_lib.FORM_HERMITIAN, _lib.FORM_STANDARD])
def test_rhs_matches_oracle(cuda_device, n, K, form):
    if _lib.load().dqb_dense_small_max_n(K) < n:
        pytest.skip('jump count beyond shared memory at this n')
    B = 3
    rng = np.random.default_rng(n * 10 + K)
    Hs, Lsets, rhos = [], [], []
    for b in range(B):
        H, Ls, rho = random_problem(n, K, seed=int(rng.integers(1 << 30)),
                                    hermitian_rho=form == _lib.FORM_HERMITIAN)
        Hs.append(H)
        Lsets.append(np.stack(Ls) if K else np.zeros((0, n, n), np.complex64))
        rhos.append(rho)
    H_d, L_d, r_d = _dev(np.stack(Hs)), _dev(np.stack(Lsets)), _dev(np.stack(rhos))
    out = torch.empty_like(r_d)
    prob = _lib.DenseProblem(n=n, n_jumps=K, batch=B, H=H_d.data_ptr(), L=L_d.data_ptr())
    lib = _lib.load()
    rc = lib.dqb_lindblad_rhs_dense(prob, form, r_d.data_ptr(), out.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream)
    _lib.check(rc, 'rhs')
    got = out.cpu().numpy()
    for b in range(B):
        Hc = Hs[b].astype(complex)
        Lc = [L.astype(complex) for L in Lsets[b]]
        rc_ = rhos[b].astype(complex)
        ref = lb.vf_hermitian(Hc, Lc, rc_) if form == _lib.FORM_HERMITIAN else lb.vf_standard(Hc, Lc, rc_)
        assert rel_frob(got[b], ref) < 2e-6


def _compare_solve(res, H, Ls, rho0, tsave, exp_ops, method, **okw):
    """GPU result vs the oracle under the bar of tests/parity.py."""
    mname = 'Tsit5' if isinstance(method, dq.Tsit5) else 'Dopri5'
    ex = res.expects.cpu().numpy() if exp_ops else None
    return assert_solve_parity(res.states.cpu().numpy(), ex, int(res.infos.nsteps), H, Ls,
                               rho0, tsave, exp_ops, mname, method.rtol, method.atol, **okw)


@pytest.mark.parametrize('method', [dq.Tsit5(rtol=1e-6, atol=1e-8), dq.Dopri5(rtol=1e-6, atol=1e-8)],
                         ids=['tsit5', 'dopri5'])
def test_lossy_oscillator_config(cuda_device, method):
    """Plain lossy oscillator: n=16, omega=1, kappa=0.1, alpha0=1, 101 saves."""
    w = workloads.lossy_oscillator()
    res = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], exp_ops=w['exp_ops'],
                     method=method)
    assert res.states.shape == (101, 16, 16)
    assert res.expects.shape == (1, 101)
    _compare_solve(res, w['H'], w['jump_ops'], w['rho0'], w['tsave'], w['exp_ops'], method)


@pytest.mark.parametrize('layout', ['dense', 'dia'])
@pytest.mark.parametrize('opts', [dq.Options(), dq.Options(assume_hermitian=False),
                                  dq.Options(vectorized=True)], ids=['herm', 'std', 'vec'])
def test_ocavity_analytic(cuda_device, layout, opts):
    """The reference's TestMESolveAdaptive.test_correctness system and tolerances."""
    p = ocavity(layout)
    res = dq.mesolve(p['H'], p['jump_ops'], p['rho0'], p['tsave'], exp_ops=p['exp_ops'],
                     options=opts)
    errs = np.linalg.norm(res.states.cpu().numpy() - p['true_states'], axis=(-2, -1))
    assert np.all(errs <= 1e-3)
    np.testing.assert_allclose(res.expects.cpu().numpy(), p['true_expects'], rtol=1e-3, atol=1e-4)


def test_batched_kerr_subset(cuda_device):
    """Batched Kerr (n=64, two jumps) on a subset of instances, each against the oracle."""
    w = workloads.batched_kerr(batch=6, seed=7)
    res = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], exp_ops=w['exp_ops'],
                     method=w['method'])
    assert res.states.shape == (6, 51, 64, 64)
    for b in range(6):
        sub = dq.MESolveResult(None, w['method'], None, None, res.states[b], res.expects[b],
                               dq.AdaptiveStepInfos(res.infos.nsteps[b], res.infos.naccepted[b],
                                                    res.infos.nrejected[b]))
        _compare_solve(sub, w['H'][b], w['jump_ops'], w['rho0'], w['tsave'], w['exp_ops'],
                       w['method'])


def test_standard_form_non_hermitian_rho(cuda_device):
    H, Ls, rho = random_problem(12, 2, seed=11, hermitian_rho=False)
    ts = np.linspace(0, 1.5, 7)
    res = dq.mesolve(H, Ls, rho, ts, options=dq.Options(assume_hermitian=False))
    _compare_solve(res, H, Ls, rho, ts, None, dq.Tsit5(), form='standard')
    with pytest.raises(RuntimeError, match='not hermitian'):
        dq.mesolve(H, Ls, rho, ts)


def test_cartesian_batching_equals_single_solves(cuda_device):
    n = 10
    a = ops.destroy(n, layout='dense')
    Hs = np.stack([w * (ops.dag(a) @ a) for w in (0.5, 1.0, 1.5)])
    L0 = np.stack([np.float32(np.sqrt(k)) * a for k in (0.1, 0.3)])
    rho0 = np.stack([ops.coherent(n, al) for al in (0.3, 0.6)])
    ts = np.linspace(0, 2, 5)
    E = [ops.number(n, layout='dense')]
    res = dq.mesolve(Hs, [L0], rho0, ts, exp_ops=E)
    assert res.states.shape == (3, 2, 2, 5, n, n)
    assert res.expects.shape == (3, 2, 2, 1, 5)
    for i in range(3):
        for j in range(2):
            for k in range(2):
                single = dq.mesolve(Hs[i], [L0[j]], rho0[k], ts, exp_ops=E)
                np.testing.assert_array_equal(res.states[i, j, k].cpu().numpy(),
                                              single.states.cpu().numpy())
    flat = dq.mesolve(Hs[:2], [L0], rho0, ts, options=dq.Options(cartesian_batching=False))
    assert flat.states.shape == (2, 5, n, n)


def test_save_states_false_and_t0(cuda_device):
    p = readme_oscillator()
    full = dq.mesolve(p['H'], p['jump_ops'], p['rho0'], p['tsave'])
    last = dq.mesolve(p['H'], p['jump_ops'], p['rho0'], p['tsave'],
                      options=dq.Options(save_states=False))
    assert last.states.shape == (1, 16, 16)
    assert rel_frob(last.final_state.cpu().numpy(), full.final_state.cpu().numpy()) < 1e-5
    shifted = dq.mesolve(p['H'], p['jump_ops'], p['rho0'], p['tsave'][50:],
                         options=dq.Options(t0=0.0))
    r = oracle_mesolve(p['H'], p['jump_ops'], p['rho0'], p['tsave'][50:], t0=0.0)
    assert rel_frob(shifted.states.cpu().numpy(), r.states).max() < STATE_RTOL


def test_max_steps_error(cuda_device):
    p = readme_oscillator()
    with pytest.raises(RuntimeError, match='maximum number of method steps'):
        dq.mesolve(p['H'], p['jump_ops'], p['rho0'], p['tsave'], method=dq.Tsit5(max_steps=5))


def test_nonfinite_status(cuda_device):
    H, Ls, rho = random_problem(4, 1, seed=1)
    H = H.copy()
    H[0, 0] = np.nan
    with pytest.raises(RuntimeError, match='non-finite'):
        dq.mesolve(H, Ls, rho, np.linspace(0, 1, 3))


def test_capi_rejects_bad_arguments(cuda_device):
    lib = _lib.load()
    opts = _lib.OdeOptions(method=7, rtol=1e-6, atol=1e-6, safety=0.9, factormin=0.2,
                           factormax=5.0, max_steps=10)
    prob = _lib.DenseProblem(n=4, n_jumps=0, n_exp=0, n_tsave=2, batch=1)
    outs = _lib.Outputs()
    assert lib.dqb_mesolve_dense(prob, opts, outs, None, 0, None) == _lib.DQB_ERR_INVALID_ARGUMENT
    assert lib.dqb_mesolve_dense(None, opts, outs, None, 0, None) == _lib.DQB_ERR_INVALID_ARGUMENT
    assert lib.dqb_dense_small_max_n(2) == 64
    assert lib.dqb_mesolve_dense_workspace_size(64, 2, 4096) > 0


def test_start_order_changes_no_result(cuda_device):
    """With more instances than resident CTAs the host starts the stiffest first
    (start_order); every result is bitwise the one of the natural order."""
    from dynamiqs_b200.mesolve import MESolveB200Integrator, make_batch_plan

    w = workloads.batched_kerr(batch=400, n=16, seed=2)
    ts = np.linspace(0.0, 1.0, 5)
    plan = make_batch_plan(w['H'], w['jump_ops'], w['rho0'], True)
    integ = MESolveB200Integrator(ts=ts, y0=w['rho0'], method=w['method'], gradient=None,
                                  options=dq.Options(), H=w['H'], Ls=w['jump_ops'],
                                  Es=w['exp_ops'], plan=plan)
    prep = integ.prepare()
    assert prep.prob.start_order
    order = prep.bufs['start_order'].cpu().numpy()
    assert sorted(order.tolist()) == list(range(400)) and order.tolist() != list(range(400))
    a = prep.launch().result()
    sa, ia = a.states.cpu().numpy().copy(), a.infos.nsteps.cpu().numpy().copy()
    prep.prob.start_order = None
    b = prep.launch().result()
    assert np.array_equal(sa, b.states.cpu().numpy())
    assert np.array_equal(ia, b.infos.nsteps.cpu().numpy())


def test_fp64_checks_of_saved_states(cuda_device):
    """result.checks: tr(rho) at every save point (FP64 sums in the kernel) and the FP64
    hermiticity defect of every saved state, on the three solve paths."""
    w = workloads.batched_kerr(batch=3, n=20, seed=1)
    res = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], exp_ops=w['exp_ops'],
                     method=w['method'])
    tr = res.checks['trace'].cpu().numpy()
    assert tr.shape == (3, 51) and np.abs(tr - 1).max() < 1e-5
    assert res.checks['hermiticity'].shape == (3, 51)
    assert float(res.checks['hermiticity'].max()) < 1e-6
    assert res.expects.shape == (3, 1, 51)  # the trace row is not among the user's expects
    std = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'],
                     options=dq.Options(assume_hermitian=False))
    assert std.expects is None and np.abs(std.checks['trace'].cpu().numpy() - 1).max() < 1e-5
    assert float(std.checks['hermiticity'].max()) < 1e-5
