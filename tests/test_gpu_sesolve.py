"""GPU parity of ``sesolve`` (the Schroedinger equation on the same Runge-Kutta engine,
``dqb_sesolve_dense``) against the oracle (``oracle.mesolve.sesolve``, complex128) and
the step counts the reference prints for its sesolve examples.  Bars: single right-hand
sides 2e-6 relative; solves 1e-5 relative on every saved ket and on expectation values."""

import numpy as np
import pytest
import torch

import dynamiqs_b200 as dq
from dynamiqs_b200 import _lib
from dynamiqs_b200 import operators as ops
from oracle.mesolve import sesolve as oracle_sesolve
from tests.systems import GOLDEN

pytestmark = pytest.mark.gpu


def _rel(x, ref):
    x, ref = np.asarray(x), np.asarray(ref)
    return np.linalg.norm(x - ref, axis=(-2, -1)) / np.linalg.norm(ref, axis=(-2, -1))


def _rand_h(n, seed):
    rng = np.random.default_rng(seed)
    X = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))) / np.sqrt(2 * n)
    return (0.5 * (X + X.conj().T)).astype(np.complex64)


def _rand_ket(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 1)) + 1j * rng.normal(size=(n, 1))
    return (v / np.linalg.norm(v)).astype(np.complex64)


@pytest.mark.parametrize('n', [2, 17, 32, 64, 100, 128])
def test_rhs_matches_numpy(cuda_device, n):
    B = 3
    Hs = np.stack([_rand_h(n, n + b) for b in range(B)])
    psi = np.stack([_rand_ket(n, 7 * n + b)[:, 0] for b in range(B)])
    H_d = torch.from_numpy(Hs).cuda()
    p_d = torch.from_numpy(psi).cuda()
    out = torch.empty_like(p_d)
    prob = _lib.DenseProblem(n=n, n_jumps=0, batch=B, H=H_d.data_ptr(), rho0=p_d.data_ptr(),
                             n_tsave=1, tsave=1)
    _lib.check(_lib.load().dqb_schrodinger_rhs_dense(prob, p_d.data_ptr(), out.data_ptr(),
                                                     torch.cuda.current_stream().cuda_stream), 'rhs')
    ref = -1j * np.einsum('bij,bj->bi', Hs.astype(complex), psi.astype(complex))
    err = np.linalg.norm(out.cpu().numpy() - ref, axis=-1) / np.linalg.norm(ref, axis=-1)
    assert err.max() < 2e-6


def test_workflow_dopri5_counts(cuda_device):
    """docs/documentation/basics/workflow.md: Dopri5(rtol=1e-6, atol=1e-8), 56 steps
    (48 accepted, 8 rejected)."""
    g = GOLDEN['workflow_dopri5_sesolve']
    H = np.float32(0.3) * ops.sigmaz(layout='dense') + 1.0 * ops.sigmax(layout='dense')
    res = dq.sesolve(H, ops.fock(2, 0), np.linspace(0.0, 10.0, 101),
                     exp_ops=[ops.sigmaz(layout='dense')], method=dq.Dopri5(rtol=1e-6, atol=1e-8))
    i = res.infos
    assert (int(i.nsteps), int(i.naccepted), int(i.nrejected)) == (g['nsteps'], g['naccepted'],
                                                                   g['nrejected'])
    assert res.states.shape == (101, 2, 1) and res.expects.shape == (1, 101)
    # Rabi oscillation of <sigma_z>: 1 - 2 Omega^2/W^2 sin^2(W t), W = sqrt(delta^2 + Omega^2)
    t = np.linspace(0.0, 10.0, 101)
    W = np.sqrt(0.3 ** 2 + 1.0)
    np.testing.assert_allclose(res.expects[0].real.cpu().numpy(),
                               1 - 2 / W ** 2 * np.sin(W * t) ** 2, atol=1e-5)


def test_docstring_counts(cuda_device):
    """dynamiqs/integrators/apis/sesolve.py docstring: 11 steps (11 accepted, 0 rejected)."""
    g = GOLDEN['sesolve_docstring']
    a = ops.destroy(16, layout='dense')
    res = dq.sesolve(ops.dag(a) @ a, ops.coherent(16, 1.0), np.linspace(0, 1.0, 11))
    i = res.infos
    assert (int(i.nsteps), int(i.naccepted), int(i.nrejected)) == (g['nsteps'], g['naccepted'],
                                                                   g['nrejected'])


@pytest.mark.parametrize('n', [5, 40, 100])
@pytest.mark.parametrize('method', ['Tsit5', 'Dopri5'])
def test_solve_matches_oracle(cuda_device, n, method):
    H = _rand_h(n, n)
    psi0 = _rand_ket(n, 3 * n)
    E = [_rand_h(n, 5 * n)]
    ts = np.linspace(0.0, 4.0, 9)
    m = dq.Tsit5() if method == 'Tsit5' else dq.Dopri5()
    res = dq.sesolve(H, psi0, ts, exp_ops=E, method=m)
    r = oracle_sesolve(H, psi0, ts, method=method, save_fn=lambda y: y)
    states = np.stack(r.ysave)
    assert _rel(res.states.cpu().numpy(), states).max() < 1e-5
    ex = np.array([[(s.conj().T @ E[0].astype(complex) @ s)[0, 0] for s in states]])
    got = res.expects.cpu().numpy()
    assert (np.abs(got - ex) / np.maximum(np.abs(ex), 1.0)).max() < 1e-5
    assert abs(int(res.infos.nsteps) - r.nsteps) <= 1


def test_batching_and_options(cuda_device):
    n = 12
    Hs = np.stack([_rand_h(n, s) for s in range(3)])
    psis = np.stack([_rand_ket(n, 10 + s) for s in range(2)])
    ts = np.linspace(0, 2, 5)
    res = dq.sesolve(Hs, psis, ts)
    assert res.states.shape == (3, 2, 5, n, 1)
    for i in range(3):
        for j in range(2):
            one = dq.sesolve(Hs[i], psis[j], ts)
            np.testing.assert_array_equal(res.states[i, j].cpu().numpy(), one.states.cpu().numpy())
    flat = dq.sesolve(Hs[:2], psis, ts, options=dq.Options(cartesian_batching=False))
    assert flat.states.shape == (2, 5, n, 1)
    last = dq.sesolve(Hs[0], psis[0], ts, options=dq.Options(save_states=False))
    assert last.states.shape == (1, n, 1)
    assert _rel(last.final_state.cpu().numpy(), res.states[0, 0, -1].cpu().numpy()) < 1e-6
    shifted = dq.sesolve(Hs[0], psis[0], ts[2:], options=dq.Options(t0=0.0))
    r = oracle_sesolve(Hs[0], psis[0], ts[2:], t0=0.0, save_fn=lambda y: y)
    assert _rel(shifted.states.cpu().numpy(), np.stack(r.ysave)).max() < 1e-5
    with pytest.raises(RuntimeError, match='maximum number of method steps'):
        dq.sesolve(Hs[0], psis[0], ts, method=dq.Tsit5(max_steps=2))


def _banded_h(n, seed, offsets=(1, 7)):
    """A hermitian banded H (main diagonal and +-offsets), complex64."""
    rng = np.random.default_rng(seed)
    H = np.diag(rng.normal(size=n)).astype(complex)
    for k in offsets:
        d = (rng.normal(size=n - k) + 1j * rng.normal(size=n - k)) / 2
        H += np.diag(d, k) + np.diag(d.conj(), -k)
    return H.astype(np.complex64)


@pytest.mark.parametrize('n', [129, 200, 333])
@pytest.mark.parametrize('method', ['Tsit5', 'Dopri5'])
def test_large_dense_solve_matches_oracle(cuda_device, n, method):
    """n > 128: the batched large-problem stepper with a dense H
    (``dqb_sesolve_dense_large``; odd n takes the product's scalar loads), every saved ket
    and the expectation values against the complex128 oracle at 1e-5, the norm check, and
    the step count."""
    H = _rand_h(n, n)
    psi0 = _rand_ket(n, 3 * n)
    E = [_rand_h(n, 5 * n)]
    ts = np.linspace(0.0, 3.0, 7)
    m = dq.Tsit5() if method == 'Tsit5' else dq.Dopri5()
    res = dq.sesolve(H, psi0, ts, exp_ops=E, method=m)
    r = oracle_sesolve(H, psi0, ts, method=method, save_fn=lambda y: y)
    states = np.stack(r.ysave)
    assert res.states.shape == (7, n, 1)
    assert _rel(res.states.cpu().numpy(), states).max() < 1e-5
    ex = np.array([[(s.conj().T @ E[0].astype(complex) @ s)[0, 0] for s in states]])
    got = res.expects.cpu().numpy()
    assert (np.abs(got - ex) / np.maximum(np.abs(ex), 1.0)).max() < 1e-5
    assert abs(int(res.infos.nsteps) - r.nsteps) <= 1
    # the norm check follows the oracle's (the method's own drift at this tolerance)
    ref_norm = (np.abs(states) ** 2).sum(axis=(-2, -1))
    assert np.abs(res.checks['norm'].cpu().numpy() - ref_norm).max() < 2e-5


@pytest.mark.parametrize('n', [150, 1024])
def test_large_dia_solve_matches_oracle_and_dense(cuda_device, n):
    """H kept in sparse-DIA storage (``dqb_sesolve_dia``): against the oracle (dense
    complex128 H) at 1e-5 on every saved ket and on the expectation values, and against the
    dense large-problem path on the same H."""
    from dynamiqs_b200.qarrays import SparseDIA

    Hd = _banded_h(n, n)
    H = SparseDIA.from_dense(Hd)
    assert set(H.offsets) == {-7, -1, 0, 1, 7}
    psi0 = _rand_ket(n, 2 * n)
    E = [np.diag(np.arange(n)).astype(np.complex64)]
    ts = np.linspace(0.0, 2.0, 5)
    res = dq.sesolve(H, psi0, ts, exp_ops=E)
    r = oracle_sesolve(Hd, psi0, ts, save_fn=lambda y: y)
    states = np.stack(r.ysave)
    assert _rel(res.states.cpu().numpy(), states).max() < 1e-5
    ex = np.array([[(s.conj().T @ E[0].astype(complex) @ s)[0, 0] for s in states]])
    got = res.expects.cpu().numpy()
    assert (np.abs(got - ex) / np.maximum(np.abs(ex), 1.0)).max() < 1e-5
    assert abs(int(res.infos.nsteps) - r.nsteps) <= 1
    assert res.checks['norm'].shape == (5,)
    ref_norm = (np.abs(states) ** 2).sum(axis=(-2, -1))
    assert np.abs(res.checks['norm'].cpu().numpy() - ref_norm).max() < 2e-5
    dense = dq.sesolve(Hd, psi0, ts, exp_ops=E)
    assert _rel(res.states.cpu().numpy(), dense.states.cpu().numpy()).max() < 1e-5


def test_large_batching_and_options(cuda_device):
    """Cartesian and flat batching on the large-problem paths: each instance bitwise equal
    to its own solve; save_states=False keeps the final ket; t0; max_steps."""
    from dynamiqs_b200.qarrays import SparseDIA

    n = 160
    Hs = np.stack([_banded_h(n, s) for s in range(3)])
    psis = np.stack([_rand_ket(n, 10 + s) for s in range(2)])
    ts = np.linspace(0, 1, 4)
    for H in (Hs, SparseDIA.from_dense(Hs)):
        res = dq.sesolve(H, psis, ts)
        assert res.states.shape == (3, 2, 4, n, 1)
        for i in range(3):
            for j in range(2):
                Hi = Hs[i] if isinstance(H, np.ndarray) else SparseDIA(H.offsets, H.diags[i])
                one = dq.sesolve(Hi, psis[j], ts)
                np.testing.assert_array_equal(res.states[i, j].cpu().numpy(), one.states.cpu().numpy())
        flat = dq.sesolve(H, psis[:1], ts, options=dq.Options(cartesian_batching=False))
        assert flat.states.shape == (3, 4, n, 1)
        H0 = Hs[0] if isinstance(H, np.ndarray) else SparseDIA(H.offsets, H.diags[0])
        last = dq.sesolve(H0, psis[0], ts, options=dq.Options(save_states=False))
        assert last.states.shape == (1, n, 1)
        assert _rel(last.final_state.cpu().numpy(), res.states[0, 0, -1].cpu().numpy()) < 1e-6
    shifted = dq.sesolve(Hs[0], psis[0], ts[2:], options=dq.Options(t0=0.0))
    r = oracle_sesolve(Hs[0], psis[0], ts[2:], t0=0.0, save_fn=lambda y: y)
    assert _rel(shifted.states.cpu().numpy(), np.stack(r.ysave)).max() < 1e-5
    with pytest.raises(RuntimeError, match='maximum number of method steps'):
        dq.sesolve(Hs[0], psis[0], ts, method=dq.Tsit5(max_steps=2))


# ---- time-dependent H (dqb_sesolve_dense_large_td, dqb_sesolve_dia_td) ------------------

def _oracle_td(Hs, psi0, ts, method='Tsit5', rtol=1e-6, atol=1e-8):
    """The Schroedinger equation with H(t) = Hs(t) in complex128 through the oracle's RK
    engine, with the same discontinuity times handed to its controller: the saved kets and
    the step-count slack of tests/parity.py (one step, or two when one of the oracle's
    accept / reject decisions was borderline: a scaled error within 0.1 of 1)."""
    from oracle.rk import solve

    out = solve(lambda t, y: -1j * (np.asarray(Hs(t), dtype=complex) @ y),
                np.asarray(psi0, dtype=complex), ts, method=method, rtol=rtol, atol=atol,
                save_fn=lambda y: y, jump_ts=Hs.discontinuity_ts)
    borderline = any(abs(e - 1.0) < 0.1 for (_, _, e) in out.errors)
    return np.stack(out.ysave), out.nsteps, (max(2, int(0.01 * out.nsteps)) if borderline else 1)


@pytest.mark.parametrize('method', ['Tsit5', 'Dopri5'])
def test_td_dense_sesolve_matches_oracle(cuda_device, method):
    """A PWC drive and a Gaussian Wave pulse (n = 40, dense): one launch of the
    large-problem stepper, against the oracle with the same jump_ts at 1e-5, step counts
    within one."""
    from dynamiqs_b200.time_qarray import as_summed

    a = ops.destroy(40, layout='dense')
    num, x = ops.dag(a) @ a, a + ops.dag(a)
    pulse = dq.Wave(1.4, 0.0, 0.6 - 0.2j, t_center=1.0, sigma=0.35, t_start=0.2, t_end=1.9)
    H = 0.5 * num + dq.pwc([0.1, 0.5, 1.3, 2.0], [0.7, -0.2, 0.4], x) + dq.modulated(pulse, 1j * (ops.dag(a) - a))
    ts = np.linspace(0.0, 2.2, 12)
    m = dq.Tsit5(rtol=1e-6, atol=1e-8) if method == 'Tsit5' else dq.Dopri5(rtol=1e-6, atol=1e-8)
    psi0 = ops.fock(40, 0)
    res = dq.sesolve(H, psi0, ts, exp_ops=[num], method=m)
    ref, nsteps, slack = _oracle_td(as_summed(H), psi0, ts, method=method)
    assert _rel(res.states.cpu().numpy(), ref).max() < 1e-5
    ex = np.array([[(s.conj().T @ num.astype(complex) @ s)[0, 0] for s in ref]])
    assert (np.abs(res.expects.cpu().numpy() - ex) / np.maximum(np.abs(ex), 1.0)).max() < 1e-5
    assert abs(int(res.infos.nsteps) - nsteps) <= slack


def test_td_dia_sesolve_and_batched_values(cuda_device):
    """H in DIA storage (n = 300) with batched PWC values (2 sets) and two initial kets:
    one launch of 4 instances, each against the oracle.  atol = 1e-6: the random kets'
    entries are ~0.06, so at atol = 1e-8 the FP32 rounding of the stage values is ~5 % of
    the error scale and moves the first steps' sizes (the complex64 error estimate of the
    first 0.007-long step reads 8.6e-4 where the complex128 one reads 2e-4), which changes
    the step count by a few while the states still agree at 5e-6."""
    from dynamiqs_b200.qarrays import SparseDIA
    from dynamiqs_b200.time_qarray import as_summed

    Hd = _banded_h(300, 3)
    H0 = SparseDIA.from_dense(Hd)
    a = ops.destroy(300, layout='dia')
    x = a + a.dag()
    vals = np.array([[0.5, -0.3, 0.8], [0.1, 0.6, -0.4]])
    times = [0.2, 0.6, 1.0, 1.5]
    H = H0 + dq.pwc(times, vals, x)
    psis = np.stack([_rand_ket(300, 11), _rand_ket(300, 12)])
    ts = np.linspace(0.0, 1.8, 7)
    m = dq.Tsit5(rtol=1e-6, atol=1e-6)
    res = dq.sesolve(H, psis, ts, method=m)
    assert res.states.shape == (2, 2, 7, 300, 1)
    for i in range(2):
        Hi = as_summed(H0 + dq.pwc(times, vals[i], x))
        for j in range(2):
            ref, nsteps, slack = _oracle_td(Hi, psis[j], ts, atol=1e-6)
            assert _rel(res.states[i, j].cpu().numpy(), ref).max() < 1e-5
            assert abs(int(res.infos.nsteps[i, j]) - nsteps) <= slack, (i, j, nsteps, slack)
