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
