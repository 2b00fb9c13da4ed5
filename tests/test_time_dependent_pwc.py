"""Piecewise-constant Hamiltonians (``dq.pwc``, ``dynamiqs/time_qarray.py:53-120,572-640``).

CPU: the split-at-discontinuities driver, run with the oracle as the constant-operator
solver, against the exact solution (matrix exponential of the Lindbladian on each constant
piece); the piece plan's save bookkeeping; the reference's PWC semantics (value c_k on
[t_k, t_{k+1}), 0 outside).  GPU: the same problem through ``dq.mesolve`` on the kernels."""

from types import SimpleNamespace

import numpy as np
import pytest
from scipy.linalg import expm

import dynamiqs_b200 as dq
from dynamiqs_b200 import operators as ops
from dynamiqs_b200.mesolve import _mesolve_piecewise
from dynamiqs_b200.time_qarray import as_summed, piecewise_plan
from oracle.mesolve import mesolve as oracle_mesolve

N = 5
TIMES = [0.3, 0.8, 1.5, 2.2]
VALUES = [1.0, -0.5, 2.0]
TSAVE = np.linspace(0.0, 3.0, 13)  # 1.5 is both a save time and a discontinuity


def _system():
    a = ops.destroy(N, layout='dense')
    H0 = 0.7 * (ops.dag(a) @ a)
    drive = a + ops.dag(a)
    H = H0 + dq.pwc(TIMES, VALUES, drive)
    L = [np.float32(np.sqrt(0.2)) * a]
    rho0 = ops.fock(N, 0)
    return H, H0, drive, L, rho0, [ops.dag(a) @ a]


def _lindbladian(H, Ls):
    n = H.shape[0]
    I = np.eye(n)
    # column-stacking vec: vec(A X B) = (B^T kron A) vec(X)
    out = -1j * (np.kron(I, H) - np.kron(H.T, I))
    for L in Ls:
        LdL = L.conj().T @ L
        out += np.kron(L.conj(), L) - 0.5 * (np.kron(I, LdL) + np.kron(LdL.T, I))
    return out


def _exact(H0, drive, Ls, rho0, tsave, values=VALUES):
    psi = np.asarray(rho0, complex).reshape(-1)
    rho = np.outer(psi, psi.conj())
    Ls = [np.asarray(L, complex) for L in Ls]
    edges = [0.0] + [t for t in TIMES if 0.0 < t < tsave[-1]] + [tsave[-1]]
    out, t, vec = [], 0.0, rho.reshape(-1, order='F')
    for a, b in zip(edges[:-1], edges[1:]):
        k = np.searchsorted(TIMES, 0.5 * (a + b), side='right') - 1
        c = values[k] if 0 <= k < len(values) else 0.0
        Lv = _lindbladian(np.asarray(H0, complex) + c * np.asarray(drive, complex), Ls)
        for ts in tsave:
            if (a < ts <= b) or (a == ts == 0.0):
                out.append((expm(Lv * (ts - a)) @ vec).reshape(N, N, order='F'))
        vec = expm(Lv * (b - a)) @ vec
    return np.stack(out)


def _oracle_solve(H, Ls, rho0, ts, *, exp_ops, method, gradient, options):
    r = oracle_mesolve(np.asarray(H), [np.asarray(L) for L in Ls], np.asarray(rho0), ts,
                       exp_ops=exp_ops, method=type(method).__name__, rtol=method.rtol,
                       atol=method.atol)
    return SimpleNamespace(states=r.states, expects=r.expects,
                           infos=SimpleNamespace(nsteps=np.array(r.nsteps),
                                                 naccepted=np.array(r.naccepted),
                                                 nrejected=np.array(r.nrejected)))


def test_pwc_semantics():
    P = dq.pwc(TIMES, VALUES, np.eye(2))
    assert P.prefactor(0.0) == 0.0 and P.prefactor(0.3) == 1.0 and P.prefactor(0.79) == 1.0
    assert P.prefactor(0.8) == -0.5 and P.prefactor(2.2) == 0.0 and P.prefactor(5.0) == 0.0
    with pytest.raises(ValueError, match='sorted'):
        dq.pwc([1.0, 0.0], [1.0], np.eye(2))
    with pytest.raises(ValueError, match='values'):
        dq.pwc([0.0, 1.0], [1.0, 2.0], np.eye(2))


def test_piece_plan_keeps_every_save_once():
    H, *_ = _system()
    plan = piecewise_plan(as_summed(H), TSAVE, 0.0)
    kept = np.concatenate([ts[keep] for _a, _b, _H, ts, keep in plan])
    assert np.array_equal(kept, TSAVE)
    edges = [(a, b) for a, b, *_ in plan]
    assert edges[0][0] == 0.0 and edges[-1][1] == 3.0
    assert [b for _a, b in edges[:-1]] == TIMES  # pieces end on every discontinuity in range
    for a, b, _H, ts, _keep in plan:
        assert ts[0] == a and ts[-1] == b


def test_piecewise_driver_with_oracle_matches_exact():
    H, H0, drive, L, rho0, E = _system()
    m = dq.Tsit5(rtol=1e-9, atol=1e-11)
    r = _mesolve_piecewise(H, L, rho0, TSAVE, exp_ops=E, method=m, gradient=None,
                           options=dq.Options(), solve=_oracle_solve)
    ref = _exact(H0, drive, L, rho0, TSAVE)
    assert r.states.shape == (len(TSAVE), N, N)
    err = np.linalg.norm(r.states - ref, axis=(-2, -1)) / np.linalg.norm(ref, axis=(-2, -1))
    assert err.max() < 1e-7
    n_ref = np.real(np.einsum('ij,tji->t', np.asarray(E[0]), ref))
    assert np.abs(r.expects[0] - n_ref).max() < 1e-7
    assert int(r.infos.nsteps) > 0


def test_piecewise_rejects_t0_after_first_save():
    """Pieces start at t0: a t0 after tsave[0] would drop save points silently, so it is
    an error."""
    H, H0, drive, L, rho0, E = _system()
    with pytest.raises(ValueError, match='must not be after the first save time'):
        _mesolve_piecewise(H, L, rho0, TSAVE, exp_ops=E, method=dq.Tsit5(), gradient=None,
                           options=dq.Options(t0=float(TSAVE[1])), solve=_oracle_solve)


@pytest.mark.gpu
def test_pwc_mesolve_on_gpu_matches_exact(cuda_device):
    H, H0, drive, L, rho0, E = _system()
    m = dq.Tsit5(rtol=1e-6, atol=1e-8)
    res = dq.mesolve(H, L, rho0, TSAVE, exp_ops=E, method=m)
    ref = _exact(H0, drive, L, rho0, TSAVE)
    got = res.states.cpu().numpy()
    err = np.linalg.norm(got - ref, axis=(-2, -1)) / np.linalg.norm(ref, axis=(-2, -1))
    assert err.max() < 1e-5
    n_ref = np.real(np.einsum('ij,tji->t', np.asarray(E[0]), ref))
    assert np.abs(res.expects.cpu().numpy()[0] - n_ref).max() < 1e-5
    # the controller clips its steps at the discontinuities as the reference's jump_ts
    # does: the oracle with the same handling takes the same steps
    o = oracle_mesolve(as_summed(H), L, rho0, TSAVE, rtol=m.rtol, atol=m.atol,
                       jump_ts=as_summed(H).discontinuity_ts)
    assert (int(res.infos.nsteps), int(res.infos.nrejected)) == (o.nsteps, o.nrejected)


VALUES2 = [[1.0, -0.5, 2.0], [0.2, 0.7, -1.0]]


def test_batched_pwc_values_with_oracle():
    """values of shape (2, N): the result has H's batch dimension first, and each item is
    the unbatched solve with that row of values."""
    a = ops.destroy(N, layout='dense')
    H0 = 0.7 * (ops.dag(a) @ a)
    H = H0 + dq.pwc(TIMES, VALUES2, a + ops.dag(a))
    L = [np.float32(np.sqrt(0.2)) * a]
    m = dq.Tsit5(rtol=1e-9, atol=1e-11)
    r = _mesolve_piecewise(H, L, ops.fock(N, 0), TSAVE, exp_ops=None, method=m, gradient=None,
                           options=dq.Options(), solve=_oracle_solve)
    assert r.states.shape == (2, len(TSAVE), N, N) and r.infos.nsteps.shape == (2,)
    for i, vals in enumerate(VALUES2):
        ref = _exact(H0, a + ops.dag(a), L, ops.fock(N, 0), TSAVE, values=vals)
        err = np.linalg.norm(r.states[i] - ref, axis=(-2, -1)) / np.linalg.norm(ref, axis=(-2, -1))
        assert err.max() < 1e-7


@pytest.mark.gpu
def test_batched_pwc_values_and_rho0_on_gpu(cuda_device):
    a = ops.destroy(N, layout='dense')
    H0 = 0.7 * (ops.dag(a) @ a)
    drive = a + ops.dag(a)
    H = H0 + dq.pwc(TIMES, VALUES2, drive)
    L = [np.float32(np.sqrt(0.2)) * a]
    rho0 = np.stack([ops.fock(N, 0), ops.fock(N, 1)])
    res = dq.mesolve(H, L, rho0, TSAVE, method=dq.Tsit5(rtol=1e-6, atol=1e-8))
    got = res.states.cpu().numpy()
    assert got.shape == (2, 2, len(TSAVE), N, N)
    for i, vals in enumerate(VALUES2):
        for j in range(2):
            ref = _exact(H0, drive, L, rho0[j], TSAVE, values=vals)
            err = np.linalg.norm(got[i, j] - ref, axis=(-2, -1)) / np.linalg.norm(ref, axis=(-2, -1))
            assert err.max() < 1e-5


def test_piece_plan_edge_cases():
    """Discontinuities outside the solve interval or repeated across terms add no piece; a
    start time before tsave[0] saves nothing at the start; a PWC-only H is zero outside its
    times."""
    P1 = dq.pwc([-1.0, 0.5, 9.0], [1.0, 2.0], np.eye(2))
    P2 = dq.pwc([0.5, 1.0], [3.0], np.eye(2))
    H = np.zeros((2, 2)) + P1 + P2
    ts = np.array([0.2, 0.5, 1.5])
    plan = piecewise_plan(as_summed(H), ts, 0.0)
    assert [(a, b) for a, b, *_ in plan] == [(0.0, 0.5), (0.5, 1.0), (1.0, 1.5)]
    kept = np.concatenate([t[k] for *_, t, k in plan])
    assert np.array_equal(kept, ts)
    assert plan[0][3][0] == 0.0 and 0 not in plan[0][4]  # t0 = 0 is not a save time
    assert np.allclose(plan[0][2], np.eye(2)) and np.allclose(plan[1][2], 5 * np.eye(2))
    assert np.allclose(plan[2][2], 2 * np.eye(2))
    only = dq.pwc([1.0, 2.0], [4.0], np.eye(2))
    assert np.allclose(as_summed(only)(0.5), 0) and np.allclose(as_summed(only)(1.5), 4 * np.eye(2))


def test_oracle_jump_ts_matches_exact():
    """The oracle's discontinuity handling (steps clipped just before each PWC time, the
    next one restarted on it with a fresh first stage) against the exact solution; with
    ``jump_ts`` no step straddles a jump, so the error is that of the tolerances."""
    H, H0, drive, L, rho0, E = _system()
    Hs = as_summed(H)
    r = oracle_mesolve(Hs, L, rho0, TSAVE, exp_ops=E, rtol=1e-9, atol=1e-11,
                       jump_ts=Hs.discontinuity_ts)
    ref = _exact(H0, drive, L, rho0, TSAVE)
    err = np.linalg.norm(r.states - ref, axis=(-2, -1)) / np.linalg.norm(ref, axis=(-2, -1))
    assert err.max() < 1e-7
    starts = [t for (t, _h, _e) in r.errors]
    for J in TIMES:
        assert any(t == J for t in starts)  # a step starts exactly on each discontinuity


def test_wave_prefactor_semantics():
    w = dq.Wave(2.0, 0.3, 1.5 - 0.5j, t_center=1.0, sigma=0.4, t_start=0.2, t_end=2.0)
    t = 1.3
    ref = (1.5 - 0.5j) * np.cos(2.0 * t + 0.3) * np.exp(-0.5 * ((t - 1.0) / 0.4) ** 2)
    assert abs(w(t) - ref) < 1e-15
    assert w(0.1) == 0.0 and w(2.0) == 0.0 and w(0.2) != 0.0
    M = dq.modulated(w, np.eye(2), discontinuity_ts=[0.7])
    assert list(M.discontinuity_ts) == [0.2, 0.7, 2.0]
    with pytest.raises(NotImplementedError, match='Wave'):
        dq.modulated(lambda t: np.cos(t), np.eye(2))



def test_dia_terms_stay_sparse_in_pieces():
    """A piecewise-constant H whose every term is a SparseDIA operator gives SparseDIA
    pieces (the sum of the terms' diagonals), so each piece's solve runs on the DIA path;
    their dense form equals the dense evaluation of H at the piece's midpoint."""
    from dynamiqs_b200.qarrays import SparseDIA

    a = ops.destroy(6, layout='dia')
    H = (a.dag() @ a) * np.float32(0.5) + dq.pwc([0.0, 1.0, 2.0], [0.3, -0.7], a + a.dag())
    Hs = as_summed(H)
    assert Hs.is_dia
    plan = piecewise_plan(Hs, np.linspace(0.0, 2.0, 5), 0.0)
    assert len(plan) == 2
    for (a_, b_, Hp, _, _) in plan:
        assert isinstance(Hp, SparseDIA)
        np.testing.assert_allclose(Hp.to_dense(), Hs(0.5 * (a_ + b_)), rtol=1e-6, atol=1e-6)
    dense = as_summed(np.asarray((a.dag() @ a).to_dense()) + dq.pwc([0.0, 1.0], [1.0], a))
    assert not dense.is_dia


def test_dia_td_routing_and_union_offsets():
    """A time-dependent H whose every term is sparse-DIA (and DIA jump operators) goes to
    the DIA stepper in one launch: its terms are laid out on the union of their offsets,
    each term's diagonals at their own offsets and zeros elsewhere; dense jump operators or
    more than four terms do not qualify."""
    from dynamiqs_b200.mesolve import _on_offsets, _td_on_dia, _td_union_offsets

    a = ops.destroy(5, layout='dia')
    n = a.dag() @ a
    x = a + a.dag()
    H = n * np.float32(0.5) + dq.pwc([0.0, 1.0], [1.0], x) + dq.modulated(dq.Wave(1.0), a @ a)
    Hs = as_summed(H)
    assert _td_union_offsets(Hs) == (-1, 0, 1, 2)
    L = [a * np.float32(0.3)]
    opts = dq.Options()
    assert _td_on_dia(Hs, L, opts)
    assert not _td_on_dia(Hs, [x.to_dense() for x in L], opts)
    five = H + dq.pwc([0.0, 1.0], [1.0], x) + dq.pwc([0.0, 1.0], [1.0], x)
    assert not _td_on_dia(as_summed(five + dq.pwc([0.0, 1.0], [1.0], x)), L, opts)
    offs = (-1, 0, 1, 2)
    laid = _on_offsets(a @ a, offs)
    assert laid.shape == (4, 5)
    assert np.array_equal(laid[3], (a @ a).diags[0]) and not laid[:3].any()
    dense = sum(np.diag(laid[q, max(k, 0):5 + min(k, 0)], k) for q, k in enumerate(offs))
    np.testing.assert_array_equal(dense, (a @ a).to_dense())
