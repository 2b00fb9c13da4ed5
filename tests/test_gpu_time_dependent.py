"""GPU parity of time-dependent Hamiltonians on the n <= 64 kernel (``dqb_mesolve_dense_td``:
PWC and Wave prefactors evaluated at every stage time, steps clipped at the
discontinuities as the reference's ``jump_ts`` does) against the oracle run with the same
time dependence and ``jump_ts`` (complex128), under the bar of tests/parity.py."""

import numpy as np
import pytest

import dynamiqs_b200 as dq
from dynamiqs_b200 import operators as ops
from dynamiqs_b200.time_qarray import as_summed
from tests.parity import assert_solve_parity

pytestmark = pytest.mark.gpu


def _check(H, L, rho0, ts, E, m=dq.Tsit5(rtol=1e-6, atol=1e-8), res=None, b=None):
    res = res if res is not None else dq.mesolve(H, L, rho0, ts, exp_ops=E, method=m)
    Hs = as_summed(H)
    st = res.states.cpu().numpy() if b is None else res.states[b].cpu().numpy()
    ex = None
    if E:
        ex = res.expects.cpu().numpy() if b is None else res.expects[b].cpu().numpy()
    ns = int(res.infos.nsteps if b is None else res.infos.nsteps[b])
    return assert_solve_parity(st, ex, ns, Hs, L, rho0, ts, E, type(m).__name__, m.rtol,
                               m.atol, jump_ts=Hs.discontinuity_ts)


def _osc(n):
    a = ops.destroy(n, layout='dense')
    return a, ops.dag(a) @ a, a + ops.dag(a)


def test_pwc_drive_one_launch(cuda_device):
    a, num, x = _osc(6)
    H = 0.7 * num + dq.pwc([0.3, 0.8, 1.5, 2.2], [1.0, -0.5, 2.0], x)
    ts = np.linspace(0.0, 3.0, 13)  # 1.5 is both a save time and a discontinuity
    assert _check(H, [np.float32(np.sqrt(0.2)) * a], ops.fock(6, 0), ts, [num]) == 'trajectory'


@pytest.mark.parametrize('method', ['Tsit5', 'Dopri5'])
def test_wave_drive(cuda_device, method):
    a, num, x = _osc(12)
    H = 0.5 * num + dq.modulated(dq.Wave(1.3, 0.2, 0.8), x)
    ts = np.linspace(0.0, 4.0, 21)
    m = dq.Tsit5(rtol=1e-6, atol=1e-8) if method == 'Tsit5' else dq.Dopri5(rtol=1e-6, atol=1e-8)
    assert _check(H, [np.float32(np.sqrt(0.1)) * a], ops.fock(12, 0), ts, [num], m=m) == 'trajectory'


def test_gaussian_pulse_with_support(cuda_device):
    """A Gaussian-enveloped pulse switched on at 0.5 and off at 2.5: both edges are
    discontinuities handed to the controller."""
    a, num, x = _osc(10)
    pulse = dq.Wave(2.0, 0.0, 1.5 - 0.3j, t_center=1.5, sigma=0.4, t_start=0.5, t_end=2.5)
    H = 0.2 * num + dq.modulated(pulse, x)
    ts = np.linspace(0.0, 3.0, 16)
    assert _check(H, [np.float32(np.sqrt(0.05)) * a], ops.fock(10, 0), ts, [num]) == 'trajectory'


def test_two_terms_n40(cuda_device):
    """PWC and Wave terms together at n = 40 (shared-memory tiles of 64), two jumps."""
    a, num, x = _osc(40)
    H = (0.3 * num + 0.02 * (ops.dag(a) @ ops.dag(a) @ a @ a)
         + dq.pwc([0.0, 0.4, 1.0], [0.5, -0.8], x)
         + dq.modulated(dq.Wave(1.0, amplitude=0.6), 1j * (ops.dag(a) - a)))
    L = [np.float32(np.sqrt(0.1)) * a, np.float32(np.sqrt(0.02)) * num]
    ts = np.linspace(0.0, 1.5, 7)
    _check(H, L, ops.fock(40, 0), ts, [num])


def test_batched_pwc_values_one_launch(cuda_device):
    """values of shape (3, N) and two initial states: one launch of 6 instances; results
    in cartesian order (H's value batch first), each equal to its single solve."""
    a, num, x = _osc(6)
    vals = np.array([[1.0, -0.5, 2.0], [0.2, 0.7, -1.0], [0.0, 1.0, 0.5]])
    times = [0.3, 0.8, 1.5, 2.2]
    H = 0.7 * num + dq.pwc(times, vals, x)
    L = [np.float32(np.sqrt(0.2)) * a]
    rho0 = np.stack([ops.fock(6, 0), ops.fock(6, 1)])
    ts = np.linspace(0.0, 3.0, 13)
    m = dq.Tsit5(rtol=1e-6, atol=1e-8)
    res = dq.mesolve(H, L, rho0, ts, method=m)
    assert res.states.shape == (3, 2, 13, 6, 6)
    for i in range(3):
        Hi = 0.7 * num + dq.pwc(times, vals[i], x)
        for j in range(2):
            one = dq.mesolve(Hi, L, rho0[j], ts, method=m)
            np.testing.assert_array_equal(res.states[i, j].cpu().numpy(), one.states.cpu().numpy())
        _check(Hi, L, rho0[0], ts, None, m=m)


# ---- the DIA stepper (dqb_mesolve_dia_td): every operator in sparse-DIA storage ----------

def _dia_modes(m):
    """Two coupled Kerr modes of m levels in DIA storage: H0, a drive operator on each mode,
    two jump operators (dense copies for the oracle) and the first mode's photon number."""
    a = ops.destroy(m, layout='dia')
    eye = ops.eye(m, layout='dia')
    a1, a2 = ops.tensor(a, eye), ops.tensor(eye, a)
    n1 = a1.dag() @ a1
    H0 = (a1.dag() @ a1.dag() @ a1 @ a1) * np.float32(0.05) + (a1.dag() @ a2 + a2.dag() @ a1) * \
        np.float32(0.1) + n1 * np.float32(0.3)
    x1 = a1 + a1.dag()
    y2 = (a2.dag() - a2) * np.complex64(1j)
    Ls = [a1 * np.float32(np.sqrt(0.1)), a2 * np.float32(np.sqrt(0.05))]
    return H0, x1, y2, Ls, [L.to_dense() for L in Ls], n1.to_dense()


def _check_dia(H, Ls, Ls_dense, rho0, ts, E, m, res=None, b=None):
    res = res if res is not None else dq.mesolve(H, Ls, rho0, ts, exp_ops=E, method=m)
    Hs = as_summed(H)
    st = res.states.cpu().numpy() if b is None else res.states[b].cpu().numpy()
    ex = None
    if E:
        ex = res.expects.cpu().numpy() if b is None else res.expects[b].cpu().numpy()
    ns = int(res.infos.nsteps if b is None else res.infos.nsteps[b])
    return assert_solve_parity(st, ex, ns, Hs, Ls_dense, rho0, ts, E, type(m).__name__, m.rtol,
                               m.atol, jump_ts=Hs.discontinuity_ts)


@pytest.mark.parametrize('method', ['Tsit5', 'Dopri5'])
def test_dia_pwc_and_wave_one_launch(cuda_device, method):
    """A PWC drive on one mode and a Gaussian-pulse Wave on the other (n = 100, DIA): one
    launch of the DIA stepper, Hnh formed at every stage time, steps clipped at the PWC
    times and the pulse's support edges (1.5 is also a save time), against the oracle with
    the same jump_ts."""
    from dynamiqs_b200.time_qarray import as_summed as _as

    H0, x1, y2, Ls, Ld, n1 = _dia_modes(10)
    pulse = dq.Wave(1.7, 0.3, 0.8 - 0.2j, t_center=1.2, sigma=0.5, t_start=0.4, t_end=2.4)
    H = H0 + dq.pwc([0.2, 0.9, 1.5, 2.6], [0.6, -0.4, 1.1], x1) + dq.modulated(pulse, y2)
    assert _as(H).is_dia
    ts = np.linspace(0.0, 3.0, 13)
    m = dq.Tsit5(rtol=1e-6, atol=1e-8) if method == 'Tsit5' else dq.Dopri5(rtol=1e-6, atol=1e-8)
    rho0 = ops.fock(100, 0)
    assert _check_dia(H, Ls, Ld, rho0, ts, [n1], m) == 'trajectory'


def test_dia_td_matches_dense_kernel_at_n36(cuda_device):
    """The same time-dependent problem (n = 36) through the DIA stepper and the n <= 64
    kernel: step counts equal and states within 1e-5."""
    H0, x1, y2, Ls, Ld, n1 = _dia_modes(6)
    H_dia = H0 + dq.pwc([0.1, 0.7, 1.3], [1.0, -0.6], x1) + dq.modulated(dq.Wave(2.0, amplitude=0.4), y2)
    H_dense = (H0.to_dense() + dq.pwc([0.1, 0.7, 1.3], [1.0, -0.6], x1.to_dense())
               + dq.modulated(dq.Wave(2.0, amplitude=0.4), y2.to_dense()))
    ts = np.linspace(0.0, 2.0, 9)
    m = dq.Tsit5(rtol=1e-6, atol=1e-8)
    rho0 = ops.fock(36, 0)
    r_dia = dq.mesolve(H_dia, Ls, rho0, ts, method=m)
    r_dense = dq.mesolve(H_dense, Ld, rho0, ts, method=m)
    assert int(r_dia.infos.nsteps) == int(r_dense.infos.nsteps)
    d = np.abs(r_dia.states.cpu().numpy() - r_dense.states.cpu().numpy()).max()
    assert d < 1e-5


def test_dia_batched_pwc_values(cuda_device):
    """PWC values of shape (3, N) with two initial states on the DIA stepper: one launch
    of 6 instances in cartesian order, each against the oracle."""
    H0, x1, y2, Ls, Ld, n1 = _dia_modes(8)
    vals = np.array([[1.0, -0.5, 2.0], [0.2, 0.7, -1.0], [0.0, 1.0, 0.5]])
    times = [0.3, 0.8, 1.5, 2.2]
    H = H0 + dq.pwc(times, vals, x1)
    rho0 = np.stack([ops.fock(64, 0), ops.fock(64, 1)])
    ts = np.linspace(0.0, 2.5, 11)
    m = dq.Tsit5(rtol=1e-6, atol=1e-8)
    res = dq.mesolve(H, Ls, rho0, ts, exp_ops=[n1], method=m)
    assert res.states.shape == (3, 2, 11, 64, 64)
    for i in range(3):
        Hi = H0 + dq.pwc(times, vals[i], x1)
        for j in range(2):
            one = type('R', (), {})()
            one.states, one.expects = res.states[i, j], res.expects[i, j]
            one.infos = type('I', (), {'nsteps': res.infos.nsteps[i, j]})()
            _check_dia(Hi, Ls, Ld, rho0[j], ts, [n1], m, res=one)


# ---- the GEMM path (dqb_mesolve_dense_large_td): dense operators beyond n = 64 ----------

@pytest.mark.parametrize('method', ['Tsit5', 'Dopri5'])
def test_large_dense_pwc_and_wave_one_launch(cuda_device, method):
    """n = 80 with dense operators: a PWC drive and a Gaussian Wave pulse in one launch of
    the GEMM path (Hnh formed at every stage time, steps clipped at the discontinuities),
    against the oracle with the same jump_ts."""
    a, num, x = _osc(80)
    pulse = dq.Wave(1.1, 0.0, 0.5 + 0.1j, t_center=1.0, sigma=0.3, t_start=0.3, t_end=1.8)
    H = (0.4 * num + 0.01 * (ops.dag(a) @ ops.dag(a) @ a @ a)
         + dq.pwc([0.1, 0.6, 1.2, 2.0], [0.8, -0.3, 0.5], x) + dq.modulated(pulse, 1j * (ops.dag(a) - a)))
    ts = np.linspace(0.0, 2.4, 9)
    m = dq.Tsit5(rtol=1e-6, atol=1e-8) if method == 'Tsit5' else dq.Dopri5(rtol=1e-6, atol=1e-8)
    assert _check(H, [np.float32(np.sqrt(0.1)) * a], ops.fock(80, 0), ts, [num], m=m) == 'trajectory'


def test_large_dense_batched_pwc_values(cuda_device):
    """PWC values of shape (2, N) with two initial states on the GEMM path: one launch of
    4 instances in cartesian order, each against the oracle."""
    a, num, x = _osc(72)
    vals = np.array([[1.0, -0.5, 0.7], [0.3, 0.9, -0.4]])
    times = [0.2, 0.7, 1.1, 1.6]
    H = 0.5 * num + dq.pwc(times, vals, x)
    L = [np.float32(np.sqrt(0.15)) * a]
    rho0 = np.stack([ops.fock(72, 0), ops.fock(72, 1)])
    ts = np.linspace(0.0, 2.0, 9)
    m = dq.Tsit5(rtol=1e-6, atol=1e-8)
    res = dq.mesolve(H, L, rho0, ts, exp_ops=[num], method=m)
    assert res.states.shape == (2, 2, 9, 72, 72)
    for i in range(2):
        Hi = 0.5 * num + dq.pwc(times, vals[i], x)
        for j in range(2):
            one = type('R', (), {})()
            one.states, one.expects = res.states[i, j], res.expects[i, j]
            one.infos = type('I', (), {'nsteps': res.infos.nsteps[i, j]})()
            _check(Hi, L, rho0[j], ts, [num], m=m, res=one)


# ---- time-dependent jump operators (DIA stepper) --------------------------------------

def _oracle_td_jumps(Hs, Ls, cfs, rho0, ts, jts, rtol=1e-6, atol=1e-8):
    """The Lindblad equation with H(t) = Hs(t) and jump operators c_k(t) L_k in complex128
    through the oracle's RK engine and hermitian vector field
    (diffrax_integrator.py:319-323), with the discontinuity times handed to its controller;
    returns the saved states, the step count and the parity step slack."""
    from oracle import lindblad as lb
    from oracle.rk import solve

    Ls = [np.asarray(L, dtype=complex) for L in Ls]

    def f(t, y):
        Lt = [complex(c(t)) * L for c, L in zip(cfs, Ls)]
        Hnh = lb.hnh_dense(np.asarray(Hs(t), dtype=complex), Lt)
        tmp = Hnh @ y
        for L in Lt:
            tmp = tmp + 0.5 * (L @ y @ L.conj().T)
        return tmp + tmp.conj().T

    psi = np.asarray(rho0, dtype=complex)
    rho = psi @ psi.conj().T if psi.shape[-1] == 1 else psi
    out = solve(f, rho, ts, rtol=rtol, atol=atol, save_fn=lambda y: y, jump_ts=jts)
    borderline = any(abs(e - 1.0) < 0.1 for (_, _, e) in out.errors)
    return np.stack(out.ysave), out.nsteps, (max(2, int(0.01 * out.nsteps)) if borderline else 1)


@pytest.mark.parametrize('td_h', [False, True])
def test_dia_time_dependent_jump_operators(cuda_device, td_h):
    """Jump operators with PWC and Wave prefactors (and one constant), with a constant or a
    time-dependent H, on the DIA stepper (n = 100): L_k(t) and Hnh(t) formed at every stage
    time, steps clipped at every discontinuity; against the oracle at 1e-5."""
    from dynamiqs_b200.time_qarray import as_summed

    H0, x1, y2, Ls, Ld, n1 = _dia_modes(10)
    a = ops.destroy(10, layout='dia')
    eye = ops.eye(10, layout='dia')
    a1, a2 = ops.tensor(a, eye), ops.tensor(eye, a)
    decay1 = dq.pwc([0.0, 0.7, 1.4], [1.0, 0.3], a1 * np.float32(np.sqrt(0.2)))
    decay2 = dq.modulated(dq.Wave(1.5, amplitude=1.0), a2 * np.float32(np.sqrt(0.1)))
    deph = (a1.dag() @ a1) * np.float32(0.05)
    jumps = [decay1, decay2, deph]
    H = H0 + dq.pwc([0.2, 0.9, 1.6], [0.5, -0.4], x1) if td_h else H0
    ts = np.linspace(0.0, 2.0, 9)
    m = dq.Tsit5(rtol=1e-6, atol=1e-8)
    rho0 = ops.fock(100, 0)
    res = dq.mesolve(H, jumps, rho0, ts, method=m)
    Hs = as_summed(H)
    jts = np.unique(np.concatenate([Hs.discontinuity_ts, decay1.discontinuity_ts,
                                    decay2.discontinuity_ts]))
    cfs = [decay1.prefactor, decay2.prefactor, lambda t: 1.0]
    ref, nsteps, slack = _oracle_td_jumps(Hs, [decay1.qarray, decay2.qarray, deph.to_dense()], cfs,
                                          rho0, ts, jts)
    err = np.linalg.norm(res.states.cpu().numpy() - ref, axis=(-2, -1)) / np.linalg.norm(ref, axis=(-2, -1))
    assert err.max() < 1e-5, err
    assert abs(int(res.infos.nsteps) - nsteps) <= slack, (int(res.infos.nsteps), nsteps)



@pytest.mark.parametrize('n', [12, 80])
def test_dense_time_dependent_jump_operators(cuda_device, n):
    """Dense operators with a PWC-modulated decay and a Wave-modulated dephasing, with a
    PWC drive on H, on the GEMM path (any n; n = 12 goes there too): the copies c_k(t) L_k
    and Hnh(t) = -iH(t) - 1/2 sum |c_k|^2 L_k^+ L_k formed at every stage time; against the
    oracle at 1e-5."""
    from dynamiqs_b200.time_qarray import as_summed

    a, num, x = _osc(n)
    decay = dq.pwc([0.0, 0.6, 1.3], [1.0, 0.4], np.float32(np.sqrt(0.2)) * a)
    deph = dq.modulated(dq.Wave(2.0, amplitude=0.8), np.float32(np.sqrt(0.02)) * num)
    H = 0.4 * num + dq.pwc([0.3, 0.9, 1.5], [0.6, -0.3], x)
    ts = np.linspace(0.0, 1.8, 7)
    m = dq.Tsit5(rtol=1e-6, atol=1e-8)
    rho0 = ops.fock(n, 1)
    res = dq.mesolve(H, [decay, deph], rho0, ts, exp_ops=[num], method=m)
    Hs = as_summed(H)
    jts = np.unique(np.concatenate([Hs.discontinuity_ts, decay.discontinuity_ts,
                                    deph.discontinuity_ts]))
    ref, nsteps, slack = _oracle_td_jumps(Hs, [decay.qarray, deph.qarray],
                                          [decay.prefactor, deph.prefactor], rho0, ts, jts)
    err = np.linalg.norm(res.states.cpu().numpy() - ref, axis=(-2, -1)) / np.linalg.norm(ref, axis=(-2, -1))
    assert err.max() < 1e-5, err
    assert abs(int(res.infos.nsteps) - nsteps) <= slack, (int(res.infos.nsteps), nsteps)
