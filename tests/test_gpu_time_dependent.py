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
