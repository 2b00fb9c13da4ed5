"""GPU parity of the vectorized master equation (``Options(vectorized=True)``:
d vec(rho)/dt = S vec(rho) with S = slindbladian(H, jump_ops), ``dqb_mesolve_vectorized``)
against the oracle's vectorized form (``oracle.mesolve.mesolve(form='vectorized')``,
complex128), under the bar of tests/parity.py; n^2 <= 128 runs S from shared memory,
128 < n^2 <= 256 from global memory."""

import numpy as np
import pytest

import dynamiqs_b200 as dq
from dynamiqs_b200 import workloads
from tests.parity import assert_solve_parity, rel_frob
from tests.systems import random_problem

pytestmark = pytest.mark.gpu

VEC = dq.Options(vectorized=True)


def test_lossy_oscillator_vectorized(cuda_device):
    """The plain lossy oscillator (n = 16: S is 256 x 256, read from global memory)."""
    w = workloads.lossy_oscillator()
    res = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], exp_ops=w['exp_ops'],
                     method=w['method'], options=VEC)
    assert res.states.shape == (101, 16, 16) and res.expects.shape == (1, 101)
    m = w['method']
    assert_solve_parity(res.states.cpu().numpy(), res.expects.cpu().numpy(),
                        int(res.infos.nsteps), w['H'], w['jump_ops'], w['rho0'], w['tsave'],
                        w['exp_ops'], 'Tsit5', m.rtol, m.atol, form='vectorized')


@pytest.mark.parametrize('n,K', [(3, 1), (8, 2), (11, 3), (13, 1)])
@pytest.mark.parametrize('method', ['Tsit5', 'Dopri5'])
def test_random_vectorized(cuda_device, n, K, method):
    H, Ls, rho = random_problem(n, K, seed=3 * n + K)
    ts = np.linspace(0.0, 1.5, 6)
    m = dq.Tsit5() if method == 'Tsit5' else dq.Dopri5()
    res = dq.mesolve(H, Ls, rho, ts, method=m, options=VEC)
    assert_solve_parity(res.states.cpu().numpy(), None, int(res.infos.nsteps), H, Ls, rho, ts,
                        None, method, m.rtol, m.atol, form='vectorized')


def test_vectorized_batching(cuda_device):
    """Cartesian batching over H and a batched jump operator: one superoperator per
    distinct (H, jump set) pair; every instance equals its single solve."""
    n = 6
    H0, Ls, rho = random_problem(n, 1, seed=1)
    H1, _, _ = random_problem(n, 1, seed=2)
    Hs = np.stack([H0, H1])
    Lb = np.stack([Ls[0], 0.5 * Ls[0]])
    ts = np.linspace(0.0, 1.0, 4)
    res = dq.mesolve(Hs, [Lb], rho, ts, options=VEC)
    assert res.states.shape == (2, 2, 4, n, n)
    for i in range(2):
        for j in range(2):
            one = dq.mesolve(Hs[i], [Lb[j]], rho, ts, options=VEC)
            np.testing.assert_array_equal(res.states[i, j].cpu().numpy(), one.states.cpu().numpy())


def test_vectorized_beyond_kernel_limit_is_standard_form(cuda_device):
    """n = 20 (n^2 = 400 > 256): the same ODE through the standard form."""
    H, Ls, rho = random_problem(20, 2, seed=5)
    ts = np.linspace(0.0, 1.0, 3)
    a = dq.mesolve(H, Ls, rho, ts, options=VEC)
    b = dq.mesolve(H, Ls, rho, ts, options=dq.Options(assume_hermitian=False))
    assert rel_frob(a.states.cpu().numpy(), b.states.cpu().numpy()).max() == 0.0
