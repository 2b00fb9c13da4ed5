"""The oracle's adaptive RK agrees with an independent FP64 integrator (scipy DOP853,
rtol 1e-12) and with the Liouvillian exponential (the reference's Expm idea,
dynamiqs/integrators/core/expm_integrator.py:59-87) to well below the 1e-5 bar."""

import numpy as np
import scipy.integrate as si
import scipy.linalg as sl

from oracle import lindblad as lb
from oracle.mesolve import mesolve
from tests.systems import random_problem


def test_oracle_vs_expm_and_dop853():
    H, Ls, rho = random_problem(6, 2, seed=3)
    H, Ls, rho = H.astype(complex), [L.astype(complex) for L in Ls], rho.astype(complex)
    tsave = np.linspace(0, 2.0, 9)
    r = mesolve(H, Ls, rho, tsave, rtol=1e-10, atol=1e-12, method='Dopri5')
    S = lb.slindbladian(H, Ls)
    ref = np.stack([lb.unvectorize(sl.expm(S * t) @ lb.vectorize(rho)) for t in tsave])
    rel = np.linalg.norm(r.states - ref, axis=(-2, -1)) / np.linalg.norm(ref, axis=(-2, -1))
    assert rel.max() < 1e-8
    sol = si.solve_ivp(lambda t, v: (S @ v[:, None])[:, 0], (0, 2.0),
                       lb.vectorize(rho)[:, 0], method='DOP853', t_eval=tsave, rtol=1e-12,
                       atol=1e-14)
    ref2 = np.stack([lb.unvectorize(sol.y[:, i:i + 1]) for i in range(len(tsave))])
    assert np.abs(ref2 - ref).max() < 1e-9


def test_tsit5_default_tolerance_error():
    H, Ls, rho = random_problem(8, 1, seed=4)
    tsave = np.linspace(0, 3.0, 7)
    r = mesolve(H, Ls, rho, tsave, rtol=1e-6, atol=1e-8)
    S = lb.slindbladian(H.astype(complex), [L.astype(complex) for L in Ls])
    ref = np.stack([lb.unvectorize(sl.expm(S * t) @ lb.vectorize(rho.astype(complex))) for t in tsave])
    rel = np.linalg.norm(r.states - ref, axis=(-2, -1)) / np.linalg.norm(ref, axis=(-2, -1))
    assert rel.max() < 1e-5
