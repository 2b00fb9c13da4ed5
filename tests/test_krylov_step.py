"""The Krylov form of the RK step used by the sparse-DIA path (``kry_*`` kernels of the
stepper), checked on the CPU: for a linear constant right-hand side dy/dt = A y, every
stage, y1, the embedded error estimate, the next first stage (FSAL) and the dense output
of one Tsit5 / Dopri5 step are the polynomials in hA that the kernels evaluate from the
basis u_q = (tau A)^q y, with the coefficients computed by the same recurrences
(alpha_{j,0} = 1, alpha_{j,m} = sum_l a_jl alpha_{l,m-1}).  The stage-by-stage step is
the oracle's tableau applied directly."""

import numpy as np
import pytest

from oracle.rk import DOPRI5, TSIT5, dense_weights


def _alpha(tab):
    al = np.zeros((7, 7))
    for j in range(7):
        al[j, 0] = 1.0
        for m in range(1, 7):
            al[j, m] = sum(tab.a[j, l] * al[l, m - 1] for l in range(j))
    return al


def _coefs(tab, r, sig1):
    """(cy, ce, cs): the coefficients of u_0..u_7 in y1, the error and tau A y1."""
    al = _alpha(tab)
    beta = np.array([1.0] + [tab.b @ al[:, q - 1] for q in range(1, 8)])
    eps = np.array([0.0] + [tab.btilde @ al[:, q - 1] for q in range(1, 8)])
    rp = r ** np.arange(8)
    s = np.ones(8)
    s[1] = sig1
    cy = beta * rp * s
    ce = eps * rp * s
    cs = np.zeros(8)
    cs[1:] = beta[:7] * rp[:7] * s[1:]
    return cy, ce, cs


def _dense(tab, theta, r, sig1):
    al = _alpha(tab)
    w = dense_weights(tab, theta)
    cw = np.array([1.0] + [w @ al[:, q - 1] * r ** q for q in range(1, 8)])
    cw[1] *= sig1
    return cw


def _stage_step(tab, A, y, h):
    k = []
    for j in range(7):
        x = y + h * sum(tab.a[j, l] * k[l] for l in range(j))
        k.append(A @ x)
    y1 = y + h * sum(tab.b[j] * k[j] for j in range(7))
    err = h * sum(tab.btilde[j] * k[j] for j in range(7))
    return k, y1, err


@pytest.mark.parametrize('tab', [TSIT5, DOPRI5], ids=['Tsit5', 'Dopri5'])
@pytest.mark.parametrize('r,sig1', [(1.0, 1.0), (0.37, 1.0), (0.8, 2.5)])
def test_krylov_step_equals_stage_step(tab, r, sig1):
    rng = np.random.default_rng(5)
    n = 6
    A = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))) * 0.7
    y = rng.normal(size=n) + 1j * rng.normal(size=n)
    tau = 0.21
    h = r * tau
    # the basis as the kernels hold it: u_1 stored divided by sig1
    u = [y]
    for _ in range(7):
        u.append(tau * (A @ u[-1]))
    stored = list(u)
    stored[1] = u[1] / sig1
    cy, ce, cs = _coefs(tab, r, sig1)
    y1 = sum(cy[q] * stored[q] for q in range(8))
    err = sum(ce[q] * stored[q] for q in range(8))
    s1 = sum(cs[q] * stored[q] for q in range(8))
    k, y1_ref, err_ref = _stage_step(tab, A, y, h)
    np.testing.assert_allclose(y1, y1_ref, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(err, err_ref, rtol=1e-9, atol=1e-13)
    np.testing.assert_allclose(s1, tau * (A @ y1_ref), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(k[6], A @ y1_ref, rtol=1e-12, atol=1e-12)  # FSAL: a_7j = b_j
    for theta in (0.0, 0.3, 0.77, 1.0):
        cw = _dense(tab, theta, r, sig1)
        yt = sum(cw[q] * stored[q] for q in range(8))
        yt_ref = y + h * sum(w * kj for w, kj in zip(dense_weights(tab, theta), k))
        np.testing.assert_allclose(yt, yt_ref, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize('tab,order', [(TSIT5, 4), (DOPRI5, 4)], ids=['Tsit5', 'Dopri5'])
def test_krylov_error_has_no_low_order_terms(tab, order):
    """The error estimate's coefficients vanish up to the embedded order (to the rounding
    of the published tableau digits), so the Krylov-form estimate is a sum of O(h^5)
    terms, not a difference of O(h) stage values."""
    _, ce, _ = _coefs(tab, 1.0, 1.0)
    assert np.all(np.abs(ce[:order + 1]) < 1e-14)
    assert np.abs(ce[order + 1:]).max() > 1e-5
    cy, _, _ = _coefs(tab, 1.0, 1.0)
    fact = np.array([1, 1, 2, 6, 24, 120], dtype=float)
    np.testing.assert_allclose(cy[:6], 1.0 / fact, rtol=1e-12)  # y1 = exp(hA) y to order 5
