"""The oracle's Runge-Kutta coefficients satisfy the order conditions of the published
pairs (Tsitouras 2011; Dormand & Prince 1980) and the dense outputs interpolate."""

import numpy as np
import pytest

from oracle.rk import DOPRI5, TSIT5, dense_weights, dopri5_dense_weights


@pytest.mark.parametrize('tab', [TSIT5, DOPRI5], ids=lambda t: t.name)
def test_order_conditions(tab):
    c, A, b = tab.c, tab.a, tab.b
    bhat = b - tab.btilde
    np.testing.assert_allclose(A.sum(1), c, atol=1e-14)
    for k in range(1, 6):  # bushy-tree conditions b . c^(k-1) = 1/k
        assert abs(b @ c ** (k - 1) - 1 / k) < 1e-13
    for k in range(1, 5):
        assert abs(bhat @ c ** (k - 1) - 1 / k) < 1e-13
    assert abs(b @ (A @ c) - 1 / 6) < 1e-13
    assert abs(b @ (A @ c ** 2) - 1 / 12) < 1e-13
    assert abs(b @ (A @ (A @ c)) - 1 / 24) < 1e-13
    assert abs(bhat @ (A @ c) - 1 / 6) < 1e-13
    np.testing.assert_allclose(A[6], b)  # FSAL


@pytest.mark.parametrize('tab', [TSIT5, DOPRI5], ids=lambda t: t.name)
def test_dense_output_endpoints(tab):
    np.testing.assert_allclose(dense_weights(tab, 0.0), 0.0, atol=1e-15)
    np.testing.assert_allclose(dense_weights(tab, 1.0), tab.b, atol=1e-14)
    for th in (0.1, 0.37, 0.8):
        # consistency: sum_i w_i(theta) = theta
        assert abs(dense_weights(tab, th).sum() - th) < 1e-14


def test_dopri5_dense_closed_form():
    """The closed form used by the CUDA kernels equals the oracle's solved quartic."""
    from oracle.rk import DOPRI5_C_MID
    for t in np.linspace(0, 1, 7):
        t2, t3, t4 = t * t, t ** 3, t ** 4
        w = DOPRI5.b * (-5 * t2 + 14 * t3 - 8 * t4) + DOPRI5_C_MID * (16 * t2 - 32 * t3 + 16 * t4)
        w[0] += t - 4 * t2 + 5 * t3 - 2 * t4
        w[6] += t2 - 3 * t3 + 2 * t4
        np.testing.assert_allclose(w, dopri5_dense_weights(t), atol=1e-13)


def test_dense_output_accuracy():
    """Interpolating y' = -y over one step reproduces exp(-t) to 4th/5th order."""
    for tab, tol in ((TSIT5, 1e-6), (DOPRI5, 1e-6)):
        h = 0.1
        ks = []
        for i in range(7):
            yi = 1.0 + h * sum(tab.a[i, j] * ks[j] for j in range(i))
            ks.append(-yi)
        for th in (0.25, 0.5, 0.75):
            w = dense_weights(tab, th)
            y = 1.0 + h * np.dot(w, ks)
            assert abs(y - np.exp(-th * h)) < tol
