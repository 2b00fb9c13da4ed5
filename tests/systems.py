"""Small problems shared by the tests: the reference's analytic test systems and the
known-answer examples of its docs (``tests/golden/known_answers.json``)."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from dynamiqs_b200 import operators as ops

GOLDEN = json.loads((Path(__file__).parent / 'golden' / 'known_answers.json').read_text())


def ocavity(layout='dense', n=8, delta=2 * np.pi, kappa=2 * np.pi, alpha0=0.5):
    """``OCavity`` (reference tests/systems/open_system.py:131-209, instances :233-240)."""
    a = ops.destroy(n, layout=layout)
    H = ops.number(n, layout=layout) * np.float32(delta)
    Ls = [a * np.float32(np.sqrt(kappa))]
    tsave = np.linspace(0.0, 0.3, 11)
    Es = [ops.position(n, layout=layout), ops.momentum(n, layout=layout)]

    def alpha(t):
        return alpha0 * np.exp(-1j * delta * t - 0.5 * kappa * t)

    states = np.stack([ops.coherent_dm(n, alpha(t)) for t in tsave])
    expects = np.stack([alpha(tsave).real, alpha(tsave).imag])
    return dict(H=H, jump_ops=Ls, rho0=ops.coherent(n, alpha0), tsave=tsave, exp_ops=Es,
                true_states=states, true_expects=expects)


def readme_oscillator(atol=1e-6):
    n = 16
    a = ops.destroy(n, layout='dense')
    return dict(H=ops.dag(a) @ a, jump_ops=[np.float32(np.sqrt(0.1)) * a],
                rho0=ops.coherent(n, 1.0), tsave=np.linspace(0, 2 * np.pi, 101),
                rtol=1e-6, atol=atol)


def docstring_oscillator():
    n = 16
    a = ops.destroy(n, layout='dense')
    return dict(H=ops.dag(a) @ a, jump_ops=[a], rho0=ops.coherent(n, 1.0),
                tsave=np.linspace(0, 1.0, 11), rtol=1e-6, atol=1e-6)


def coherent_alpha_t(alpha0, omega, kappa, t):
    return alpha0 * np.exp(-1j * omega * t - 0.5 * kappa * t)


def random_problem(n, K, seed=0, hermitian_rho=True, batch=None):
    """Random dense H (hermitian), K random jump operators, random density matrix."""
    rng = np.random.default_rng(seed)

    def cplx(*shape):
        return (rng.normal(size=shape) + 1j * rng.normal(size=shape)) / np.sqrt(2 * n)

    shape = (batch,) if batch else ()
    X = cplx(*shape, n, n)
    H = 0.5 * (X + np.conj(np.swapaxes(X, -1, -2)))
    Ls = [0.5 * cplx(n, n) for _ in range(K)]
    Y = cplx(n, n)
    rho = Y @ np.conj(Y.T)
    rho = rho / np.trace(rho)
    if not hermitian_rho:
        rho = rho + 0.05 * cplx(n, n)
    c = np.ascontiguousarray
    return c(H, np.complex64), [c(L, np.complex64) for L in Ls], c(rho, np.complex64)
