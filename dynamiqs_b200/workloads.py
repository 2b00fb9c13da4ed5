"""Seeded synthetic mesolve workloads of the benchmark shapes.

No dataset is involved: every problem is generated from a NumPy ``default_rng(seed)``.

* :func:`lossy_oscillator` -- n=16, H = omega a^+a, L = sqrt(kappa) a, rho0 = |alpha0>,
  tsave = linspace(0, 2 pi, 101), Tsit5 rtol 1e-6 atol 1e-8 (one instance).
* :func:`batched_kerr` -- n=64, B=4096, H_b = Delta a^+a + (K/2) a^+2 a^2
  + eps (a + a^+) with Delta~U(-1,1), K~U(0,0.5), eps~U(0,2); L = sqrt(0.1) a,
  sqrt(0.01) a^+a; rho0 = vacuum; t in [0,10], 51 saves; Tsit5 rtol 1e-6 atol 1e-8.
* :func:`transmon_cavity` -- transmon(4) x cavity(64), n=256, B=256.
* :func:`coupled_kerr_dia` -- two Kerr modes of 64 levels in sparse DIA (n=4096), B=8.
* :func:`serving_requests` -- a Poisson request stream of random Kerr problems.
"""

from __future__ import annotations

import numpy as np

from . import operators as ops
from .method import Tsit5
from .qarrays import SparseDIA

__all__ = ['lossy_oscillator', 'batched_kerr', 'transmon_cavity', 'coupled_kerr_dia',
           'serving_requests', 'kerr_hamiltonians']


def lossy_oscillator(n: int = 16, omega: float = 1.0, kappa: float = 0.1,
                     alpha0: float = 1.0, layout: str = 'dense') -> dict:
    a = ops.destroy(n, layout=layout)
    H = omega * (ops.dag(a) @ a)
    return dict(H=H, jump_ops=[np.float32(np.sqrt(kappa)) * a],
                rho0=ops.coherent(n, alpha0), tsave=np.linspace(0.0, 2 * np.pi, 101),
                exp_ops=[ops.number(n, layout='dense')], method=Tsit5(rtol=1e-6, atol=1e-8))


def kerr_hamiltonians(n: int, delta, kerr, eps) -> np.ndarray:
    """Dense H_b = Delta_b a^+a + (K_b/2) a^+2 a^2 + eps_b (a + a^+), shape (B, n, n).
    a^+a and a^+2 a^2 are diagonal, a + a^+ is tridiagonal."""
    delta, kerr, eps = (np.asarray(x, dtype=np.float64) for x in (delta, kerr, eps))
    k = np.arange(n, dtype=np.float64)
    num = k
    kk = k * (k - 1)
    B = delta.shape[0]
    H = np.zeros((B, n, n), dtype=np.complex64)
    idx = np.arange(n)
    H[:, idx, idx] = (delta[:, None] * num + 0.5 * kerr[:, None] * kk).astype(np.complex64)
    off = np.sqrt(np.arange(1, n, dtype=np.float64))
    H[:, idx[:-1], idx[1:]] = (eps[:, None] * off).astype(np.complex64)
    H[:, idx[1:], idx[:-1]] = (eps[:, None] * off).astype(np.complex64)
    return H


def batched_kerr(batch: int = 4096, n: int = 64, seed: int = 0) -> dict:
    rng = np.random.default_rng(seed)
    delta = rng.uniform(-1.0, 1.0, batch)
    kerr = rng.uniform(0.0, 0.5, batch)
    eps = rng.uniform(0.0, 2.0, batch)
    a = ops.destroy(n, layout='dense')
    H = kerr_hamiltonians(n, delta, kerr, eps)
    Ls = [np.float32(np.sqrt(0.1)) * a, np.float32(np.sqrt(0.01)) * (ops.dag(a) @ a)]
    return dict(H=H, jump_ops=Ls, rho0=ops.fock(n, 0), tsave=np.linspace(0.0, 10.0, 51),
                exp_ops=[ops.number(n, layout='dense')], method=Tsit5(rtol=1e-6, atol=1e-8),
                params=dict(delta=delta, kerr=kerr, eps=eps, seed=seed))


def transmon_cavity(batch: int = 256, nq: int = 4, nc: int = 64, seed: int = 0) -> dict:
    rng = np.random.default_rng(seed)
    wc = rng.uniform(0.9, 1.1, batch)
    wq = rng.uniform(0.8, 1.2, batch)
    chi = rng.uniform(1e-3, 1e-2, batch)
    eps = rng.uniform(0.0, 0.5, batch)
    alpha = 0.2
    b = np.kron(ops.destroy(nq, layout='dense'), np.eye(nc, dtype=np.complex64))
    a = np.kron(np.eye(nq, dtype=np.complex64), ops.destroy(nc, layout='dense'))
    na = ops.dag(a) @ a
    nb = ops.dag(b) @ b
    bb = ops.dag(b) @ ops.dag(b) @ b @ b
    H = (wc[:, None, None] * na + wq[:, None, None] * nb - 0.5 * alpha * bb
         + chi[:, None, None] * (na @ nb) + eps[:, None, None] * (a + ops.dag(a)))
    n = nq * nc
    rho0 = np.zeros((n, 1), dtype=np.complex64)
    rho0[0, 0] = 1.0
    return dict(H=H.astype(np.complex64),
                jump_ops=[np.float32(np.sqrt(0.01)) * a, np.float32(np.sqrt(0.005)) * b],
                rho0=rho0, tsave=np.linspace(0.0, 20.0, 41), exp_ops=[na.astype(np.complex64)],
                method=Tsit5(rtol=1e-6, atol=1e-8),
                params=dict(wc=wc, wq=wq, chi=chi, eps=eps, seed=seed))


def coupled_kerr_dia(batch: int = 8, m: int = 64, seed: int = 0, kerr: float = 0.05,
                     g: float = 0.1, eps: float = 1.0, kappa: float = 0.05) -> dict:
    rng = np.random.default_rng(seed)
    deltas = rng.uniform(-0.5, 0.5, (batch, 2))
    a = ops.destroy(m, layout='dia')
    I = ops.eye(m, layout='dia')
    a1 = ops.tensor(a, I)
    a2 = ops.tensor(I, a)
    n1 = a1.dag() @ a1
    n2 = a2.dag() @ a2
    k1 = a1.dag() @ a1.dag() @ a1 @ a1
    k2 = a2.dag() @ a2.dag() @ a2 @ a2
    hop = a1.dag() @ a2 + a2.dag() @ a1
    drive = a1 + a1.dag()
    static = k1 * np.float32(kerr / 2) + k2 * np.float32(kerr / 2) + hop * np.float32(g) \
        + drive * np.float32(eps)
    Hs = []
    for b in range(batch):
        Hs.append(static + n1 * np.float32(deltas[b, 0]) + n2 * np.float32(deltas[b, 1]))
    offsets = Hs[0].offsets
    H = SparseDIA(offsets, np.stack([h.diags for h in Hs]))
    n = m * m
    rho0 = np.zeros((n, 1), dtype=np.complex64)
    rho0[0, 0] = 1.0
    Ls = [a1 * np.float32(np.sqrt(kappa)), a2 * np.float32(np.sqrt(kappa))]
    return dict(H=H, jump_ops=Ls, rho0=rho0, tsave=np.linspace(0.0, 5.0, 11),
                exp_ops=None, method=Tsit5(rtol=1e-5, atol=1e-7),
                params=dict(deltas=deltas, seed=seed))


def serving_requests(num: int, rate: float = 2000.0, seed: int = 0,
                     dims=(8, 16, 32, 64, 128, 256),
                     weights=(0.30, 0.25, 0.20, 0.15, 0.07, 0.03)) -> list[dict]:
    """Poisson arrivals (mean ``rate`` req/s) of random Kerr problems: dim drawn from
    ``dims`` with ``weights``; 1-3 jumps (sqrt(kappa) a with kappa~U(0.01, 0.2), then
    optionally sqrt(gamma) a^+a and sqrt(gamma2) a^2); t_end~U(1, 20); 11-201 saves;
    Tsit5 rtol 1e-6."""
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for i in range(num):
        t += rng.exponential(1.0 / rate)
        n = int(rng.choice(dims, p=np.asarray(weights) / np.sum(weights)))
        delta, kerr, eps = rng.uniform(-1, 1), rng.uniform(0, 0.5), rng.uniform(0, 2)
        H = kerr_hamiltonians(n, [delta], [kerr], [eps])[0]
        a = ops.destroy(n, layout='dense')
        nj = int(rng.integers(1, 4))
        Ls = [np.float32(np.sqrt(rng.uniform(0.01, 0.2))) * a]
        if nj >= 2:
            Ls.append(np.float32(np.sqrt(rng.uniform(0.001, 0.02))) * (ops.dag(a) @ a))
        if nj >= 3:
            Ls.append(np.float32(np.sqrt(rng.uniform(0.001, 0.02))) * (a @ a))
        t_end = rng.uniform(1.0, 20.0)
        nsave = int(rng.integers(11, 202))
        reqs.append(dict(id=i, arrival=t, n=n, H=H, jump_ops=Ls, rho0=ops.fock(n, 0),
                         tsave=np.linspace(0.0, t_end, nsave),
                         exp_ops=[ops.number(n, layout='dense')],
                         method=Tsit5(rtol=1e-6, atol=1e-6)))
    return reqs
