"""Operator and state constructors used to define mesolve problems.

Same definitions and default layouts as the reference's constructors
(``dynamiqs/utils/operators.py``, ``dynamiqs/utils/states.py``): ``destroy``,
``create``, ``number``, ``position``, ``momentum`` and the Pauli operators return
:class:`~dynamiqs_b200.qarrays.SparseDIA` by default (``layout='dia'``, the reference's
default layout, ``dynamiqs/qarrays/layout.py:20``) or dense numpy arrays with
``layout='dense'``; ``displace``, ``coherent``, ``fock`` and ``coherent_dm`` are dense.
All values are complex64 like the reference's default ``cdtype``.
"""

from __future__ import annotations

import numpy as np

from .qarrays import SparseDIA, dense, dia, kron, to_dense

__all__ = ['destroy', 'create', 'number', 'eye', 'position', 'momentum', 'sigmax',
           'sigmay', 'sigmaz', 'sigmap', 'sigmam', 'displace', 'fock', 'coherent',
           'coherent_dm', 'tensor', 'dag', 'todm', 'expect']

CDTYPE = np.complex64


def _layout(layout):
    return dia if layout is None else layout


def _finish(x: SparseDIA, layout):
    return x if _layout(layout) == dia else x.to_dense()


def eye(n: int, *, layout=None):
    """Identity (``operators.py:46``)."""
    return _finish(SparseDIA((0,), np.ones((1, n), dtype=CDTYPE)), layout)


def destroy(n: int, *, layout=None):
    """Annihilation operator a, a[j-1, j] = sqrt(j) (``operators.py:242-307``)."""
    d = np.zeros((1, n), dtype=CDTYPE)
    d[0, 1:] = np.sqrt(np.arange(1, n))
    return _finish(SparseDIA((1,), d), layout)


def create(n: int, *, layout=None):
    """Creation operator a^+ (``operators.py:310``)."""
    d = np.zeros((1, n), dtype=CDTYPE)
    d[0, :-1] = np.sqrt(np.arange(1, n))
    return _finish(SparseDIA((-1,), d), layout)


def number(n: int, *, layout=None):
    """Number operator a^+ a (``operators.py:378``)."""
    return _finish(SparseDIA((0,), np.arange(n, dtype=CDTYPE)[None]), layout)


def position(n: int, *, layout=None, hbar: float = 0.5):
    """x = sqrt(hbar/2) (a^+ + a) (``operators.py:576-597``)."""
    a = destroy(n, layout=dia)
    return _finish((a.dag() + a) * np.float32(np.sqrt(hbar / 2)), layout)


def momentum(n: int, *, layout=None, hbar: float = 0.5):
    """p = i sqrt(hbar/2) (a^+ - a) (``operators.py:600-621``)."""
    a = destroy(n, layout=dia)
    return _finish((a.dag() - a) * np.complex64(1j * np.sqrt(hbar / 2)), layout)


def _pauli(mat, layout):
    x = np.asarray(mat, dtype=CDTYPE)
    return x if _layout(layout) == dense else SparseDIA.from_dense(x)


def sigmax(*, layout=None):
    return _pauli([[0, 1], [1, 0]], layout)


def sigmay(*, layout=None):
    return _pauli([[0, -1j], [1j, 0]], layout)


def sigmaz(*, layout=None):
    return _pauli([[1, 0], [0, -1]], layout)


def sigmap(*, layout=None):
    return _pauli([[0, 1], [0, 0]], layout)


def sigmam(*, layout=None):
    return _pauli([[0, 0], [1, 0]], layout)


def _expm_antihermitian(G: np.ndarray) -> np.ndarray:
    """exp(G) for anti-hermitian G via the eigendecomposition of the hermitian iG."""
    w, v = np.linalg.eigh(1j * G)
    return (v * np.exp(-1j * w)[..., None, :]) @ np.conj(np.swapaxes(v, -1, -2))


def displace(n: int, alpha) -> np.ndarray:
    """D(alpha) = exp(alpha a^+ - alpha^* a) in the truncated space (``operators.py:476-505``)."""
    alpha = np.asarray(alpha, dtype=np.complex128)[..., None, None]
    a = destroy(n, layout=dense).astype(np.complex128)
    G = alpha * a.conj().T - np.conj(alpha) * a
    return _expm_antihermitian(G).astype(CDTYPE)


def fock(n: int, k) -> np.ndarray:
    """Fock ket |k> of shape (n, 1) (``states.py:33``)."""
    k = np.asarray(k)
    out = np.zeros((*k.shape, n, 1), dtype=CDTYPE)
    np.put_along_axis(out, k[..., None, None], 1.0, axis=-2)
    return out


def coherent(n: int, alpha) -> np.ndarray:
    """Coherent ket D(alpha)|0> (``states.py:196-264``)."""
    return displace(n, alpha) @ fock(n, 0)


def coherent_dm(n: int, alpha) -> np.ndarray:
    psi = coherent(n, alpha)
    return psi @ np.conj(np.swapaxes(psi, -1, -2))


def tensor(*ops):
    out = ops[0]
    for o in ops[1:]:
        out = kron(out, o)
    return out


def dag(x):
    if isinstance(x, SparseDIA):
        return x.dag()
    x = np.asarray(x)
    return np.conj(np.swapaxes(x, -1, -2))


def todm(x):
    x = to_dense(x)
    return x @ np.conj(np.swapaxes(x, -1, -2)) if x.shape[-1] == 1 else x


def expect(E, rho):
    """tr(E rho) as ``(E * rho.mT).sum((-2, -1))`` (``dynamiqs/utils/general.py:276``)."""
    E, rho = to_dense(E), to_dense(rho)
    return (E * np.swapaxes(rho, -1, -2)).sum((-2, -1))
