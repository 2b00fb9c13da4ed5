"""Vectorization and superoperators (``dynamiqs/utils/vectorization.py``), in numpy with
the reference's conventions: ``vectorize`` stacks the columns of an operator
(``:25-59``), ``spre(A) = I (x) A``, ``spost(A) = A^T (x) I``, ``sprepost(A, B) =
B^T (x) A`` (``:100-175``), ``sdissipator`` and ``slindbladian`` (``:178-259``).  The
superoperators feed the vectorized master-equation kernel (``dqb_mesolve_vectorized``);
arithmetic is complex64 like the reference's default.
"""

from __future__ import annotations

import numpy as np

__all__ = ['vectorize', 'unvectorize', 'spre', 'spost', 'sprepost', 'sdissipator',
           'slindbladian']


def _dag(x):
    return np.conj(np.swapaxes(x, -1, -2))


def vectorize(x) -> np.ndarray:
    """(..., n, n) -> (..., n^2, 1), columns stacked."""
    x = np.asarray(x)
    return np.swapaxes(x, -1, -2).reshape(*x.shape[:-2], -1, 1)


def unvectorize(x) -> np.ndarray:
    """(..., n^2, 1) -> (..., n, n)."""
    x = np.asarray(x)
    n = int(round(np.sqrt(x.shape[-2])))
    return np.swapaxes(x.reshape(*x.shape[:-2], n, n), -1, -2)


def _kron(a, b):
    """Batched Kronecker product of (..., n, n) with (..., m, m)."""
    a, b = np.asarray(a), np.asarray(b)
    bs = np.broadcast_shapes(a.shape[:-2], b.shape[:-2])
    n, m = a.shape[-1], b.shape[-1]
    out = a[..., :, None, :, None] * b[..., None, :, None, :]
    return np.broadcast_to(out, (*bs, n, m, n, m)).reshape(*bs, n * m, n * m)


def spre(x) -> np.ndarray:
    x = np.asarray(x)
    return _kron(np.eye(x.shape[-1], dtype=x.dtype), x)


def spost(x) -> np.ndarray:
    x = np.asarray(x)
    return _kron(np.swapaxes(x, -1, -2), np.eye(x.shape[-1], dtype=x.dtype))


def sprepost(x, y) -> np.ndarray:
    return _kron(np.swapaxes(np.asarray(y), -1, -2), np.asarray(x))


def sdissipator(L) -> np.ndarray:
    L = np.asarray(L)
    Ld = _dag(L)
    LdL = Ld @ L
    return sprepost(L, Ld) - 0.5 * spre(LdL) - 0.5 * spost(LdL)


def slindbladian(H, jump_ops) -> np.ndarray:
    """-i (I (x) H) + i (H^T (x) I) + sum_k D[L_k] (``:213-259``)."""
    H = np.asarray(H)
    S = -1j * spre(H) + 1j * spost(H)
    for L in jump_ops:
        S = S + sdissipator(L)
    return S.astype(np.result_type(H.dtype, np.complex64))
