"""Operator layouts accepted by ``dynamiqs_b200.mesolve``.

* dense: any array-like of shape ``(..., n, n)`` (numpy, torch, nested lists), as the
  reference's ``DenseDataArray`` (``dynamiqs/qarrays/dense_dataarray.py``).
* sparse DIA: :class:`SparseDIA`, the storage of ``SparseDIADataArray``
  (``dynamiqs/qarrays/sparsedia_dataarray.py:42-71``): a static tuple of distinct
  ``offsets`` and ``diags`` of shape ``(..., ndiags, n)``, column-indexed -- for offset
  k, ``diags[..., d, j] = A[j - k, j]`` -- with the out-of-range entries (the first k
  for k >= 0, the last |k| for k < 0) equal to zero, which the constructor checks as the
  reference does (``sparsedia_dataarray.py:62-71``).

The host-side algebra here (``+``, scalar ``*``, ``@`` between DIA operators,
``dag``) builds inputs the way ``dq.destroy(n) ...`` expressions do; it runs once per
problem definition, never inside the solve.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ['SparseDIA', 'dense', 'dia', 'to_dense', 'isdia']

dense = 'dense'
dia = 'dia'


def _sl(k: int) -> slice:
    return slice(k, None) if k >= 0 else slice(None, k)


@dataclass(frozen=True, eq=False)
class SparseDIA:
    offsets: tuple
    diags: np.ndarray

    def __post_init__(self):
        offsets = tuple(int(k) for k in self.offsets)
        object.__setattr__(self, 'offsets', offsets)
        diags = np.asarray(self.diags)
        if not np.iscomplexobj(diags):
            diags = diags.astype(np.complex64)
        object.__setattr__(self, 'diags', diags)
        if diags.ndim < 2 or diags.shape[-2] != len(offsets):
            raise ValueError(
                f'Argument `diags` must have shape (..., {len(offsets)}, n), but has shape '
                f'{diags.shape}.')
        if len(set(offsets)) != len(offsets):
            raise ValueError('Argument `offsets` must contain distinct values.')
        n = diags.shape[-1]
        for d, k in enumerate(offsets):
            if abs(k) > n - 1:
                raise ValueError(f'Offset {k} is out of range for dimension {n}.')
            pad = diags[..., d, :k] if k >= 0 else diags[..., d, n + k:]
            if np.any(pad != 0):
                raise ValueError(
                    'Diagonals must be filled with zeros outside the matrix (the first '
                    f'{k} entries for offset {k} >= 0, the last |k| entries for offset '
                    '< 0).')

    # ---- shape ------------------------------------------------------------------
    @property
    def n(self) -> int:
        return self.diags.shape[-1]

    @property
    def shape(self) -> tuple:
        return (*self.diags.shape[:-2], self.n, self.n)

    @property
    def ndim(self) -> int:
        return len(self.shape)

    @property
    def dtype(self):
        return self.diags.dtype

    # ---- conversions --------------------------------------------------------------
    def to_dense(self) -> np.ndarray:
        n = self.n
        out = np.zeros(self.shape, dtype=self.diags.dtype)
        for d, k in enumerate(self.offsets):
            cols = np.arange(max(k, 0), n + min(k, 0))
            out[..., cols - k, cols] = self.diags[..., d, cols]
        return out

    @staticmethod
    def from_dense(x, offsets=None, dtype=np.complex64) -> SparseDIA:
        x = np.asarray(x, dtype=dtype)
        n = x.shape[-1]
        if offsets is None:
            offsets = tuple(k for k in range(-(n - 1), n)
                            if np.any(np.diagonal(x, offset=k, axis1=-2, axis2=-1) != 0))
        diags = np.zeros((*x.shape[:-2], len(offsets), n), dtype=dtype)
        for d, k in enumerate(offsets):
            diags[..., d, _sl(k)] = np.diagonal(x, offset=k, axis1=-2, axis2=-1)
        return SparseDIA(tuple(offsets), diags)

    def astype(self, dtype) -> SparseDIA:
        return SparseDIA(self.offsets, self.diags.astype(dtype))

    # ---- algebra (host side, mirrors sparsedia_primitives.py) -----------------------
    def dag(self) -> SparseDIA:
        out = np.zeros_like(self.diags)
        for d, k in enumerate(self.offsets):
            out[..., d, _sl(-k)] = self.diags[..., d, _sl(k)]
        return SparseDIA(tuple(-k for k in self.offsets), np.conj(out))

    def __neg__(self):
        return SparseDIA(self.offsets, -self.diags)

    def __mul__(self, s):
        if np.ndim(s) == 0:
            return SparseDIA(self.offsets, (self.diags * s).astype(np.result_type(self.diags, s)))
        s = np.asarray(s)[..., None, None]
        return SparseDIA(self.offsets, self.diags * s)

    __rmul__ = __mul__

    def __truediv__(self, s):
        return self * (1.0 / s)

    def __add__(self, other):
        if not isinstance(other, SparseDIA):
            return NotImplemented
        offsets = tuple(int(k) for k in np.union1d(self.offsets, other.offsets))
        bshape = np.broadcast_shapes(self.diags.shape[:-2], other.diags.shape[:-2])
        out = np.zeros((*bshape, len(offsets), self.n),
                       dtype=np.promote_types(self.dtype, other.dtype))
        for i, k in enumerate(offsets):
            if k in self.offsets:
                out[..., i, :] += self.diags[..., self.offsets.index(k), :]
            if k in other.offsets:
                out[..., i, :] += other.diags[..., other.offsets.index(k), :]
        return SparseDIA(offsets, out)

    def __sub__(self, other):
        return self + (-other)

    def __matmul__(self, other):
        if isinstance(other, SparseDIA):
            n = self.n
            bshape = np.broadcast_shapes(self.diags.shape[:-2], other.diags.shape[:-2])
            dtype = np.promote_types(self.dtype, other.dtype)
            acc: dict[int, np.ndarray] = {}
            for i, lk in enumerate(self.offsets):
                for j, rk in enumerate(other.offsets):
                    k = lk + rk
                    if abs(k) > n - 1:
                        continue
                    rs = _sl(rk)
                    v = self.diags[..., i, _sl(-rk)] * other.diags[..., j, rs]
                    if k not in acc:
                        acc[k] = np.zeros((*bshape, n), dtype=dtype)
                    acc[k][..., rs] += v
            ks = tuple(sorted(acc))
            if not ks:
                return SparseDIA((0,), np.zeros((*bshape, 1, n), dtype=dtype))
            return SparseDIA(ks, np.stack([acc[k] for k in ks], axis=-2))
        return self.to_dense() @ np.asarray(other)

    def __rmatmul__(self, other):
        return np.asarray(other) @ self.to_dense()

    def __repr__(self):
        return f'SparseDIA(shape={self.shape}, offsets={self.offsets}, dtype={self.dtype})'


def isdia(x) -> bool:
    return isinstance(x, SparseDIA)


def to_dense(x) -> np.ndarray:
    if isinstance(x, SparseDIA):
        return x.to_dense()
    if hasattr(x, 'detach'):  # torch tensor
        return x.detach().cpu().numpy()
    return np.asarray(x)


def kron(a, b):
    """Tensor product of two operators (dense or DIA), ``dq.tensor`` for two factors."""
    if isinstance(a, SparseDIA) and isinstance(b, SparseDIA):
        nb = b.n
        offs = np.ravel(np.asarray(a.offsets)[:, None] * nb + np.asarray(b.offsets)[None, :])
        diags = np.einsum('...ai,...bj->...abij', a.diags, b.diags)
        diags = diags.reshape(*diags.shape[:-4], len(a.offsets) * len(b.offsets), a.n * nb)
        uniq, inv = np.unique(offs, return_inverse=True)
        out = np.zeros((*diags.shape[:-2], len(uniq), a.n * nb), dtype=diags.dtype)
        for i in range(len(uniq)):
            out[..., i, :] = diags[..., inv == i, :].sum(-2)
        return SparseDIA(tuple(int(k) for k in uniq), out)
    return np.kron(to_dense(a), to_dense(b))
