"""CPU restatement (test infrastructure only) of the Lindblad vector fields and the
sparse-DIA primitives of dynamiqs' ``mesolve`` hot path.

Imported only by ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs,
as the checker; never by the product package.

Vector fields (``dynamiqs/integrators/core/diffrax_integrator.py:312-336``):

* hermitian (default, ``assume_hermitian=True``, ``:319-323``)::

      Hnh = -1j * H - 0.5 * sum(L^dag L)
      tmp = Hnh @ rho + 0.5 * sum(L @ rho @ L^dag)
      out = tmp + tmp^dag

* standard (``assume_hermitian=False``, ``:312-317``)::

      out = (-1j H - 0.5 sum L^dag L) @ rho + rho @ (1j H - 0.5 sum L^dag L)
            + sum(L @ rho @ L^dag)

* vectorized (``vectorized=True``, ``:325-327``): ``slindbladian(H, Ls) @ vec(rho)``
  with column-stacking ``vec`` (``dynamiqs/utils/vectorization.py:25-58,213-259``).

Sparse-DIA storage (``dynamiqs/qarrays/sparsedia_dataarray.py:42-71``,
``sparsedia_primitives.py:11-15``): a static tuple ``offsets`` and ``diags`` of shape
``(..., ndiags, n)``, column-indexed: for offset k, ``diags[d, j] = A[j - k, j]``;
entries whose row falls outside ``[0, n)`` must be zero (k >= 0: the first k entries;
k < 0: the last |k| entries).
"""

from __future__ import annotations

import numpy as np

# --------------------------------------------------------------------------------------
# dense helpers
# --------------------------------------------------------------------------------------


def dag(x: np.ndarray) -> np.ndarray:
    return np.conj(np.swapaxes(x, -1, -2))


def hnh_dense(H: np.ndarray, Ls: list[np.ndarray]) -> np.ndarray:
    """Hnh = -iH - 1/2 sum_k L_k^dag L_k (``diffrax_integrator.py:321``)."""
    out = -1j * H
    for L in Ls:
        out = out - 0.5 * (dag(L) @ L)
    return out.astype(H.dtype)


def vf_hermitian(H: np.ndarray, Ls: list[np.ndarray], rho: np.ndarray) -> np.ndarray:
    """``vector_field_unvec_hermitian`` (``diffrax_integrator.py:319-323``)."""
    Hnh = hnh_dense(H, Ls)
    tmp = Hnh @ rho
    for L in Ls:
        tmp = tmp + 0.5 * (L @ rho @ dag(L))
    return (tmp + dag(tmp)).astype(rho.dtype)


def vf_standard(H: np.ndarray, Ls: list[np.ndarray], rho: np.ndarray) -> np.ndarray:
    """``vector_field_unvec_standard`` (``diffrax_integrator.py:312-317``)."""
    half = sum(0.5 * (dag(L) @ L) for L in Ls) if Ls else 0.0 * H
    out = (-1j * H - half) @ rho + rho @ (1j * H - half)
    for L in Ls:
        out = out + L @ rho @ dag(L)
    return out.astype(rho.dtype)


def vectorize(x: np.ndarray) -> np.ndarray:
    """Column-stacking vec: (..., n, n) -> (..., n^2, 1) (``vectorization.py:25-58``)."""
    n = x.shape[-1]
    return np.swapaxes(x, -1, -2).reshape(*x.shape[:-2], n * n, 1)


def unvectorize(x: np.ndarray) -> np.ndarray:
    """Inverse of ``vectorize`` (``vectorization.py:61-97``)."""
    n = int(round(np.sqrt(x.shape[-2])))
    return np.swapaxes(x.reshape(*x.shape[:-2], n, n), -1, -2)


def spre(x: np.ndarray) -> np.ndarray:
    """Superoperator of left multiplication: vec(X rho) = spre(X) vec(rho)."""
    n = x.shape[-1]
    return np.kron(np.eye(n, dtype=x.dtype), x)


def spost(x: np.ndarray) -> np.ndarray:
    """Superoperator of right multiplication: vec(rho X) = spost(X) vec(rho)."""
    n = x.shape[-1]
    return np.kron(x.T, np.eye(n, dtype=x.dtype))


def slindbladian(H: np.ndarray, Ls: list[np.ndarray]) -> np.ndarray:
    """Lindbladian superoperator (``vectorization.py:213-259``)."""
    out = -1j * (spre(H) - spost(H))
    for L in Ls:
        LdL = dag(L) @ L
        out = out + spre(L) @ spost(dag(L)) - 0.5 * spre(LdL) - 0.5 * spost(LdL)
    return out


def vf_vectorized(H, Ls, rho_vec):
    return slindbladian(H, Ls) @ rho_vec


def expect(E: np.ndarray, rho: np.ndarray) -> np.ndarray:
    """tr(E rho) as ``(E * rho.mT).sum((-2, -1))`` (``dynamiqs/utils/general.py:241-276``)."""
    return (E * np.swapaxes(rho, -1, -2)).sum((-2, -1))


# --------------------------------------------------------------------------------------
# sparse-DIA primitives (``dynamiqs/qarrays/sparsedia_primitives.py``)
# --------------------------------------------------------------------------------------


def _sl(offset: int) -> slice:
    """Non-zero slice of a stored diagonal (``sparsedia_primitives.py:11-15``)."""
    return slice(offset, None) if offset >= 0 else slice(None, offset)


def dia_to_dense(offsets, diags: np.ndarray) -> np.ndarray:
    """``sparsedia_to_array`` (``sparsedia_primitives.py:123-127``)."""
    n = diags.shape[-1]
    out = np.zeros((*diags.shape[:-2], n, n), dtype=diags.dtype)
    for d, k in enumerate(offsets):
        cols = np.arange(max(k, 0), n + min(k, 0))
        out[..., cols - k, cols] = diags[..., d, cols]
    return out


def dense_to_dia(x: np.ndarray, offsets=None):
    """Extract the diagonals of ``x`` (all non-zero ones when ``offsets`` is None)."""
    n = x.shape[-1]
    if offsets is None:
        offsets = tuple(k for k in range(-(n - 1), n)
                        if np.any(np.diagonal(x, offset=k, axis1=-2, axis2=-1) != 0))
    diags = np.zeros((*x.shape[:-2], len(offsets), n), dtype=x.dtype)
    for d, k in enumerate(offsets):
        diags[..., d, _sl(k)] = np.diagonal(x, offset=k, axis1=-2, axis2=-1)
    return tuple(int(k) for k in offsets), diags


def dia_transpose(offsets, diags):
    """``transpose_sparsedia`` (``sparsedia_primitives.py:18-29``)."""
    out = np.zeros_like(diags)
    for d, k in enumerate(offsets):
        out[..., d, _sl(-k)] = diags[..., d, _sl(k)]
    return tuple(-k for k in offsets), out


def dia_dag(offsets, diags):
    o, d = dia_transpose(offsets, diags)
    return o, np.conj(d)


def dia_add(lo, ld, ro, rd):
    """``add_sparsedia_sparsedia`` (``sparsedia_primitives.py:172-196``)."""
    out_offsets = tuple(int(k) for k in np.union1d(lo, ro))
    shape = (*np.broadcast_shapes(ld.shape[:-2], rd.shape[:-2]), len(out_offsets),
             ld.shape[-1])
    out = np.zeros(shape, dtype=np.promote_types(ld.dtype, rd.dtype))
    for i, k in enumerate(out_offsets):
        if k in lo:
            out[..., i, :] += ld[..., list(lo).index(k), :]
        if k in ro:
            out[..., i, :] += rd[..., list(ro).index(k), :]
    return out_offsets, out


def dia_matmul_dia(lo, ld, ro, rd):
    """``matmul_sparsedia_sparsedia`` (``sparsedia_primitives.py:199-229``)."""
    n = ld.shape[-1]
    batch = np.broadcast_shapes(ld.shape[:-2], rd.shape[:-2])
    dtype = np.promote_types(ld.dtype, rd.dtype)
    acc: dict[int, np.ndarray] = {}
    for i, lk in enumerate(lo):
        for j, rk in enumerate(ro):
            k = lk + rk
            if abs(k) > n - 1:
                continue
            rs = _sl(rk)
            diag = ld[..., i, _sl(-rk)] * rd[..., j, rs]
            if k not in acc:
                acc[k] = np.zeros((*batch, n), dtype=dtype)
            acc[k][..., rs] += diag
    out_offsets = tuple(sorted(acc))
    if not out_offsets:
        return (), np.zeros((*batch, 0, n), dtype=dtype)
    return out_offsets, np.stack([acc[k] for k in out_offsets], axis=-2)


def dia_matmul_dense(offsets, diags, x):
    """``matmul_sparsedia_array`` (``sparsedia_primitives.py:232-245``)."""
    shape = (*np.broadcast_shapes(diags.shape[:-2], x.shape[:-2]), diags.shape[-1],
             x.shape[-1])
    out = np.zeros(shape, dtype=np.promote_types(diags.dtype, x.dtype))
    for d, k in enumerate(offsets):
        sin, sout = _sl(k), _sl(-k)
        out[..., sout, :] += diags[..., d, sin, None] * x[..., sin, :]
    return out


def dense_matmul_dia(x, offsets, diags):
    """``matmul_array_sparsedia`` (``sparsedia_primitives.py:248-261``)."""
    shape = (*np.broadcast_shapes(x.shape[:-2], diags.shape[:-2]), x.shape[-2],
             diags.shape[-1])
    out = np.zeros(shape, dtype=np.promote_types(x.dtype, diags.dtype))
    for d, k in enumerate(offsets):
        sin, sout = _sl(k), _sl(-k)
        out[..., :, sin] += x[..., :, sout] * diags[..., d, None, sin]
    return out


def hnh_dia(H, Ls):
    """H_nh = -iH - 1/2 sum L^dag L in DIA form; ``H`` and each ``L`` are
    ``(offsets, diags)`` pairs."""
    ho, hd = H
    out = (tuple(ho), (-1j * hd).astype(hd.dtype))
    for lo, ld in Ls:
        do, dd = dia_dag(lo, ld)
        po, pd = dia_matmul_dia(do, dd, lo, ld)
        out = dia_add(out[0], out[1], po, (-0.5 * pd).astype(pd.dtype))
    return out


def vf_hermitian_dia(H, Ls, rho):
    """The hermitian vector field with DIA operators and dense ``rho``; products
    dispatch as in ``QArray.__matmul__`` (``dynamiqs/qarrays/qarray.py:555-586``):
    DIA @ dense -> ``matmul_sparsedia_array``, dense @ DIA ->
    ``matmul_array_sparsedia``."""
    ho, hd = hnh_dia(H, Ls)
    tmp = dia_matmul_dense(ho, hd, rho)
    for lo, ld in Ls:
        do, dd = dia_dag(lo, ld)
        tmp = tmp + 0.5 * dense_matmul_dia(dia_matmul_dense(lo, ld, rho), do, dd)
    return (tmp + dag(tmp)).astype(rho.dtype)
