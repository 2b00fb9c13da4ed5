"""Sparse-DIA primitives of the oracle and of the host-side SparseDIA type against dense
arithmetic, in the reference's pattern (tests/qarrays/test_sparse_dia_qarray.py:28-46,
239-240: N=10, offsets (-2, 0, 2) and (-2, -1, 1, 3), random normal diagonals with the
out-of-range entries zeroed, allclose(rtol=1e-5, atol=1e-8))."""

import numpy as np
import pytest

from dynamiqs_b200.qarrays import SparseDIA, kron
from oracle import lindblad as lb

N = 10
OFF_A = (-2, 0, 2)
OFF_B = (-2, -1, 1, 3)


def _rand_diags(offsets, seed):
    rng = np.random.default_rng(seed)
    d = (rng.normal(size=(len(offsets), N)) + 1j * rng.normal(size=(len(offsets), N))).astype(np.complex64)
    for i, k in enumerate(offsets):
        if k >= 0:
            d[i, :k] = 0
        else:
            d[i, N + k:] = 0
    return d


def close(x, y):
    np.testing.assert_allclose(x, y, rtol=1e-5, atol=1e-5)


@pytest.fixture
def AB():
    return (OFF_A, _rand_diags(OFF_A, 42)), (OFF_B, _rand_diags(OFF_B, 43))


def test_to_dense_convention(AB):
    (oa, da), _ = AB
    A = lb.dia_to_dense(oa, da)
    for d, k in enumerate(oa):
        for j in range(N):
            if 0 <= j - k < N:
                assert A[j - k, j] == da[d, j]  # column-indexed storage
    o2, d2 = lb.dense_to_dia(A, oa)
    close(d2, da)


def test_matmul_dia_dense(AB):
    (oa, da), _ = AB
    A = lb.dia_to_dense(oa, da)
    X = np.random.default_rng(0).normal(size=(N, N)).astype(np.complex64)
    close(lb.dia_matmul_dense(oa, da, X), A @ X)
    close(lb.dense_matmul_dia(X, oa, da), X @ A)


def test_matmul_dia_dia_add_transpose(AB):
    (oa, da), (ob, db) = AB
    A, B = lb.dia_to_dense(oa, da), lb.dia_to_dense(ob, db)
    close(lb.dia_to_dense(*lb.dia_matmul_dia(oa, da, ob, db)), A @ B)
    close(lb.dia_to_dense(*lb.dia_add(oa, da, ob, db)), A + B)
    close(lb.dia_to_dense(*lb.dia_transpose(oa, da)), A.T)
    close(lb.dia_to_dense(*lb.dia_dag(oa, da)), A.conj().T)


def test_hnh_and_vector_field(AB):
    (oa, da), (ob, db) = AB
    A, B = lb.dia_to_dense(oa, da), lb.dia_to_dense(ob, db)
    rng = np.random.default_rng(1)
    Y = rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N))
    rho = (Y @ Y.conj().T).astype(np.complex64)
    H = 0.5 * (A + A.conj().T)
    Hd = lb.dense_to_dia(H)
    close(lb.dia_to_dense(*lb.hnh_dia(Hd, [(ob, db)])), lb.hnh_dense(H, [B]))
    close(lb.vf_hermitian_dia(Hd, [(ob, db)], rho), lb.vf_hermitian(H, [B], rho))


def test_vector_field_forms_agree_on_hermitian_rho():
    rng = np.random.default_rng(2)
    n = 6
    X = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    H = X + X.conj().T
    Ls = [rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)) for _ in range(2)]
    Y = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    rho = Y @ Y.conj().T
    f1 = lb.vf_hermitian(H, Ls, rho)
    f2 = lb.vf_standard(H, Ls, rho)
    f3 = lb.unvectorize(lb.vf_vectorized(H, Ls, lb.vectorize(rho)))
    np.testing.assert_allclose(f1, f2, atol=1e-10)
    np.testing.assert_allclose(f3, f2, atol=1e-10)


def test_host_sparsedia_algebra(AB):
    (oa, da), (ob, db) = AB
    A, B = SparseDIA(oa, da), SparseDIA(ob, db)
    close((A @ B).to_dense(), A.to_dense() @ B.to_dense())
    close((A + B).to_dense(), A.to_dense() + B.to_dense())
    close(A.dag().to_dense(), A.to_dense().conj().T)
    close((A * 2.5).to_dense(), 2.5 * A.to_dense())
    close(kron(A, B).to_dense(), np.kron(A.to_dense(), B.to_dense()))


def test_host_sparsedia_rejects_nonzero_padding():
    d = np.ones((1, 4), np.complex64)
    with pytest.raises(ValueError):
        SparseDIA((1,), d)  # first entry of offset 1 must be zero
