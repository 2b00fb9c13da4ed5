"""GPU checks of the tensor-core form of the n <= 64 kernel (``precision='f16x3'``:
tcgen05 products on FP16 hi + lo splits of power-of-two-scaled operands) against the
oracle, through the C ABI (``dqb_lindblad_rhs_dense_prec``, ``dqb_mesolve_dense``) and
the public ``mesolve``.

Single right-hand sides: 2e-6 relative Frobenius error (the CUDA-core kernel's bar).
Solves: the accuracy bar of tests/parity.py (error against a tight FP64 solution at most
twice the oracle's own), not step counts.  FP16 keeps ~38 bits of dynamic range below a
matrix's largest entry, and the entries it flushes -- the far tail of a density matrix,
10^-12 and below -- are ones the reference's complex64 arithmetic still resolves and its
error control (atol 1e-8 on every entry) still sees: on the batched-Kerr workload this mode
accepts larger steps (about 4 % fewer on the benchmark, up to 30 % fewer on short
horizons).  The mode is opt-in for that reason."""

import numpy as np
import pytest
import torch

import dynamiqs_b200 as dq
from dynamiqs_b200 import _lib, workloads
from oracle import lindblad as lb
from tests.parity import assert_accuracy, rel_frob
from tests.systems import random_problem

pytestmark = pytest.mark.gpu


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).to('cuda', torch.complex64)


def _rhs_f16x3(Hs, Lsets, rhos, n, K):
    B = len(Hs)
    H_d, r_d = _dev(np.stack(Hs)), _dev(np.stack(rhos))
    L_d = _dev(np.stack(Lsets)) if K else torch.zeros(1, dtype=torch.complex64, device='cuda')
    out = torch.empty_like(r_d)
    ws = torch.empty(B * 32768, dtype=torch.uint8, device='cuda')
    prob = _lib.DenseProblem(n=n, n_jumps=K, batch=B, H=H_d.data_ptr(), L=L_d.data_ptr())
    lib = _lib.load()
    _lib.check(lib.dqb_lindblad_rhs_dense_prec(prob, _lib.FORM_HERMITIAN, _lib.PREC_F16X3,
                                               r_d.data_ptr(), out.data_ptr(), ws.data_ptr(),
                                               ws.numel(), torch.cuda.current_stream().cuda_stream),
               'rhs f16x3')
    return out.cpu().numpy()


@pytest.mark.parametrize('n', [33, 48, 64])
@pytest.mark.parametrize('K', [0, 1, 2])
@pytest.mark.parametrize('hermitian_rho', [True, False])
def test_rhs_f16x3_matches_oracle(cuda_device, n, K, hermitian_rho):
    """The hermitian form's right-hand side; for a non-hermitian X it still equals the
    reference's tmp + tmp^+ (the kernel's L X^+ L^+ differs from (L X) L^+ by a term that
    the symmetrisation cancels)."""
    B = 3
    rng = np.random.default_rng(1000 + 10 * n + K)
    Hs, Lsets, rhos = [], [], []
    for b in range(B):
        H, Ls, rho = random_problem(n, K, seed=int(rng.integers(1 << 30)), hermitian_rho=hermitian_rho)
        Hs.append(H)
        Lsets.append(np.stack(Ls) if K else np.zeros((0, n, n), np.complex64))
        rhos.append(rho)
    got = _rhs_f16x3(Hs, Lsets, rhos, n, K)
    for b in range(B):
        ref = lb.vf_hermitian(Hs[b].astype(complex), [L.astype(complex) for L in Lsets[b]],
                              rhos[b].astype(complex))
        assert rel_frob(got[b], ref) < 2e-6


def test_rhs_f16x3_kerr_operators(cuda_device):
    """The batched-Kerr operators (largest Hnh entries ~10^3 next to jump entries ~1: the
    per-matrix scales differ by 2^10) on a state with a decaying spectrum."""
    w = workloads.batched_kerr(batch=4, seed=11)
    rng = np.random.default_rng(5)
    rhos = []
    for _ in range(4):
        Y = (rng.normal(size=(64, 64)) + 1j * rng.normal(size=(64, 64))) * np.exp(-np.arange(64) / 4)[:, None]
        X = Y @ Y.conj().T
        rhos.append((X / np.trace(X)).astype(np.complex64))
    Ls = np.stack(w['jump_ops'])
    got = _rhs_f16x3(list(w['H']), [Ls] * 4, rhos, 64, 2)
    for b in range(4):
        ref = lb.vf_hermitian(w['H'][b].astype(complex), [L.astype(complex) for L in Ls],
                              rhos[b].astype(complex))
        assert rel_frob(got[b], ref) < 2e-6


def test_rhs_f16x3_rejects_what_it_does_not_cover(cuda_device):
    lib = _lib.load()
    prob = _lib.DenseProblem(n=64, n_jumps=3, batch=1, H=1, L=1)
    assert lib.dqb_lindblad_rhs_dense_prec(prob, _lib.FORM_HERMITIAN, _lib.PREC_F16X3, 1, 1, 1,
                                           1 << 20, None) == _lib.DQB_ERR_UNSUPPORTED
    prob = _lib.DenseProblem(n=32, n_jumps=1, batch=1, H=1, L=1)
    assert lib.dqb_lindblad_rhs_dense_prec(prob, _lib.FORM_HERMITIAN, _lib.PREC_F16X3, 1, 1, 1,
                                           1 << 20, None) == _lib.DQB_ERR_UNSUPPORTED
    prob = _lib.DenseProblem(n=64, n_jumps=1, batch=2, H=1, L=1)
    assert lib.dqb_lindblad_rhs_dense_prec(prob, _lib.FORM_HERMITIAN, _lib.PREC_F16X3, 1, 1, 1,
                                           32768, None) == _lib.DQB_ERR_WORKSPACE_TOO_SMALL


def test_batched_kerr_subset_f16x3(cuda_device):
    """Batched Kerr (n = 64, two jumps, the benchmark's workload) on three instances,
    including a stiff one (thousands of steps)."""
    w = workloads.batched_kerr(batch=3, seed=7)
    res = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], exp_ops=w['exp_ops'],
                     method=w['method'], options=dq.Options(precision='f16x3'))
    assert res.states.shape == (3, 51, 64, 64)
    m = w['method']
    for b in range(3):
        assert_accuracy(res.states[b].cpu().numpy(), w['H'][b], w['jump_ops'], w['rho0'],
                        w['tsave'], 'Tsit5', m.rtol, m.atol)


@pytest.mark.parametrize('n,K', [(33, 0), (48, 1), (64, 2)])
@pytest.mark.parametrize('method', ['Tsit5', 'Dopri5'])
def test_random_problems_f16x3(cuda_device, n, K, method):
    H, Ls, rho = random_problem(n, K, seed=n + K)
    ts = np.linspace(0, 1.5, 7)
    m = dq.Tsit5() if method == 'Tsit5' else dq.Dopri5()
    res = dq.mesolve(H, Ls, rho, ts, method=m, options=dq.Options(precision='f16x3'))
    assert_accuracy(res.states.cpu().numpy(), H, Ls, rho, ts, method, m.rtol, m.atol)


def test_many_instances_f16x3(cuda_device):
    """More instances than SMs (the persistent kernel takes new ones as CTAs free up):
    every instance finishes with status OK and a trace-one state; a sample of them meets
    the accuracy bar."""
    w = workloads.batched_kerr(batch=300, seed=3)
    ts = np.linspace(0.0, 2.0, 5)
    a = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, method=w['method'],
                   options=dq.Options(precision='f16x3'))
    tr = torch.diagonal(a.states[:, -1], dim1=-2, dim2=-1).sum(-1)
    assert float((tr - 1).abs().max()) < 1e-5
    m = w['method']
    for b in (0, 13, 299):
        assert_accuracy(a.states[b].cpu().numpy(), w['H'][b], w['jump_ops'], w['rho0'], ts,
                        'Tsit5', m.rtol, m.atol)
