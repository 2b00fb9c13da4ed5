"""GPU parity of the tensor-core (tcgen05) products of the dense GEMM path.

The right-hand side through ``dqb_lindblad_rhs_dense_large_prec`` is compared with the
oracle's hermitian vector field (complex128) for every precision mode, and full solves in
3xTF32 / 3xBF16 are compared with the oracle and with the FP32 CUDA-core path.  Bars:
3xTF32 1e-5 on a right-hand side and 1e-5 on solves (the FP32 CUDA-core path reaches
~1e-6 on the same right-hand sides: the tensor core's FP32 accumulation loses a few bits
more than FMA round-to-nearest over a 2n-long real contraction); 3xBF16 1e-4 on a
right-hand side (its products carry ~2^-17 relative error) and 1e-4 on solves; single-pass
TF32 3e-3.
"""

import numpy as np
import pytest
import torch

import dynamiqs_b200 as dq
from dynamiqs_b200 import _lib, workloads
from oracle import lindblad as lb
from oracle.mesolve import mesolve as oracle_mesolve
from tests.systems import random_problem

pytestmark = pytest.mark.gpu

RHS_TOL = {'tf32x3': 1e-5, 'bf16x3': 1e-4, 'tf32': 3e-3, 'fp32': 3e-6}


def rel_frob(x, ref):
    return np.linalg.norm(np.asarray(x) - ref, axis=(-2, -1)) / np.maximum(
        np.linalg.norm(ref, axis=(-2, -1)), 1e-30)


def _rhs(n, K, prec, B=2, seed=0):
    Hs, Lsets, rhos = [], [], []
    for b in range(B):
        H, Ls, rho = random_problem(n, K, seed=seed + 1000 * n + 10 * K + b)
        Hs.append(H)
        Lsets.append(np.stack(Ls) if K else np.zeros((0, n, n), np.complex64))
        rhos.append(rho)
    dev = 'cuda'
    H_d = torch.from_numpy(np.ascontiguousarray(np.stack(Hs))).to(dev)
    L_d = torch.from_numpy(np.ascontiguousarray(np.stack(Lsets))).to(dev)
    r_d = torch.from_numpy(np.ascontiguousarray(np.stack(rhos))).to(dev)
    out = torch.full_like(r_d, float('nan'))
    lib = _lib.load()
    wsb = lib.dqb_mesolve_dense_large_workspace_size(n, K, 0, 1, B)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    prob = _lib.DenseProblem(n=n, n_jumps=K, batch=B, H=H_d.data_ptr(), L=L_d.data_ptr())
    _lib.check(lib.dqb_lindblad_rhs_dense_large_prec(prob, _lib.FORM_HERMITIAN, _lib.PRECISIONS[prec],
                                                      r_d.data_ptr(), out.data_ptr(), ws.data_ptr(), wsb,
                                                      torch.cuda.current_stream().cuda_stream), 'rhs')
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    errs = []
    for b in range(B):
        ref = lb.vf_hermitian(Hs[b].astype(complex), [L.astype(complex) for L in Lsets[b]],
                              rhos[b].astype(complex))
        errs.append(rel_frob(got[b], ref))
    print(f'rhs n={n} K={K} {prec}: max rel Frobenius error {max(errs):.3e}')
    return max(errs)


@pytest.mark.parametrize('prec', ['tf32x3', 'bf16x3', 'tf32', 'fp32'])
@pytest.mark.parametrize('n', [128, 256])
@pytest.mark.parametrize('K', [0, 2])
def test_rhs_tc_matches_oracle(cuda_device, prec, n, K):
    assert _rhs(n, K, prec) < RHS_TOL[prec]


@pytest.mark.parametrize('n,K', [(66, 1), (200, 3), (130, 5)])
@pytest.mark.parametrize('prec', ['tf32x3', 'bf16x3'])
def test_rhs_tc_ragged_tiles_and_long_sums(cuda_device, n, K, prec):
    """n not a multiple of the 128 x 128 tile or of the contraction stage; K = 5 sums
    Hnh X + 5 T_k L_k^+ over two accumulating launches."""
    assert _rhs(n, K, prec) < RHS_TOL[prec]


def test_rhs_tc_rejects_standard_form_and_odd_n(cuda_device):
    lib = _lib.load()
    n, K, B = 129, 1, 1
    H, Ls, rho = random_problem(n, K, seed=1)
    H_d = torch.from_numpy(H).cuda()
    L_d = torch.from_numpy(np.stack(Ls)).cuda()
    r_d = torch.from_numpy(rho).cuda()
    out = torch.empty_like(r_d)
    wsb = lib.dqb_mesolve_dense_large_workspace_size(n, K, 0, 1, B)
    ws = torch.empty(wsb, dtype=torch.uint8, device='cuda')
    prob = _lib.DenseProblem(n=n, n_jumps=K, batch=B, H=H_d.data_ptr(), L=L_d.data_ptr())
    s = torch.cuda.current_stream().cuda_stream
    rc = lib.dqb_lindblad_rhs_dense_large_prec(prob, _lib.FORM_HERMITIAN, _lib.PREC_TF32X3, r_d.data_ptr(),
                                               out.data_ptr(), ws.data_ptr(), wsb, s)
    assert rc == _lib.DQB_ERR_UNSUPPORTED
    prob.n = 128
    rc = lib.dqb_lindblad_rhs_dense_large_prec(prob, _lib.FORM_STANDARD, _lib.PREC_BF16X3, r_d.data_ptr(),
                                               out.data_ptr(), ws.data_ptr(), wsb, s)
    assert rc == _lib.DQB_ERR_UNSUPPORTED
    rc = lib.dqb_lindblad_rhs_dense_large_prec(prob, _lib.FORM_HERMITIAN, 7, r_d.data_ptr(),
                                               out.data_ptr(), ws.data_ptr(), wsb, s)
    assert rc == _lib.DQB_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize('prec,tol', [('tf32x3', 1e-5), ('bf16x3', 1e-4)])
def test_solve_tc_transmon_cavity(cuda_device, prec, tol):
    """Transmon(2) x cavity(64): n = 128, 3 instances, t in [0, 4]: tensor-core solve vs
    the oracle (complex128 state) and vs the FP32 CUDA-core solve."""
    w = workloads.transmon_cavity(batch=3, nq=2, nc=64, seed=5)
    ts = np.linspace(0.0, 4.0, 9)
    kw = dict(exp_ops=w['exp_ops'], method=w['method'])
    tc = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, options=dq.Options(precision=prec), **kw)
    fp = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, **kw)
    assert int((tc.infos.nsteps > 0).sum()) == 3
    got = tc.states.cpu().numpy()
    e_fp = rel_frob(got, fp.states.cpu().numpy()).max()
    print(f'solve {prec}: vs FP32 path {e_fp:.3e}, steps {tc.infos.nsteps.tolist()} vs '
          f'{fp.infos.nsteps.tolist()}')
    assert e_fp < tol
    for b in range(3):
        r = oracle_mesolve(w['H'][b], w['jump_ops'], w['rho0'], ts, exp_ops=w['exp_ops'],
                           rtol=w['method'].rtol, atol=w['method'].atol)
        e_or = rel_frob(got[b], r.states).max()
        e_fo = rel_frob(fp.states[b].cpu().numpy(), r.states).max()
        eerr = np.abs(tc.expects[b].cpu().numpy() - r.expects) / np.maximum(np.abs(r.expects), 1.0)
        print(f'  instance {b}: {prec} vs oracle {e_or:.3e} (FP32 path {e_fo:.3e}), expects {eerr.max():.3e}')
        assert e_or < tol
        assert eerr.max() < tol


def test_solve_tc_full_dim_short_horizon(cuda_device):
    """n = 256 (transmon 4 x cavity 64), 2 instances, t in [0, 1], 3xTF32 vs FP32 path."""
    w = workloads.transmon_cavity(batch=2, seed=3)
    ts = np.linspace(0.0, 1.0, 3)
    kw = dict(exp_ops=w['exp_ops'], method=w['method'])
    tc = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, options=dq.Options(precision='tf32x3'), **kw)
    fp = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, **kw)
    assert rel_frob(tc.states.cpu().numpy(), fp.states.cpu().numpy()).max() < 1e-5
    assert np.abs(tc.infos.nsteps.cpu().numpy() - fp.infos.nsteps.cpu().numpy()).max() <= 1


def test_solve_auto_precision_picks_a_qualified_mode(cuda_device, tmp_path, monkeypatch):
    """precision='auto': the autotuner picks FP32 or 3xTF32 (the modes that meet 1e-5) for
    this (n, K, batch), caches it, and the solve matches the FP32 path within 1e-5."""
    from dynamiqs_b200 import autotune
    from dynamiqs_b200.mesolve import MESolveB200Integrator, make_batch_plan

    monkeypatch.setenv('DQB_AUTOTUNE_CACHE', str(tmp_path / 'tune.json'))
    autotune.clear_memory_cache()
    w = workloads.transmon_cavity(batch=4, nq=2, nc=64, seed=7)
    ts = np.linspace(0.0, 1.0, 3)
    opts = dq.Options(precision='auto')
    plan = make_batch_plan(w['H'], w['jump_ops'], w['rho0'], True)
    integ = MESolveB200Integrator(ts=ts, y0=w['rho0'], method=w['method'], gradient=None,
                                  options=opts, H=w['H'], Ls=w['jump_ops'], Es=w['exp_ops'],
                                  plan=plan)
    res = integ.prepare().launch().result()
    assert integ._tuned['precision'] in (_lib.PREC_FP32, _lib.PREC_TF32X3)
    assert (tmp_path / 'tune.json').exists()
    fp = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, exp_ops=w['exp_ops'], method=w['method'])
    assert rel_frob(res.states.cpu().numpy(), fp.states.cpu().numpy()).max() < 1e-5
    autotune.clear_memory_cache()
