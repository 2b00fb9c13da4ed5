"""GPU parity of the dense GEMM path for n > 64 (``dqb_lindblad_rhs_dense_large``,
``dqb_mesolve_dense_large``) against the oracle, and against the shared-memory kernel
at n <= 64.  Bars as in test_gpu_dense."""

import numpy as np
import pytest
import torch

import dynamiqs_b200 as dq
from dynamiqs_b200 import _lib, workloads
from dynamiqs_b200.mesolve import MESolveB200Integrator, make_batch_plan
from oracle import lindblad as lb
from oracle.mesolve import mesolve as oracle_mesolve
from tests.parity import assert_solve_parity
from tests.systems import random_problem

pytestmark = pytest.mark.gpu


def rel_frob(x, ref):
    return np.linalg.norm(np.asarray(x) - ref, axis=(-2, -1)) / np.maximum(
        np.linalg.norm(ref, axis=(-2, -1)), 1e-30)


@pytest.mark.parametrize('n', [65, 100, 256])
@pytest.mark.parametrize('K', [0, 1, 3, 5])
@pytest.mark.parametrize('form', [_lib.FORM_HERMITIAN, _lib.FORM_STANDARD])
def test_rhs_large_matches_oracle(cuda_device, n, K, form):
    B = 2
    Hs, Lsets, rhos = [], [], []
    for b in range(B):
        H, Ls, rho = random_problem(n, K, seed=100 * n + 10 * K + b,
                                    hermitian_rho=form == _lib.FORM_HERMITIAN)
        Hs.append(H)
        Lsets.append(np.stack(Ls) if K else np.zeros((0, n, n), np.complex64))
        rhos.append(rho)
    dev = 'cuda'
    # the C ABI reads raw row-major buffers: make every input C-contiguous
    H_d = torch.from_numpy(np.ascontiguousarray(np.stack(Hs))).to(dev)
    L_d = torch.from_numpy(np.ascontiguousarray(np.stack(Lsets))).to(dev)
    r_d = torch.from_numpy(np.ascontiguousarray(np.stack(rhos))).to(dev)
    out = torch.empty_like(r_d)
    lib = _lib.load()
    wsb = lib.dqb_mesolve_dense_large_workspace_size(n, K, 0, 1, B)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    prob = _lib.DenseProblem(n=n, n_jumps=K, batch=B, H=H_d.data_ptr(), L=L_d.data_ptr())
    _lib.check(lib.dqb_lindblad_rhs_dense_large(prob, form, r_d.data_ptr(), out.data_ptr(),
                                                 ws.data_ptr(), wsb,
                                                 torch.cuda.current_stream().cuda_stream), 'rhs')
    got = out.cpu().numpy()
    for b in range(B):
        Hc = Hs[b].astype(complex)
        Lc = [L.astype(complex) for L in Lsets[b]]
        rc = rhos[b].astype(complex)
        ref = lb.vf_hermitian(Hc, Lc, rc) if form == _lib.FORM_HERMITIAN else lb.vf_standard(Hc, Lc, rc)
        assert rel_frob(got[b], ref) < 3e-6


def _check_vs_oracle(res, H, Ls, rho0, ts, Es, method, b=None):
    st = res.states if b is None else res.states[b]
    ex = None if not Es else (res.expects if b is None else res.expects[b]).cpu().numpy()
    ns = int(res.infos.nsteps if b is None else res.infos.nsteps[b])
    return assert_solve_parity(st.cpu().numpy(), ex, ns, H, Ls, rho0, ts, Es,
                               type(method).__name__, method.rtol, method.atol)


def test_transmon_cavity_small_vs_oracle(cuda_device):
    """Transmon(2) x cavity(40): n = 80 through the GEMM path, 3 instances."""
    w = workloads.transmon_cavity(batch=3, nq=2, nc=40, seed=1)
    ts = np.linspace(0.0, 5.0, 11)
    res = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, exp_ops=w['exp_ops'], method=w['method'])
    assert res.states.shape == (3, 11, 80, 80)
    for b in range(3):
        _check_vs_oracle(res, w['H'][b], w['jump_ops'], w['rho0'], ts, w['exp_ops'], w['method'], b)


def test_transmon_cavity_full_dim_short_horizon(cuda_device):
    """n = 256 (transmon 4 x cavity 64), 2 instances, t in [0, 2]."""
    w = workloads.transmon_cavity(batch=2, seed=3)
    ts = np.linspace(0.0, 2.0, 5)
    res = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, exp_ops=w['exp_ops'], method=w['method'])
    _check_vs_oracle(res, w['H'][0], w['jump_ops'], w['rho0'], ts, w['exp_ops'], w['method'], 0)


def test_large_path_equals_small_kernel_at_n48(cuda_device):
    H, Ls, rho = random_problem(48, 2, seed=9)
    ts = np.linspace(0, 2.0, 6)
    small = dq.mesolve(H, Ls, rho, ts)
    plan = make_batch_plan(H, Ls, rho, True)
    integ = MESolveB200Integrator(ts=ts, y0=rho, method=dq.Tsit5(), gradient=None,
                                  options=dq.Options(), H=H, Ls=Ls, Es=None, plan=plan)
    large = integ._run_dense_large(_lib.load())
    assert rel_frob(large.states.cpu().numpy(), small.states.cpu().numpy()).max() < 1e-5
    assert abs(int(large.infos.nsteps) - int(small.infos.nsteps)) <= 1


def test_large_standard_form_and_save_states_false(cuda_device):
    H, Ls, rho = random_problem(90, 3, seed=12, hermitian_rho=False)
    ts = np.linspace(0, 1.0, 4)
    res = dq.mesolve(H, Ls, rho, ts, options=dq.Options(assume_hermitian=False))
    r = oracle_mesolve(H, Ls, rho, ts, form='standard')
    assert rel_frob(res.states.cpu().numpy(), r.states).max() < 1e-5
    last = dq.mesolve(H, Ls, rho, ts, options=dq.Options(assume_hermitian=False, save_states=False))
    assert last.states.shape == (1, 90, 90)
    assert rel_frob(last.states[0].cpu().numpy(), r.states[-1]) < 1e-5


def test_large_path_dopri5_vs_oracle(cuda_device):
    """Dopri5 (its tableau, embedded error and Shampine dense output) through the GEMM
    path: transmon(2) x cavity(40), n = 80, 2 instances."""
    w = workloads.transmon_cavity(batch=2, nq=2, nc=40, seed=4)
    ts = np.linspace(0.0, 3.0, 7)
    m = dq.Dopri5(rtol=1e-6, atol=1e-8)
    res = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, exp_ops=w['exp_ops'], method=m)
    for b in range(2):
        _check_vs_oracle(res, w['H'][b], w['jump_ops'], w['rho0'], ts, w['exp_ops'], m, b)


def test_transmon_full_size_full_horizon(cuda_device):
    """The transmon x cavity workload at its size (n = 256, two instances) over its whole
    horizon t in [0, 20] with 41 saves, in 3xTF32 tensor-core arithmetic (the benchmark's
    precision); instance 0 against the oracle under the bar of tests/parity.py, instance 1
    checked for trace and hermiticity of every saved state."""
    w = workloads.transmon_cavity(batch=2, seed=0)
    res = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], w['tsave'], exp_ops=w['exp_ops'],
                     method=w['method'], options=dq.Options(precision='tf32x3'))
    assert res.states.shape == (2, 41, 256, 256)
    _check_vs_oracle(res, w['H'][0], w['jump_ops'], w['rho0'], w['tsave'], w['exp_ops'],
                     w['method'], 0)
    st = res.states[1]
    tr = torch.diagonal(st, dim1=-2, dim2=-1).sum(-1)
    assert float((tr - 1).abs().max()) < 1e-5
    assert float((st - st.conj().transpose(-1, -2)).abs().max()) < 1e-6


@pytest.mark.parametrize('precision', ['fp32', 'tf32x3'])
@pytest.mark.parametrize('method', ['Tsit5', 'Dopri5'])
def test_large_path_krylov_stepper_vs_oracle(cuda_device, precision, method):
    """The Krylov form of the step on the GEMM path (Options(stepper='krylov')):
    transmon(2) x cavity(40), n = 80, 3 instances, against the oracle under the parity bar,
    and against the stage form (step counts within two)."""
    w = workloads.transmon_cavity(batch=3, nq=2, nc=40, seed=1)
    ts = np.linspace(0.0, 5.0, 11)
    m = (dq.Tsit5 if method == 'Tsit5' else dq.Dopri5)(rtol=1e-6, atol=1e-8)
    res = {}
    for stepper in ('krylov', 'stages'):
        res[stepper] = dq.mesolve(w['H'], w['jump_ops'], w['rho0'], ts, exp_ops=w['exp_ops'],
                                  method=m, options=dq.Options(stepper=stepper, precision=precision))
    kr = res['krylov']
    for b in range(3):
        _check_vs_oracle(kr, w['H'][b], w['jump_ops'], w['rho0'], ts, w['exp_ops'], m, b)
    dn = np.abs(kr.infos.nsteps.cpu().numpy() - res['stages'].infos.nsteps.cpu().numpy())
    assert dn.max() <= 2


def test_large_path_krylov_standard_form(cuda_device):
    """The Krylov form on the GEMM path in the standard form (a non-hermitian rho0, FP32
    products): n = 90, three jumps, against the oracle's standard form."""
    H, Ls, rho = random_problem(90, 3, seed=21, hermitian_rho=False)
    ts = np.linspace(0, 1.0, 5)
    res = dq.mesolve(H, Ls, rho, ts, options=dq.Options(assume_hermitian=False, stepper='krylov'))
    m = dq.Tsit5()
    assert_solve_parity(res.states.cpu().numpy(), None, int(res.infos.nsteps), H, Ls, rho, ts,
                        None, 'Tsit5', m.rtol, m.atol, form='standard')
