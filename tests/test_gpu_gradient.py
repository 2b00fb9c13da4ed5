"""Gradients through the GPU solve (``torch.autograd`` over the adjoint kernel,
``dqb_mesolve_dense_adjoint``), as the reference tests them
(``tests/mesolve/test_adaptive.py::test_gradient``, ``tests/integrator_tester.py:50-110``):
the analytic gradients of the ``OCavity`` system (``tests/systems/open_system.py:
96-130``) with respect to delta, alpha0 and kappa, for a loss on the final state and on
the final expectation values, at the reference's tolerances (rtol 1e-3, atol 1e-4), for
every gradient option; and a random system against central finite differences of a tight
FP64 solution."""

import numpy as np
import pytest
import torch

import dynamiqs_b200 as dq
from dynamiqs_b200 import operators as ops
from oracle.mesolve import mesolve as oracle_mesolve

pytestmark = pytest.mark.gpu

N = 8
TS = np.linspace(0.0, 0.3, 11)
DELTA, ALPHA0, KAPPA = 2 * np.pi, 0.5, 2 * np.pi


def _ocavity(delta, alpha0, kappa):
    a = torch.as_tensor(ops.destroy(N, layout='dense'), dtype=torch.complex128)
    ad = a.conj().T
    H = delta.to(torch.complex128) * (ad @ a)
    L = torch.sqrt(kappa).to(torch.complex128) * a
    D = torch.linalg.matrix_exp(alpha0.to(torch.complex128) * (ad - a))
    psi0 = D[:, :1]
    c = torch.complex64
    return H.to(c), [L.to(c)], psi0.to(c), [(a + ad).to(c) * 0.5, (1j * (ad - a)).to(c) * 0.5]


def _params():
    return [torch.tensor(v, dtype=torch.float64, requires_grad=True) for v in (DELTA, ALPHA0, KAPPA)]


@pytest.mark.parametrize('gradient', [dq.gradient.Direct(), dq.gradient.BackwardCheckpointed(),
                                      dq.gradient.Forward()], ids=lambda g: type(g).__name__)
def test_ocavity_state_gradient(cuda_device, gradient):
    p = _params()
    H, Ls, psi0, Es = _ocavity(*p)
    res = dq.mesolve(H, Ls, psi0, TS, gradient=gradient)
    num = torch.as_tensor(ops.number(N, layout='dense')).to(res.states.device)
    loss = torch.einsum('ij,ji->', num, res.states[-1]).real
    loss.backward()
    T = TS[-1]
    true = [0.0, 2 * ALPHA0 * np.exp(-KAPPA * T), -(ALPHA0 ** 2) * T * np.exp(-KAPPA * T)]
    got = [float(x.grad) for x in p]
    np.testing.assert_allclose(got, true, rtol=1e-3, atol=1e-4)


def test_ocavity_expect_gradient(cuda_device):
    """Loss on the final expectation values <x> and <p> (one gradient per output, through
    their sum with weights 1 and -0.5)."""
    p = _params()
    H, Ls, psi0, Es = _ocavity(*p)
    res = dq.mesolve(H, Ls, psi0, TS, exp_ops=Es)
    loss = res.expects[0, -1].real - 0.5 * res.expects[1, -1].real
    loss.backward()
    T = TS[-1]
    c, s, e = np.cos(DELTA * T), np.sin(DELTA * T), np.exp(-0.5 * KAPPA * T)
    gx = [-ALPHA0 * T * s * e, c * e, -0.5 * ALPHA0 * T * c * e]
    gp = [-ALPHA0 * T * c * e, -s * e, 0.5 * ALPHA0 * T * s * e]
    true = [gx[i] - 0.5 * gp[i] for i in range(3)]
    np.testing.assert_allclose([float(x.grad) for x in p], true, rtol=1e-3, atol=1e-4)


def test_random_system_vs_finite_differences(cuda_device):
    """Dense random H (n = 5) and two jump operators; the gradient of a weighted sum of the
    saved states' populations and coherences with respect to every real parameter of H's
    generator, against central differences of a tight FP64 oracle solve."""
    rng = np.random.default_rng(3)
    n, ts = 5, np.linspace(0.0, 1.0, 6)
    G = [rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)) for _ in range(2)]
    H1, H2 = [(g + g.conj().T) / 4 for g in G]
    Ls = [0.3 * (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))) / np.sqrt(n) for _ in range(2)]
    W = rng.normal(size=(len(ts), n, n)) + 1j * rng.normal(size=(len(ts), n, n))
    rho0 = np.diag(rng.uniform(size=n)).astype(complex)
    rho0 /= np.trace(rho0)

    def loss_np(th):
        r = oracle_mesolve(th[0] * H1 + th[1] * H2, Ls, rho0, ts, rtol=1e-10, atol=1e-12)
        return float(np.real(np.sum(np.conj(W) * r.states)))

    th = np.array([0.7, -1.1])
    eps = 1e-4
    fd = [(loss_np(th + eps * np.eye(2)[i]) - loss_np(th - eps * np.eye(2)[i])) / (2 * eps)
          for i in range(2)]
    tt = torch.tensor(th, dtype=torch.float64, requires_grad=True)
    c = torch.complex64
    H = (tt[0] * torch.as_tensor(H1) + tt[1] * torch.as_tensor(H2)).to(c)
    res = dq.mesolve(H, [torch.as_tensor(L, dtype=c) for L in Ls], torch.as_tensor(rho0, dtype=c), ts)
    loss = torch.sum(torch.conj(torch.as_tensor(W, dtype=c, device=res.states.device)) * res.states).real
    loss.backward()
    np.testing.assert_allclose(tt.grad.numpy(), fd, rtol=2e-3, atol=1e-4)


def test_gradient_wrt_jump_operator_and_rho0(cuda_device):
    """d loss / d L and d loss / d rho0 as complex matrices, against central differences of
    the tight oracle along random complex directions."""
    rng = np.random.default_rng(8)
    n, ts = 4, np.linspace(0.0, 0.8, 5)
    g = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    H = (g + g.conj().T) / 4
    L = 0.4 * (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    Y = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    rho0 = Y @ Y.conj().T
    rho0 /= np.trace(rho0)
    E = np.diag(np.arange(n)).astype(complex)

    def loss_np(Lx, rx):
        r = oracle_mesolve(H, [Lx], rx, ts, exp_ops=[E], rtol=1e-10, atol=1e-12)
        return float(np.real(r.expects[0, -1]) + np.real(np.trace(r.states[2] @ E)))

    c = torch.complex64
    Lt = torch.tensor(L, dtype=c, requires_grad=True)
    rt = torch.tensor(rho0, dtype=c, requires_grad=True)
    res = dq.mesolve(torch.as_tensor(H, dtype=c), [Lt], rt, ts, exp_ops=[E])
    Et = torch.as_tensor(E, dtype=c, device=res.states.device)
    loss = res.expects[0, -1].real + torch.trace(res.states[2] @ Et).real
    loss.backward()
    for grad, which in ((Lt.grad.numpy(), 'L'), (rt.grad.numpy(), 'rho')):
        D = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        if which == 'rho':
            D = D + D.conj().T  # a hermitian direction keeps rho0 a valid input
        eps = 1e-5
        if which == 'L':
            fd = (loss_np(L + eps * D, rho0) - loss_np(L - eps * D, rho0)) / (2 * eps)
        else:
            fd = (loss_np(L, rho0 + eps * D) - loss_np(L, rho0 - eps * D)) / (2 * eps)
        got = float(np.real(np.sum(np.conj(grad) * D)))  # dLoss = Re tr(G^+ D)
        assert abs(got - fd) <= 2e-3 * abs(fd) + 1e-4, (which, got, fd)


def test_gradient_with_batched_jump_operators(cuda_device):
    """Jump operators batched (two decay rates) with a batched H (cartesian: 2 x 2
    instances): the gradient of a loss summed over the batch, with respect to each batched
    operator, equals the sum of the gradients of the single solves that used each item
    (those are checked against finite differences above)."""
    rng = np.random.default_rng(3)
    n, ts = 5, np.linspace(0.0, 0.6, 4)
    c = torch.complex64
    a = torch.as_tensor(ops.destroy(n, layout='dense'), dtype=c)
    E = torch.as_tensor(np.diag(np.arange(n)), dtype=c)
    Hs = []
    for _ in range(2):
        g = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        Hs.append((g + g.conj().T) / 4)
    H = torch.tensor(np.stack(Hs), dtype=c, requires_grad=True)
    kap = torch.tensor([0.2, 0.5], dtype=torch.float32)
    L = (torch.sqrt(kap)[:, None, None].to(c) * a).detach().requires_grad_(True)
    psi0 = torch.as_tensor(ops.fock(n, 1), dtype=c)
    res = dq.mesolve(H, [L], psi0, ts, exp_ops=[E])
    assert res.expects.shape == (2, 2, 1, 4)
    loss = res.expects[..., 0, -1].real.sum()
    loss.backward()
    gL = torch.zeros_like(L)
    gH = torch.zeros_like(H)
    for i in range(2):
        for j in range(2):
            Hi = H.detach()[i].clone().requires_grad_(True)
            Lj = L.detach()[j].clone().requires_grad_(True)
            r = dq.mesolve(Hi, [Lj], psi0, ts, exp_ops=[E])
            r.expects[0, -1].real.backward()
            gL[j] += Lj.grad
            gH[i] += Hi.grad
    np.testing.assert_allclose(L.grad.numpy(), gL.numpy(), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(H.grad.numpy(), gH.numpy(), rtol=1e-5, atol=1e-6)
