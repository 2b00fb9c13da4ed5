"""Host-side logic of the drop-in API: argument checks with the reference's messages,
batching plans (cartesian and flat, mesolve.py:307-336) and the no-fallback rule."""

import numpy as np
import pytest

import dynamiqs_b200 as dq
from dynamiqs_b200 import _lib
from dynamiqs_b200 import operators as ops
from dynamiqs_b200.mesolve import make_batch_plan


def _problem(n=4):
    a = ops.destroy(n, layout='dense')
    return ops.dag(a) @ a, [a], ops.fock(n, 0), np.linspace(0, 1, 5)


def test_check_times_messages():
    H, Ls, r, _ = _problem()
    with pytest.raises(ValueError, match='strictly ascending'):
        dq.mesolve(H, Ls, r, [0.0, 1.0, 0.5])
    with pytest.raises(ValueError, match='1D array'):
        dq.mesolve(H, Ls, r, np.zeros((2, 2)))


def test_shape_messages():
    H, Ls, r, ts = _problem()
    with pytest.raises(ValueError, match=r'Argument `H` must have shape'):
        dq.mesolve(np.zeros((4, 3)), Ls, r, ts)
    with pytest.raises(ValueError, match=r'Argument `jump_ops\[0\]` must have shape'):
        dq.mesolve(H, [np.zeros((4, 3))], r, ts)
    with pytest.raises(ValueError, match=r'Argument `rho0` must have shape'):
        dq.mesolve(H, Ls, np.zeros((4, 3)), ts)
    with pytest.raises(ValueError, match=r'exp_ops\[0\]'):
        dq.mesolve(H, Ls, r, ts, exp_ops=[np.zeros((2, 4, 4))])
    with pytest.raises(ValueError, match='layout `dense`'):
        dq.mesolve(H, Ls, ops.number(4), ts)


def test_options_and_method_checks():
    H, Ls, r, ts = _problem()
    with pytest.raises(ValueError, match='Option `save_propagators`'):
        dq.mesolve(H, Ls, r, ts, options=dq.Options(save_propagators=False))

    class Euler(dq.method.Method):
        pass

    with pytest.raises(TypeError, match='Method of type `Euler` is not supported'):
        dq.mesolve(H, Ls, r, ts, method=Euler())
    with pytest.raises(ValueError, match='does not support gradient `object`'):
        dq.mesolve(H, Ls, r, ts, gradient=object())
    from dynamiqs_b200.mesolve import _stepper_code

    assert _stepper_code(dq.Options()) == _lib.STEPPER_AUTO
    assert _stepper_code(dq.Options(stepper='stages')) == _lib.STEPPER_STAGES
    with pytest.raises(ValueError, match='Option `stepper` must be one of'):
        _stepper_code(dq.Options(stepper='rk4'))
    with pytest.raises(ValueError, match='Option `stepper` was set'):
        dq.sesolve(H, r, ts, options=dq.Options(stepper='stages'))


def test_cartesian_batch_plan():
    n = 3
    H = np.zeros((2, 3, n, n), np.complex64)
    L0 = np.zeros((4, n, n), np.complex64)
    L1 = np.zeros((n, n), np.complex64)
    r = np.zeros((5, n, 1), np.complex64)
    p = make_batch_plan(H, [L0, L1], r, cartesian=True)
    assert p.bshape == (2, 3, 4, 5)
    idx = np.arange(p.batch).reshape(p.bshape + (1,))
    hi, li, ri = (x.reshape(p.bshape) for x in (p.H_index, p.L_index, p.rho_index))
    I = np.indices(p.bshape)
    np.testing.assert_array_equal(hi, I[0] * 3 + I[1])
    np.testing.assert_array_equal(li, I[2])
    np.testing.assert_array_equal(ri, I[3])
    assert p.L_sets.shape == (4, 2, n, n)
    del idx


def test_flat_batch_plan_broadcasts():
    n = 2
    rng = np.random.default_rng(0)
    H = rng.normal(size=(2, 3, n, n)).astype(np.complex64)
    L0 = rng.normal(size=(3, n, n)).astype(np.complex64)
    L1 = rng.normal(size=(2, 1, n, n)).astype(np.complex64)
    r = rng.normal(size=(3, n, n)).astype(np.complex64)
    p = make_batch_plan(H, [L0, L1], r, cartesian=False)
    assert p.bshape == (2, 3)
    for b in range(6):
        i, j = divmod(b, 3)
        np.testing.assert_array_equal(p.H_items[p.H_index[b]], H[i, j])
        np.testing.assert_array_equal(p.L_sets[p.L_index[b], 0], L0[j])
        np.testing.assert_array_equal(p.L_sets[p.L_index[b], 1], L1[i, 0])
        np.testing.assert_array_equal(p.rho_items[p.rho_index[b]], r[j])


def test_no_cpu_fallback(monkeypatch):
    import torch

    monkeypatch.setattr(torch.cuda, 'is_available', lambda: False)
    H, Ls, r, ts = _problem()
    with pytest.raises(RuntimeError, match='no CPU fallback'):
        dq.mesolve(H, Ls, r, ts)


def test_operator_constructors_match_reference_examples():
    # dq.position(3) and dq.displace(4, 0.5) printed in the reference docstrings
    # (dynamiqs/utils/operators.py:586-590, 496-500)
    np.testing.assert_allclose(ops.position(3).to_dense(),
                               [[0, .5, 0], [.5, 0, .70710678], [0, .70710678, 0]], atol=1e-6)
    np.testing.assert_allclose(ops.displace(4, 0.5)[:, 0], [0.882, 0.441, 0.156, 0.047], atol=1e-3)


def test_start_order_is_stiffest_first_permutation():
    """The host's start order for the persistent kernel: a permutation of the instances,
    largest stiffness bound (row-sum norm of H plus 1/2 sum ||L||^2) first."""
    from dynamiqs_b200 import workloads
    from dynamiqs_b200.mesolve import MESolveB200Integrator

    w = workloads.batched_kerr(batch=300, n=16, seed=4)
    plan = make_batch_plan(w['H'], w['jump_ops'], w['rho0'], True)
    integ = MESolveB200Integrator(ts=w['tsave'], y0=w['rho0'], method=w['method'], gradient=None,
                                  options=dq.Options(), H=w['H'], Ls=w['jump_ops'], Es=None,
                                  plan=plan)
    order = integ._start_order()
    assert order.dtype == np.int32 and sorted(order.tolist()) == list(range(300))
    h = np.abs(w['H']).sum(-1).max(-1)
    assert np.all(np.diff(h[order]) <= 1e-6)  # the jump operators are shared: H decides


def test_sesolve_path_selection():
    """sesolve picks its kernel by size and storage: one warp per instance up to n = 128
    (sparse-DIA H densified), then the large-problem stepper with a dense H or with H kept
    in DIA storage; beyond n = 8192 it refuses before touching a GPU."""
    from dynamiqs_b200.mesolve import make_batch_plan
    from dynamiqs_b200.qarrays import SparseDIA
    from dynamiqs_b200.sesolve import SESolveB200Integrator

    def path(H, n):
        psi = np.zeros((n, 1), np.complex64)
        plan = make_batch_plan(H, [], psi, True)
        return SESolveB200Integrator(ts=np.array([0.0, 1.0]), y0=psi, method=dq.Tsit5(),
                                     gradient=None, options=dq.Options(), H=H, Es=None,
                                     plan=plan).path

    assert path(np.eye(64, dtype=np.complex64), 64) == 'warp'
    assert path(np.eye(200, dtype=np.complex64), 200) == 'dense_large'
    assert path(SparseDIA.from_dense(np.eye(200, dtype=np.complex64)), 200) == 'dia'
    big = SparseDIA((0,), np.ones((1, 8193), np.complex64))
    with pytest.raises(NotImplementedError, match='n <= 8192'):
        dq.sesolve(big, np.zeros((8193, 1), np.complex64), [0.0, 1.0])


def test_sesolve_time_dependent_checks_before_the_gpu():
    """A time-dependent sesolve with more than four time-dependent terms, or a callable
    operator, is refused before any device work."""
    a = ops.destroy(4, layout='dense')
    x = a + ops.dag(a)
    H = ops.dag(a) @ a
    for _ in range(5):
        H = H + dq.pwc([0.0, 1.0], [1.0], x)
    with pytest.raises(NotImplementedError, match='At most 4'):
        dq.sesolve(H, ops.fock(4, 0), [0.0, 1.0])


@pytest.mark.parametrize('cartesian', [True, False])
def test_jump_operator_gradients_map_back_to_batched_operators(cartesian):
    """The per-instance jump-operator gradients of the adjoint are summed onto each jump
    operator's own batch shape: every instance adds its gradient to the item of each
    operator that it used (cartesian: each operator's own dimensions of the result; flat:
    the broadcast to the full batch), checked against a brute-force sum over instances."""
    import torch

    from dynamiqs_b200.autodiff import _jump_grads

    n = 3
    rng = np.random.default_rng(0)
    H = rng.normal(size=(2, n, n)).astype(np.complex64)
    if cartesian:
        Ls = [rng.normal(size=(3, n, n)).astype(np.complex64), rng.normal(size=(2, n, n)).astype(np.complex64)]
    else:
        Ls = [rng.normal(size=(2, n, n)).astype(np.complex64), rng.normal(size=(1, n, n)).astype(np.complex64)]
    rho = np.eye(n, dtype=np.complex64)
    plan = make_batch_plan(H, Ls, rho, cartesian)
    B, K = plan.batch, len(Ls)
    grad_L = torch.as_tensor(rng.normal(size=(B, K, n, n)) + 1j * rng.normal(size=(B, K, n, n)),
                             dtype=torch.complex64)
    got = _jump_grads(grad_L, plan, [torch.as_tensor(L) for L in Ls], cartesian, n, 'cpu')
    # brute force: instance b used item idx_k(b) of operator k
    for k, L in enumerate(Ls):
        exp = np.zeros(L.shape, np.complex64)
        items = L.reshape(-1, n, n)
        sets = plan.L_sets[:, k]
        for b in range(B):
            s = plan.L_index[b]
            # the item of operator k inside jump set s
            i = next(j for j in range(items.shape[0]) if np.array_equal(items[j], sets[s]))
            exp.reshape(-1, n, n)[i] += grad_L[b, k].numpy()
        np.testing.assert_allclose(got[k].numpy(), exp, rtol=1e-5, atol=1e-5)


def test_time_dependent_jump_operators_need_one_storage():
    """Time-dependent jump operators run with every operator dense (GEMM path) or every one
    in sparse-DIA storage (DIA stepper); a dense H with a DIA jump operator, or a jump
    operator with batched prefactor values, is refused before any GPU work."""
    a = ops.destroy(6, layout='dense')
    a_dia = ops.destroy(6, layout='dia')
    with pytest.raises(NotImplementedError, match='every operator dense'):
        dq.mesolve(ops.dag(a) @ a, [dq.pwc([0.0, 1.0], [1.0], a_dia)], ops.fock(6, 0), [0.0, 1.0])
    with pytest.raises(NotImplementedError, match='unbatched values'):
        dq.mesolve(ops.dag(a) @ a, [dq.pwc([0.0, 1.0], [[1.0], [0.5]], a)], ops.fock(6, 0),
                   [0.0, 1.0])
