"""Reverse-mode derivatives of ``mesolve`` through ``torch.autograd``.

``mesolve`` routes here when ``H``, a jump operator or ``rho0`` is a torch tensor that
requires grad: the forward pass is a taped GPU solve (``dqb_mesolve_dense_taped``, the
same steps and results as ``dqb_mesolve_dense``), the backward pass the adjoint kernel
(``dqb_mesolve_dense_adjoint``) -- the exact derivative of the discrete solve, which is
what the reference's ``Direct`` / ``BackwardCheckpointed`` gradients compute through
diffrax (``dynamiqs/integrators/core/diffrax_integrator.py:88-99``).  Scope: dense
constant operators with n <= 64; ``H``, the jump operators and ``rho0`` may be batched
(cartesian or flat).  The per-instance gradients the kernel writes are summed back onto the
input tensors they came from: over the instances that share an item, and, for a jump
operator, over the batch dimensions it was broadcast along.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

__all__ = ['needs_autograd', 'mesolve_autograd']


def _is_grad_tensor(x) -> bool:
    return getattr(x, 'requires_grad', False)


def needs_autograd(H, jump_ops, rho0) -> bool:
    import torch

    return torch.is_grad_enabled() and (
        _is_grad_tensor(H) or _is_grad_tensor(rho0) or any(_is_grad_tensor(L) for L in jump_ops))


def _solve_taped(integ, lib):
    """Taped solve: a first solve tells how many steps each instance accepts, the second
    (the same deterministic kernel) records them."""
    import torch

    prep = integ._prepare_dense(lib, 'small')
    prep.launch()
    cap = max(int(prep.bufs['infos'][:, 1].max().item()), 1)
    B = integ.plan.batch
    n = prep.prob.n
    dev = prep.dev
    tape_t = torch.empty((B, cap), dtype=torch.float64, device=dev)
    tape_h = torch.empty((B, cap), dtype=torch.float64, device=dev)
    tape_y = torch.empty(lib.dqb_mesolve_dense_tape_bytes(n, cap, B), dtype=torch.uint8, device=dev)
    tape = _lib.Tape(t=tape_t.data_ptr(), h=tape_h.data_ptr(), y=tape_y.data_ptr(), capacity=cap)
    rc = lib.dqb_mesolve_dense_taped(prep.prob, integ._ode_options(), prep.outs, tape,
                                     prep.bufs['workspace'].data_ptr(), prep.ws_bytes,
                                     torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(rc, 'dqb_mesolve_dense_taped')
    prep.bufs['tape'] = (tape, tape_t, tape_h, tape_y)
    return prep


def _jump_grads(grad_L, plan, Lts, cartesian, n, dev):
    """Per-instance jump-operator gradients ``grad_L`` (B, K, n, n) summed onto each jump
    operator's own batch shape: first onto the jump sets the instances used (``L_index``),
    then, for operator k, over the dimensions of the set batch that it was broadcast along
    (cartesian: the other operators' dimensions; flat: the broadcast to the full shape)."""
    import torch

    K = len(Lts)
    nsets = plan.L_sets.shape[0]
    lidx = torch.as_tensor(plan.L_index, dtype=torch.long, device=dev)
    gsets = torch.zeros((nsets, max(K, 1), n, n), dtype=grad_L.dtype, device=dev).index_add_(0, lidx, grad_L)
    bs = [tuple(L.shape[:-2]) for L in Lts]
    out = []
    if cartesian:
        lcat = tuple(d for b in bs for d in b)
        pos = 0
        for k, L in enumerate(Lts):
            g = gsets[:, k].reshape(*lcat, n, n)
            keep = set(range(pos, pos + len(bs[k])))
            other = tuple(d for d in range(len(lcat)) if d not in keep)
            if other:
                g = g.sum(dim=other)
            out.append(g.reshape(L.shape).to(L.device, L.dtype))
            pos += len(bs[k])
    else:
        full = tuple(plan.bshape)
        for k, L in enumerate(Lts):
            g = gsets[0, k] if nsets == 1 else gsets[:, k].reshape(*full, n, n).sum_to_size(*L.shape)
            out.append(g.reshape(L.shape).to(L.device, L.dtype))
    return out


def mesolve_autograd(H, jump_ops, rho0, tsave, *, exp_ops, method, gradient, options, integ_cls,
                     make_plan, check):
    """``mesolve`` with ``torch.autograd`` support; returns an ``MESolveResult`` whose
    ``states`` and ``expects`` are differentiable with respect to ``H``, ``jump_ops`` and
    ``rho0``."""
    import torch

    from .mesolve import _as_op

    to_t = lambda x: x if isinstance(x, torch.Tensor) else torch.as_tensor(_as_op(x))  # noqa: E731
    Ht = to_t(H)
    Lts = [to_t(L) for L in jump_ops]
    rt = to_t(rho0)
    H_np, Ls_np, r_np = _as_op(Ht), [_as_op(L) for L in Lts], _as_op(rt)
    Es = [_as_op(E) for E in exp_ops] if exp_ops else None
    check(H_np, Ls_np, r_np, Es)
    plan = make_plan(H_np, Ls_np, r_np, options.cartesian_batching)
    integ = integ_cls(ts=tsave, y0=r_np, method=method, gradient=gradient, options=options,
                      H=H_np, Ls=Ls_np, Es=Es, plan=plan)
    lib = _lib.load()
    n = H_np.shape[-1]
    if n > lib.dqb_dense_small_max_n(len(Ls_np)):
        raise NotImplementedError('Gradients on the B200 path are available for n <= 64.')

    prep = _solve_taped(integ, lib)

    class _Solve(torch.autograd.Function):
        @staticmethod
        def forward(ctx, Hx, rx, *Lx):
            b = prep.bufs
            return b['states'].clone(), b['expects'].clone()

        @staticmethod
        def backward(ctx, g_states, g_expects):
            b = prep.bufs
            dev = prep.dev
            B, K, nn = plan.batch, len(Ls_np), n * n
            c64 = torch.complex64
            gs = None if g_states is None else g_states.to(dev, c64).contiguous()
            ge = None
            if g_expects is not None:
                ge = g_expects.to(dev, c64).clone()
                ge[:, integ._n_user_E:] = 0  # the trace row is not an output of the solve
                ge = ge.contiguous()
            is_ket = r_np.shape[-1] == 1 and n > 1
            grad_r = torch.zeros((B, n) if is_ket else (B, n, n), dtype=c64, device=dev)
            grad_H = torch.zeros((B, n, n), dtype=c64, device=dev)
            grad_L = torch.zeros((B, max(K, 1), n, n), dtype=c64, device=dev)
            ws_bytes = lib.dqb_mesolve_dense_adjoint_workspace_size(n, K, B)
            ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
            cot = _lib.Cotangents(states=None if gs is None else gs.data_ptr(),
                                  expects=None if ge is None else ge.data_ptr())
            grads = _lib.Gradients(rho0=grad_r.data_ptr(), H=grad_H.data_ptr(), L=grad_L.data_ptr())
            nacc = b['infos'][:, 1].contiguous()
            rc = lib.dqb_mesolve_dense_adjoint(prep.prob, integ._ode_options(), b['tape'][0],
                                               ctypes.c_void_p(nacc.data_ptr()), cot, grads,
                                               ws.data_ptr(), ws_bytes,
                                               torch.cuda.current_stream(dev).cuda_stream)
            _lib.check(rc, 'dqb_mesolve_dense_adjoint')
            # sum the per-instance gradients back onto the items they came from
            hidx = torch.as_tensor(plan.H_index, dtype=torch.long, device=dev)
            ridx = torch.as_tensor(plan.rho_index, dtype=torch.long, device=dev)
            gH = torch.zeros((plan.H_items.shape[0], n, n), dtype=c64, device=dev).index_add_(0, hidx, grad_H)
            gr = torch.zeros((plan.rho_items.shape[0], *grad_r.shape[1:]), dtype=c64,
                             device=dev).index_add_(0, ridx, grad_r)
            gH = gH.reshape(Ht.shape).to(Ht.device, Ht.dtype)
            gr = gr.reshape(rt.shape).to(rt.device, rt.dtype)
            gL = _jump_grads(grad_L, plan, Lts, options.cartesian_batching, n, dev)
            return (gH, gr, *gL)

    states, expects = _Solve.apply(Ht, rt, *Lts)
    # the rest of the result (shapes, infos, checks) as for any solve
    return integ._result(states, expects, prep.bufs['infos'], prep.bufs['status'])
