"""``mesolve``: the reference's public entry point over the B200 kernels.

Mirrors ``dq.mesolve`` (``dynamiqs/integrators/apis/mesolve.py:62-304``): the same
arguments, checks and error messages (``_check_mesolve_args`` ``:390-414``,
``check_times`` ``dynamiqs/_checks.py:70-91``, ``check_options``
``dynamiqs/options.py:80-123``, ``assert_method_supported``
``dynamiqs/integrators/_utils.py:84-90``), the same batching semantics
(``_vectorized_mesolve`` ``mesolve.py:307-336``: cartesian by default, broadcast when
``cartesian_batching=False``) and the same result layout (``MESolveResult``).

Where the reference registers ``mesolve_tsit5_integrator_constructor`` /
``mesolve_dopri5_integrator_constructor`` in ``_mesolve`` (``mesolve.py:349-381``),
this module uses :class:`MESolveB200Integrator`, built with the same keyword arguments
(``ts, y0, method, gradient, options, H, Ls, Es``) and exposing ``run()``.  Instead of
one vmapped diffrax loop, the whole batch is flattened into instances described by
index arrays (which H, which jump-operator set, which rho0) and solved by one kernel
launch in which every instance keeps its own t, dt and accept/reject state.
"""

from __future__ import annotations

import math
import warnings
from dataclasses import dataclass

import numpy as np

from . import _lib
from .method import Dopri5, Method, Tsit5
from .options import Options, check_options
from .qarrays import SparseDIA, to_dense
from .result import AdaptiveStepInfos, MESolveResult

__all__ = ['mesolve', 'MESolveB200Integrator']

_MAX_STEPS_MSG = (
    'The maximum number of method steps has been reached (the default value is '
    '`max_steps=100_000`). Try increasing `max_steps` with the `method` argument, e.g. '
    '`method=dq.method.Tsit5(max_steps=1_000_000)`.')


# --------------------------------------------------------------------------------------
# argument conversion and checks
# --------------------------------------------------------------------------------------


def _as_op(x):
    if isinstance(x, SparseDIA):
        return x
    if hasattr(x, 'detach'):
        x = x.detach().cpu().numpy()
    if callable(getattr(x, 'to_numpy', None)):
        x = x.to_numpy()
    x = np.asarray(x)
    if not np.iscomplexobj(x):
        x = x.astype(np.complex64)
    return x


def _shape(x):
    return tuple(x.shape)


def _check_shape(x, argname: str, *shapes: str, subs: dict | None = None) -> None:
    """``check_shape`` (``dynamiqs/_checks.py:21-57``) for the patterns mesolve uses."""
    shp = _shape(x)
    for pattern in shapes:
        if pattern == '(..., n, n)' and len(shp) >= 2 and shp[-1] == shp[-2]:
            return
        if pattern == '(..., n, 1)' and len(shp) >= 2 and shp[-1] == 1:
            return
        if pattern == '(n, n)' and len(shp) == 2 and shp[-1] == shp[-2]:
            return
    shapes_str = ' or '.join(shapes)
    for k, v in (subs or {}).items():
        shapes_str = shapes_str.replace(k, v)
    raise ValueError(f'Argument `{argname}` must have shape {shapes_str}, but has shape '
                     f'{argname}.shape={shp}.')


def check_times(tsave: np.ndarray, argname: str) -> np.ndarray:
    if tsave.ndim != 1:
        raise ValueError(f'Argument {argname} must be a 1D array, but is a {tsave.ndim}D array.')
    if len(tsave) == 0:
        raise ValueError(f'Argument {argname} must contain at least one element.')
    if np.any(tsave[1:] < tsave[:-1]):
        raise ValueError(f'Argument {argname} must be sorted in strictly ascending order.')
    return tsave


def _check_mesolve_args(H, Ls, rho0, exp_ops) -> None:
    _check_shape(H, 'H', '(..., n, n)', subs={'...': '...H'})
    for i, L in enumerate(Ls):
        _check_shape(L, f'jump_ops[{i}]', '(..., n, n)', subs={'...': f'...L{i}'})
    if len(Ls) == 0 and _shape(rho0)[-1] == 1:
        warnings.warn(
            'Argument `jump_ops` is an empty list and argument `rho0` is a ket, consider '
            'using `dq.sesolve()` to solve the Schrödinger equation.', stacklevel=3)
    _check_shape(rho0, 'rho0', '(..., n, 1)', '(..., n, n)', subs={'...': '...rho0'})
    if isinstance(rho0, SparseDIA):
        raise ValueError('Argument rho0 must have layout `dense` but has layout '
                         'rho0.layout=dia.')
    if exp_ops is not None:
        for i, E in enumerate(exp_ops):
            _check_shape(E, f'exp_ops[{i}]', '(n, n)')


def assert_method_supported(method) -> None:
    supported = (Tsit5, Dopri5)
    if not isinstance(method, supported):
        supported_str = ', '.join(f'`{x.__name__}`' for x in supported)
        raise TypeError(f'Method of type `{type(method).__name__}` is not supported '
                        f'(supported method types: {supported_str}).')


# --------------------------------------------------------------------------------------
# batching plan
# --------------------------------------------------------------------------------------


@dataclass
class BatchPlan:
    bshape: tuple  # leading result dims
    H_items: np.ndarray  # (nH, n, n) or SparseDIA with diags (nH, nd, n)
    L_sets: np.ndarray  # (nLsets, K, n, n)
    rho_items: np.ndarray  # (nrho, n, n) or (nrho, n, 1)
    H_index: np.ndarray  # int32 [B]
    L_index: np.ndarray
    rho_index: np.ndarray

    @property
    def batch(self) -> int:
        return int(np.prod(self.bshape, dtype=np.int64)) if self.bshape else 1


def _place(n_items_shape: tuple, start: int, full: tuple) -> np.ndarray:
    """Flat item index of every instance for an argument whose batch dims sit at
    ``full[start:start + len(n_items_shape)]``."""
    a = np.arange(int(np.prod(n_items_shape, dtype=np.int64))).reshape(n_items_shape)
    shape = (1,) * start + n_items_shape + (1,) * (len(full) - start - len(n_items_shape))
    return np.broadcast_to(a.reshape(shape), full).reshape(-1)


def make_batch_plan(H, Ls, rho0, cartesian: bool) -> BatchPlan:
    """Flatten the reference's batching into per-instance index arrays
    (``mesolve.py:307-336``; ``cartesian_vmap`` / ``multi_vmap``,
    ``dynamiqs/integrators/_utils.py:93-187``)."""
    Hd = to_dense(H) if not isinstance(H, SparseDIA) else H
    n = _shape(H)[-1]
    H_b = _shape(H)[:-2]
    L_bs = [_shape(L)[:-2] for L in Ls]
    r_b = _shape(rho0)[:-2]
    K = len(Ls)
    Ld = [to_dense(L) for L in Ls]
    rd = np.asarray(rho0)
    if cartesian:
        Lcat = tuple(d for b in L_bs for d in b)
        full = H_b + Lcat + r_b
        H_index = _place(H_b, 0, full)
        L_index = _place(Lcat, len(H_b), full)
        rho_index = _place(r_b, len(H_b) + len(Lcat), full)
        # materialise one stacked jump set per combination of the L batch indices
        mats = []
        pos = 0
        for Lk, b in zip(Ld, L_bs):
            shape = (1,) * pos + b + (1,) * (len(Lcat) - pos - len(b)) + (n, n)
            mats.append(np.broadcast_to(Lk.reshape(shape), Lcat + (n, n)).reshape(-1, n, n))
            pos += len(b)
        L_sets = np.stack(mats, axis=1) if K else np.zeros((1, 0, n, n), np.complex64)
    else:
        full = np.broadcast_shapes(H_b, *L_bs, r_b)
        H_index = np.broadcast_to(np.arange(int(np.prod(H_b, dtype=np.int64))).reshape(H_b), full).reshape(-1)
        rho_index = np.broadcast_to(np.arange(int(np.prod(r_b, dtype=np.int64))).reshape(r_b), full).reshape(-1)
        if all(len(b) == 0 for b in L_bs):
            L_sets = np.stack(Ld, axis=0)[None] if K else np.zeros((1, 0, n, n), np.complex64)
            L_index = np.zeros(int(np.prod(full, dtype=np.int64)), dtype=np.int64)
        else:
            mats = [np.broadcast_to(Lk, full + (n, n)).reshape(-1, n, n) for Lk in Ld]
            L_sets = np.stack(mats, axis=1)
            L_index = np.arange(int(np.prod(full, dtype=np.int64)))
    if isinstance(Hd, SparseDIA):
        H_items = SparseDIA(Hd.offsets, Hd.diags.reshape(-1, len(Hd.offsets), n))
    else:
        H_items = Hd.reshape(-1, n, n)
    rho_items = rd.reshape(-1, *rd.shape[-2:])
    return BatchPlan(tuple(full), H_items, np.ascontiguousarray(L_sets), rho_items,
                     H_index.astype(np.int32), L_index.astype(np.int32),
                     rho_index.astype(np.int32))


# --------------------------------------------------------------------------------------
# integrator
# --------------------------------------------------------------------------------------


def _device():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError('dynamiqs_b200.mesolve needs a CUDA device (sm_100a); there is '
                           'no CPU fallback.')
    return torch.device('cuda', torch.cuda.current_device())


def _to_dev(x, dtype, device):
    import torch

    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(x)).to(device=device, dtype=dtype).contiguous()


class MESolveB200Integrator:
    """Registry-compatible integrator: ``constructor(ts=, y0=, method=, gradient=,
    options=, H=, Ls=, Es=)`` then ``.run() -> MESolveResult``
    (``dynamiqs/integrators/apis/mesolve.py:372-384``)."""

    def __init__(self, *, ts, y0, method, gradient, options, H, Ls, Es, plan: BatchPlan):
        self.ts = ts
        self.y0 = y0
        self.method = method
        self.gradient = gradient
        self.options = options
        self.H = H
        self.Ls = Ls
        self.Es = Es
        self.plan = plan

    @property
    def t0(self) -> float:
        return float(self.ts[0] if self.options.t0 is None else self.options.t0)

    def _ode_options(self) -> _lib.OdeOptions:
        o = self.options
        m = self.method
        form = (_lib.FORM_STANDARD if (o.vectorized or not o.assume_hermitian)
                else _lib.FORM_HERMITIAN)
        return _lib.OdeOptions(
            method=_lib.METHOD_TSIT5 if isinstance(m, Tsit5) else _lib.METHOD_DOPRI5,
            form=form, rtol=float(m.rtol), atol=float(m.atol), safety=float(m.safety_factor),
            factormin=float(m.min_factor), factormax=float(m.max_factor),
            max_steps=int(m.max_steps), t0=self.t0, save_states=int(bool(o.save_states)),
            check_hermitian=int(bool(o.assume_hermitian)))

    def run(self) -> MESolveResult:
        import torch

        lib = _lib.load()
        dev = _device()
        plan = self.plan
        n = _shape(self.H)[-1]
        K = len(self.Ls)
        ntsave = len(self.ts)
        B = plan.batch
        nE = len(self.Es) if self.Es else 0
        nsave = ntsave if self.options.save_states else 1
        if n > lib.dqb_dense_small_max_n(K):
            raise NotImplementedError(
                f'Hilbert dimension n={n} with {K} jump operators is beyond the dense '
                'shared-memory kernel of this build.')
        H_items = plan.H_items.to_dense() if isinstance(plan.H_items, SparseDIA) else plan.H_items
        c64 = torch.complex64
        H_d = _to_dev(H_items, c64, dev)
        L_d = _to_dev(plan.L_sets, c64, dev)
        r_items = plan.rho_items
        is_ket = r_items.shape[-1] == 1 and n > 1
        r_d = _to_dev(r_items, c64, dev)
        E_d = (_to_dev(np.stack([to_dense(E) for E in self.Es]), c64, dev) if nE
               else torch.zeros(1, dtype=c64, device=dev))
        ts_d = _to_dev(np.asarray(self.ts, dtype=np.float64), torch.float64, dev)
        idx = [_to_dev(a, torch.int32, dev) for a in (plan.H_index, plan.L_index, plan.rho_index)]
        states = torch.empty((B, nsave, n, n), dtype=c64, device=dev)
        expects = torch.empty((B, max(nE, 1), ntsave), dtype=c64, device=dev)
        infos = torch.empty((B, 3), dtype=torch.int32, device=dev)
        status = torch.empty((B,), dtype=torch.int32, device=dev)
        prob = _lib.DenseProblem(
            n=n, n_jumps=K, n_exp=nE, n_tsave=ntsave, batch=B, H=H_d.data_ptr(),
            L=L_d.data_ptr(), rho0=r_d.data_ptr(), rho0_is_ket=int(is_ket),
            E=E_d.data_ptr(), tsave=ts_d.data_ptr(), H_index=idx[0].data_ptr(),
            L_index=idx[1].data_ptr(), rho0_index=idx[2].data_ptr())
        outs = _lib.Outputs(states=states.data_ptr(), expects=expects.data_ptr(),
                            infos=infos.data_ptr(), status=status.data_ptr())
        opts = self._ode_options()
        ws_bytes = lib.dqb_mesolve_dense_workspace_size(n, K, B)
        ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = lib.dqb_mesolve_dense(prob, opts, outs, ws.data_ptr(), ws_bytes, stream)
        _lib.check(rc, 'dqb_mesolve_dense')
        return self._result(states, expects if nE else None, infos, status)

    def _result(self, states, expects, infos, status) -> MESolveResult:
        import torch

        st = status.cpu()
        if bool((st == _lib.INST_NOT_HERMITIAN).any()):
            raise RuntimeError('Argument y0 is not hermitian.')
        if bool((st == _lib.INST_MAX_STEPS).any()):
            raise RuntimeError(_MAX_STEPS_MSG)
        if bool((st == _lib.INST_NONFINITE).any()):
            raise RuntimeError('The solution became non-finite (NaN or inf) during the '
                               'integration.')
        bshape = self.plan.bshape
        n = states.shape[-1]
        states = states.reshape(*bshape, states.shape[1], n, n)
        if expects is not None:
            expects = expects.reshape(*bshape, expects.shape[1], expects.shape[2])
        infos = infos.reshape(*bshape, 3)
        info = AdaptiveStepInfos(infos[..., 0], infos[..., 1], infos[..., 2])
        extra = None
        if self.options.save_extra is not None:
            if not self.options.save_states:
                raise NotImplementedError('`save_extra` needs `save_states=True` on the '
                                          'B200 path (it is applied to the saved states).')
            flat = states.reshape(-1, n, n)
            vals = [self.options.save_extra(s) for s in flat]
            try:
                extra = torch.stack([torch.as_tensor(v) for v in vals]).reshape(
                    *states.shape[:-2], *torch.as_tensor(vals[0]).shape)
            except (TypeError, RuntimeError):
                extra = vals
        return MESolveResult(tsave=self.ts, method=self.method, gradient=self.gradient,
                             options=self.options, states=states, expects=expects,
                             infos=info, extra=extra)


# --------------------------------------------------------------------------------------
# public entry point
# --------------------------------------------------------------------------------------


def mesolve(H, jump_ops, rho0, tsave, *, exp_ops=None, method: Method = Tsit5(),  # noqa: B008
            gradient=None, options: Options = Options()) -> MESolveResult:  # noqa: B008
    r"""Solve the Lindblad master equation
    d rho/dt = -i[H, rho] + sum_k (L_k rho L_k^+ - 1/2 {L_k^+ L_k, rho})
    on the GPU (``dq.mesolve``, ``dynamiqs/integrators/apis/mesolve.py:62-304``).

    Args and result follow the reference: ``H`` ``(...H, n, n)``, ``jump_ops`` list of
    ``(...Lk, n, n)``, ``rho0`` ``(...rho0, n, 1)`` or ``(..., n, n)``, ``tsave``
    ``(ntsave,)``; ``exp_ops`` list of ``(n, n)``.  Operators may be dense array-likes or
    :class:`~dynamiqs_b200.qarrays.SparseDIA`.  ``method`` is ``Tsit5`` (default) or
    ``Dopri5``.
    """
    if getattr(H, '__class__', None).__name__.endswith('TimeQArray'):
        raise NotImplementedError('Time-dependent operators are not supported on the B200 '
                                  'mesolve path yet.')
    H = _as_op(H)
    Ls = [_as_op(L) for L in jump_ops]
    rho0 = _as_op(rho0)
    tsave = np.asarray(tsave.detach().cpu().numpy() if hasattr(tsave, 'detach') else tsave,
                       dtype=np.float64)
    if exp_ops is not None:
        exp_ops = [_as_op(E) for E in exp_ops] if len(exp_ops) > 0 else None

    _check_mesolve_args(H, Ls, rho0, exp_ops)
    tsave = check_times(tsave, 'tsave')
    check_options(options, 'mesolve')
    options = options.initialise()
    assert_method_supported(method)
    method.assert_supports_gradient(gradient)

    n = _shape(H)[-1]
    for i, L in enumerate(Ls):
        if _shape(L)[-1] != n:
            raise ValueError(f'Argument `jump_ops[{i}]` must have shape (..., {n}, {n}).')
    if _shape(rho0)[-2] != n:
        raise ValueError(f'Argument `rho0` must have shape (..., {n}, 1) or (..., {n}, {n}).')

    plan = make_batch_plan(H, Ls, rho0, options.cartesian_batching)
    integrator = MESolveB200Integrator(ts=tsave, y0=rho0, method=method, gradient=gradient,
                                       options=options, H=H, Ls=Ls, Es=exp_ops, plan=plan)
    return integrator.run()


def _prod(shape) -> int:
    return int(math.prod(shape)) if shape else 1
