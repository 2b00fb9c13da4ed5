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

# Largest n^2 of the vectorized master-equation kernel (n <= 16); beyond it
# options.vectorized=True solves the standard form, the same ODE with the same RMS norm.
VECTORIZED_MAX_N2 = 256

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
    H_items: object  # (nH, n, n) dense, or SparseDIA with diags (nH, nd, n)
    L_sets: object  # (nLsets, K, n, n) dense, or list of K SparseDIA with diags (nLsets, nd_k, n)
    rho_items: np.ndarray  # (nrho, n, n) or (nrho, n, 1)
    H_index: np.ndarray  # int32 [B]
    L_index: np.ndarray
    rho_index: np.ndarray

    @property
    def batch(self) -> int:
        return int(np.prod(self.bshape, dtype=np.int64)) if self.bshape else 1

    def L_sets_dense(self) -> np.ndarray:
        if isinstance(self.L_sets, np.ndarray):
            return self.L_sets
        if not self.L_sets:
            return np.zeros((1, 0, 1, 1), np.complex64)
        return np.stack([L.to_dense() for L in self.L_sets], axis=1)

    def H_items_dense(self) -> np.ndarray:
        return self.H_items.to_dense() if isinstance(self.H_items, SparseDIA) else self.H_items


def _place(n_items_shape: tuple, start: int, full: tuple) -> np.ndarray:
    """Flat item index of every instance for an argument whose batch dims sit at
    ``full[start:start + len(n_items_shape)]``."""
    a = np.arange(int(np.prod(n_items_shape, dtype=np.int64))).reshape(n_items_shape)
    shape = (1,) * start + n_items_shape + (1,) * (len(full) - start - len(n_items_shape))
    return np.broadcast_to(a.reshape(shape), full).reshape(-1)


def _stack_sets(Ls, L_bs, n, cartesian, full):
    """Jump sets indexed like ``L_index``: dense (nsets, K, n, n) when every operator is
    dense, else one SparseDIA per jump with diags (nsets, nd_k, n)."""
    K = len(Ls)
    dia_mode = any(isinstance(L, SparseDIA) for L in Ls)
    if dia_mode:
        Ls = [L if isinstance(L, SparseDIA) else SparseDIA.from_dense(L) for L in Ls]
        items = [(L.diags, L.diags.shape[-2:]) for L in Ls]
    else:
        items = [(np.asarray(L), (n, n)) for L in Ls]
    if cartesian:
        Lcat = tuple(d for b in L_bs for d in b)
        mats, pos = [], 0
        for (arr, tail), b in zip(items, L_bs):
            shape = (1,) * pos + b + (1,) * (len(Lcat) - pos - len(b)) + tail
            mats.append(np.broadcast_to(arr.reshape(shape), Lcat + tail).reshape(-1, *tail))
            pos += len(b)
        L_index_shape = Lcat
    elif all(len(b) == 0 for b in L_bs):
        mats = [arr.reshape(1, *tail) for arr, tail in items]
        L_index_shape = None
    else:
        mats = [np.broadcast_to(arr, full + tail).reshape(-1, *tail) for arr, tail in items]
        L_index_shape = full
    if dia_mode:
        sets = [SparseDIA(L.offsets, np.ascontiguousarray(m)) for L, m in zip(Ls, mats)]
    else:
        sets = (np.ascontiguousarray(np.stack(mats, axis=1)) if K
                else np.zeros((1, 0, n, n), np.complex64))
    return sets, L_index_shape


def make_batch_plan(H, Ls, rho0, cartesian: bool) -> BatchPlan:
    """Flatten the reference's batching into per-instance index arrays
    (``mesolve.py:307-336``; ``cartesian_vmap`` / ``multi_vmap``,
    ``dynamiqs/integrators/_utils.py:93-187``)."""
    n = _shape(H)[-1]
    H_b = _shape(H)[:-2]
    L_bs = [_shape(L)[:-2] for L in Ls]
    r_b = _shape(rho0)[:-2]
    rd = np.asarray(rho0)
    if cartesian:
        Lcat = tuple(d for b in L_bs for d in b)
        full = H_b + Lcat + r_b
        H_index = _place(H_b, 0, full)
        L_index = _place(Lcat, len(H_b), full)
        rho_index = _place(r_b, len(H_b) + len(Lcat), full)
        L_sets, _ = _stack_sets(Ls, L_bs, n, True, full)
    else:
        full = tuple(np.broadcast_shapes(H_b, *L_bs, r_b))
        H_index = np.broadcast_to(np.arange(int(np.prod(H_b, dtype=np.int64))).reshape(H_b), full).reshape(-1)
        rho_index = np.broadcast_to(np.arange(int(np.prod(r_b, dtype=np.int64))).reshape(r_b), full).reshape(-1)
        L_sets, shp = _stack_sets(Ls, L_bs, n, False, full)
        nb = int(np.prod(full, dtype=np.int64))
        L_index = np.zeros(nb, dtype=np.int64) if shp is None else np.arange(nb)
    if isinstance(H, SparseDIA):
        H_items = SparseDIA(H.offsets, H.diags.reshape(-1, len(H.offsets), n))
    else:
        H_items = np.asarray(H).reshape(-1, n, n)
    rho_items = rd.reshape(-1, *rd.shape[-2:])
    return BatchPlan(tuple(full), H_items, L_sets, rho_items, H_index.astype(np.int32),
                     L_index.astype(np.int32), rho_index.astype(np.int32))


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
    a = np.ascontiguousarray(x)
    if not a.flags.writeable:  # a read-only view (e.g. a broadcast): torch wants its own copy
        a = a.copy()
    return torch.from_numpy(a).to(device=device, dtype=dtype).contiguous()


class PreparedSolve:
    """A bound C-ABI solve with device-resident inputs, outputs and workspace."""

    def __init__(self, integrator, fn, name, prob, outs, bufs, ws_bytes, dev, nE):
        self.integrator = integrator
        self.fn = fn
        self.name = name
        self.prob = prob
        self.outs = outs
        self.bufs = bufs
        self.ws_bytes = ws_bytes
        self.dev = dev
        self.nE = nE

    def launch(self, stream=None) -> PreparedSolve:
        import torch

        s = stream if stream is not None else torch.cuda.current_stream(self.dev).cuda_stream
        rc = self.fn(self.prob, self.integrator._ode_options(), self.outs,
                     self.bufs['workspace'].data_ptr(), self.ws_bytes, s)
        _lib.check(rc, self.name)
        return self

    def result(self) -> MESolveResult:
        b = self.bufs
        return self.integrator._result(b['states'], b['expects'] if self.nE else None,
                                       b['infos'], b['status'])


# Shape codes of the sparse-DIA stencil (dqb_ode_options.tile) the autotuner times: the
# generic kernel, the tiled one with 4, 8, 16 rows per thread, the staged one with 8 or 16
# rows per CTA, the wide one with 4 or 2 columns per thread and 8 or 16 rows per CTA (and
# 8 rows with two rows' loads in flight per thread: 408, 508; 8 rows and 2 columns with
# registers capped for more resident CTAs: 708), and the bulk-staged one with
# stages of 4 or 8 rows (604, 608; hermitian form).
DIA_STENCIL_SHAPES = (1, 4, 8, 16, 108, 116, 208, 216, 308, 316, 408, 508, 604, 608, 708)


def _stepper_code(o) -> int:
    """DQB_STEPPER_* for ``Options.stepper``."""
    try:
        return _lib.STEPPERS[o.stepper]
    except KeyError:
        raise ValueError(f'Option `stepper` must be one of {sorted(_lib.STEPPERS)}, '
                         f'got {o.stepper!r}.') from None


def _dia_tune_form(form: int, stepper: int) -> int:
    """Form in which the DIA solve's stencils write, for the autotuner to time: the stage
    form of the hermitian form fills only the stage slots' upper 32 x 32 tiles
    (FORM_HERMITIAN_UPPER); the Krylov basis and the standard form write whole matrices."""
    if form == _lib.FORM_HERMITIAN and stepper != _lib.STEPPER_KRYLOV:
        return _lib.FORM_HERMITIAN_UPPER
    return form


def _precision_code(o, form: int, path: str = 'large') -> int:
    """DQB_PREC_* for ``Options.precision`` on `path` ('small': the n <= 64 kernel,
    'large': the GEMM path, 'dia'); the tensor-core modes need the hermitian form.
    'f16x3' applies to the n <= 64 kernel only and the TF32/BF16 modes to the GEMM path
    only: elsewhere they mean FP32.  ``'auto'`` maps to FP32 here (the n <= 64 kernel keeps
    the reference's error control only in FP32: see Options.precision); the GEMM path's
    prepare step replaces it with the autotuner's choice."""
    if o.precision == 'auto':
        return _lib.PREC_FP32
    try:
        code = _lib.PRECISIONS[o.precision]
    except KeyError:
        raise ValueError(f'Option `precision` must be one of {sorted(_lib.PRECISIONS)}, '
                         f'got {o.precision!r}.') from None
    if code != _lib.PREC_FP32 and form != _lib.FORM_HERMITIAN:
        raise ValueError('Option `precision` other than "fp32" needs the hermitian form '
                         '(assume_hermitian=True, vectorized=False).')
    if (code == _lib.PREC_F16X3) != (path == 'small'):
        return _lib.PREC_FP32
    return code


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
        # The identity is appended to the expectation operators: its FP64-summed expectation
        # value at every save point is the trace check of the saved states (result.checks).
        self._n_user_E = len(Es) if Es else 0
        self.Es = list(Es or []) + [np.eye(_shape(H)[-1], dtype=np.complex64)]
        self.plan = plan
        self._tuned: dict = {}  # launch choices made by the autotuner at prepare time
        self._path = 'large'  # 'small', 'large' or 'dia': set by prepare()

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
            check_hermitian=int(bool(o.assume_hermitian)),
            precision=self._tuned.get('precision', _precision_code(o, form, self._path)),
            tile=self._tuned.get('tile', 0), stepper=_stepper_code(o))

    def _form(self) -> int:
        o = self.options
        return (_lib.FORM_STANDARD if (o.vectorized or not o.assume_hermitian)
                else _lib.FORM_HERMITIAN)

    def run(self) -> MESolveResult:
        return self.prepare().launch().result()

    def prepare(self) -> PreparedSolve:
        """Copy the inputs to the device, size the workspace and bind the C-ABI call;
        ``launch()`` may then be called repeatedly (the device inputs stay resident)."""
        lib = _lib.load()
        n = _shape(self.H)[-1]
        K = len(self.Ls)
        dia_ops = isinstance(self.H, SparseDIA) or any(isinstance(L, SparseDIA) for L in self.Ls)
        if self.options.vectorized and n * n <= VECTORIZED_MAX_N2:
            return self._prepare_vectorized(lib)
        if n <= lib.dqb_dense_small_max_n(K):
            return self._prepare_dense(lib, 'small')
        if dia_ops:
            return self._prepare_dia(lib)
        return self._prepare_dense(lib, 'large')


    def _prepare_vectorized(self, lib) -> PreparedSolve:
        """``options.vectorized=True`` (``diffrax_integrator.py:325-345``): the ODE
        d vec(rho)/dt = S vec(rho) with S = slindbladian(H, jump_ops), one superoperator
        per distinct (H item, jump set) pair of the batch, solved by dqb_mesolve_vectorized
        on vec(rho) (n^2 entries: the error norm runs over them, as in the reference)."""
        import torch

        from .vectorization import slindbladian, vectorize

        self._path = 'vectorized'
        dev = _device()
        n, K, ntsave, B, nE, nsave = self._sizes()
        N = n * n
        plan = self.plan
        c64 = torch.complex64
        Hs = plan.H_items_dense()
        Lsets = plan.L_sets_dense()
        pairs = np.stack([plan.H_index, plan.L_index], axis=1)
        uniq, inverse = np.unique(pairs, axis=0, return_inverse=True)
        S_T = np.stack([np.ascontiguousarray(
            slindbladian(Hs[h], [Lsets[l, k] for k in range(K)]).T) for h, l in uniq])
        rho = plan.rho_items
        if rho.shape[-1] == 1 and n > 1:
            rho = rho @ np.conj(np.swapaxes(rho, -1, -2))  # todm
        if self.options.assume_hermitian:
            herm = np.abs(rho - np.conj(np.swapaxes(rho, -1, -2))) <= 1e-5 + 1e-5 * np.abs(rho)
            if not herm.all():
                raise RuntimeError('Argument y0 is not hermitian.')
        bufs = {
            'superop_t': _to_dev(S_T, c64, dev),
            'rho0': _to_dev(vectorize(rho)[..., 0], c64, dev),
            'E': (_to_dev(np.stack([to_dense(E).reshape(-1) for E in self.Es]), c64, dev) if nE
                  else torch.zeros(1, dtype=c64, device=dev)),
            'tsave': _to_dev(np.asarray(self.ts, dtype=np.float64), torch.float64, dev),
            'S_index': _to_dev(inverse.reshape(-1).astype(np.int32), torch.int32, dev),
            'rho0_index': _to_dev(plan.rho_index, torch.int32, dev),
            'states': torch.empty((B, nsave, N), dtype=c64, device=dev),
            'expects': torch.empty((B, max(nE, 1), ntsave), dtype=c64, device=dev),
            'infos': torch.empty((B, 3), dtype=torch.int32, device=dev),
            'status': torch.empty((B,), dtype=torch.int32, device=dev),
            'workspace': torch.empty(256, dtype=torch.uint8, device=dev),
        }
        prob = _lib.DenseProblem(
            n=N, n_jumps=0, n_exp=nE, n_tsave=ntsave, batch=B, H=bufs['superop_t'].data_ptr(),
            rho0=bufs['rho0'].data_ptr(), rho0_is_ket=1, E=bufs['E'].data_ptr(),
            tsave=bufs['tsave'].data_ptr(), H_index=bufs['S_index'].data_ptr(),
            rho0_index=bufs['rho0_index'].data_ptr())
        outs = _lib.Outputs(states=bufs['states'].data_ptr(), expects=bufs['expects'].data_ptr(),
                            infos=bufs['infos'].data_ptr(), status=bufs['status'].data_ptr())
        S_ptr = bufs['superop_t'].data_ptr()

        def fn(prob_, opts, outs_, ws, wsb, stream):
            return lib.dqb_mesolve_vectorized(prob_, S_ptr, opts, outs_, ws, wsb, stream)

        return PreparedSolve(self, fn, 'dqb_mesolve_vectorized', prob, outs, bufs, 256, dev, nE)

    def _common_buffers(self, dev, n, ntsave, nE, B, nsave):
        import torch

        c64 = torch.complex64
        plan = self.plan
        r_items = plan.rho_items
        is_ket = r_items.shape[-1] == 1 and n > 1
        bufs = {
            'rho0': _to_dev(r_items, c64, dev),
            'E': (_to_dev(np.stack([to_dense(E) for E in self.Es]), c64, dev) if nE
                  else torch.zeros(1, dtype=c64, device=dev)),
            'tsave': _to_dev(np.asarray(self.ts, dtype=np.float64), torch.float64, dev),
            'H_index': _to_dev(plan.H_index, torch.int32, dev),
            'L_index': _to_dev(plan.L_index, torch.int32, dev),
            'rho0_index': _to_dev(plan.rho_index, torch.int32, dev),
            'states': torch.empty((B, nsave, n, n), dtype=c64, device=dev),
            'expects': torch.empty((B, max(nE, 1), ntsave), dtype=c64, device=dev),
            'infos': torch.empty((B, 3), dtype=torch.int32, device=dev),
            'status': torch.empty((B,), dtype=torch.int32, device=dev),
        }
        outs = _lib.Outputs(states=bufs['states'].data_ptr(), expects=bufs['expects'].data_ptr(),
                            infos=bufs['infos'].data_ptr(), status=bufs['status'].data_ptr())
        return bufs, outs, is_ket

    def _sizes(self):
        n = _shape(self.H)[-1]
        ntsave = len(self.ts)
        nE = len(self.Es) if self.Es else 0
        nsave = ntsave if self.options.save_states else 1
        return n, len(self.Ls), ntsave, self.plan.batch, nE, nsave

    def _prepare_dense(self, lib, kind, extra_mats: int = 0) -> PreparedSolve:
        """`extra_mats`: shared-memory matrices the kernel needs beyond the jump operators
        (1 for a time-dependent H: its constant part)."""
        import torch

        self._path = kind
        dev = _device()
        n, K, ntsave, B, nE, nsave = self._sizes()
        c64 = torch.complex64
        bufs, outs, is_ket = self._common_buffers(dev, n, ntsave, nE, B, nsave)
        bufs['H'] = _to_dev(self.plan.H_items_dense(), c64, dev)
        bufs['L'] = _to_dev(self.plan.L_sets_dense(), c64, dev)
        prob = _lib.DenseProblem(
            n=n, n_jumps=K, n_exp=nE, n_tsave=ntsave, batch=B, H=bufs['H'].data_ptr(),
            L=bufs['L'].data_ptr(), rho0=bufs['rho0'].data_ptr(), rho0_is_ket=int(is_ket),
            E=bufs['E'].data_ptr(), tsave=bufs['tsave'].data_ptr(),
            H_index=bufs['H_index'].data_ptr(), L_index=bufs['L_index'].data_ptr(),
            rho0_index=bufs['rho0_index'].data_ptr())
        if kind == 'small':
            ws_bytes = lib.dqb_mesolve_dense_workspace_size(n, K + extra_mats, B)
            fn, name = lib.dqb_mesolve_dense, 'dqb_mesolve_dense'
            if B > 256:  # more instances than resident CTAs: start the stiffest first
                bufs['start_order'] = _to_dev(self._start_order(), torch.int32, dev)
                prob.start_order = bufs['start_order'].data_ptr()
        else:
            ws_bytes = lib.dqb_mesolve_dense_large_workspace_size(n, K, nE, ntsave, B)
            fn, name = lib.dqb_mesolve_dense_large, 'dqb_mesolve_dense_large'
        bufs['workspace'] = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
        if kind == 'large' and self.options.precision == 'auto':
            self._tune_gemm_precision(lib, prob, bufs['workspace'], ws_bytes, dev)
        return PreparedSolve(self, fn, name, prob, outs, bufs, ws_bytes, dev, nE)

    def _start_order(self) -> np.ndarray:
        """Instances sorted by a stiffness estimate, largest first: the infinity norm of
        Hnh = -iH - 1/2 sum L^+L bounded by ||H|| + 1/2 sum ||L||^2 (row sums).  An
        explicit RK step size scales roughly with the inverse of that spectral radius, so
        this starts the longest solves first and leaves short ones for the tail of the
        persistent kernel.  Changes only the order of work, not any result."""
        plan = self.plan
        H = plan.H_items_dense()
        h = np.abs(H).sum(-1).max(-1)
        Ls = plan.L_sets_dense()
        if Ls.shape[1]:
            lnorm = np.abs(Ls).sum(-1).max(-1)
            l_est = 0.5 * (lnorm ** 2).sum(-1)
        else:
            l_est = np.zeros(Ls.shape[0])
        est = h[np.asarray(plan.H_index)] + l_est[np.asarray(plan.L_index)]
        return np.argsort(-est, kind='stable').astype(np.int32)

    def _tune_gemm_precision(self, lib, prob, ws, ws_bytes, dev) -> None:
        """``precision='auto'``: the faster of FP32 and 3xTF32 products for this (n, K,
        batch), timed on one right-hand side of up to 256 instances."""
        import ctypes

        import torch

        from . import autotune

        n, K, B, form = prob.n, prob.n_jumps, prob.batch, self._form()
        cands = [_lib.PREC_FP32]
        if form == _lib.FORM_HERMITIAN and n % 2 == 0:
            cands.append(_lib.PREC_TF32X3)
        Bt = min(B, 256)
        pt = _lib.DenseProblem.from_buffer_copy(prob)
        pt.batch = Bt
        g = torch.Generator(device='cpu').manual_seed(0)
        Y = torch.randn(Bt, n, n, dtype=torch.complex64, generator=g)
        rho = (Y @ Y.mH / n).to(dev)
        out = torch.empty_like(rho)
        stream = torch.cuda.current_stream(dev).cuda_stream

        def make_run(c):
            def run():
                _lib.check(lib.dqb_lindblad_rhs_dense_large_prec(
                    ctypes.byref(pt), form, c, rho.data_ptr(), out.data_ptr(), ws.data_ptr(),
                    ws_bytes, stream), 'dqb_lindblad_rhs_dense_large_prec')
            return run

        key = ('gemm_precision', torch.cuda.get_device_name(dev), n, K, 'dense',
               autotune.batch_bucket(B), form)
        self._tuned['precision'] = autotune.choose(key, cands, make_run, _lib.PREC_FP32)

    def _prepare_dia(self, lib) -> PreparedSolve:
        import ctypes

        import torch

        self._path = 'dia'
        dev = _device()
        n, K, ntsave, B, nE, nsave = self._sizes()
        plan = self.plan
        c64 = torch.complex64
        bufs, outs, is_ket = self._common_buffers(dev, n, ntsave, nE, B, nsave)
        H = plan.H_items if isinstance(plan.H_items, SparseDIA) else SparseDIA.from_dense(plan.H_items)
        Lsets = plan.L_sets if isinstance(plan.L_sets, list) else [
            SparseDIA.from_dense(plan.L_sets[:, k]) for k in range(plan.L_sets.shape[1])]
        bufs['H'] = _to_dev(H.diags, c64, dev)
        bufs['L'] = (_to_dev(np.concatenate([L.diags for L in Lsets], axis=-2), c64, dev)
                     if Lsets else torch.zeros(1, dtype=c64, device=dev))
        l_off_list = [k for L in Lsets for k in L.offsets]
        host = {  # host arrays the C ABI reads during the call
            'h_off': (ctypes.c_int32 * max(len(H.offsets), 1))(*H.offsets),
            'l_nd': (ctypes.c_int32 * max(len(Lsets), 1))(*[len(L.offsets) for L in Lsets]),
            'l_off': (ctypes.c_int32 * max(len(l_off_list), 1))(*l_off_list),
        }
        vp = ctypes.c_void_p
        prob = _lib.DiaProblem(
            n=n, n_jumps=len(Lsets), n_exp=nE, n_tsave=ntsave, batch=B, h_ndiag=len(H.offsets),
            h_offsets=ctypes.cast(host['h_off'], vp), h_diags=bufs['H'].data_ptr(),
            l_ndiag=ctypes.cast(host['l_nd'], vp), l_offsets=ctypes.cast(host['l_off'], vp),
            l_diags=bufs['L'].data_ptr(), rho0=bufs['rho0'].data_ptr(), rho0_is_ket=int(is_ket),
            E=bufs['E'].data_ptr(), tsave=bufs['tsave'].data_ptr(),
            H_index=bufs['H_index'].data_ptr(), L_index=bufs['L_index'].data_ptr(),
            rho0_index=bufs['rho0_index'].data_ptr())
        ws_bytes = lib.dqb_mesolve_dia_workspace_size(prob)
        if ws_bytes == 0:
            raise NotImplementedError('DIA problem outside the limits of this build '
                                      '(diagonal counts or batch size).')
        bufs['workspace'] = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
        bufs['host'] = host
        self._tune_dia_tile(lib, prob, bufs['workspace'], ws_bytes, dev,
                            (tuple(H.offsets), tuple(tuple(L.offsets) for L in Lsets)))
        return PreparedSolve(self, lib.dqb_mesolve_dia, 'dqb_mesolve_dia', prob, outs, bufs,
                             ws_bytes, dev, nE)

    def _tune_dia_tile(self, lib, prob, ws, ws_bytes, dev, pattern) -> None:
        """Launch shape of the DIA stencil for this (n, sparsity pattern), among
        ``DIA_STENCIL_SHAPES``, timed on one right-hand side of the instances that run
        together (the solve's first instances, at most 1 GiB of states): the grid the solve
        launches, so that its tail and occupancy effects are the ones timed."""
        import ctypes

        import torch

        from . import autotune

        n = prob.n
        form = _dia_tune_form(self._form(), _stepper_code(self.options))
        bt = int(max(1, min(prob.batch, (1 << 30) // (8 * n * n))))
        pt = _lib.DiaProblem.from_buffer_copy(prob)
        pt.batch = bt
        g = torch.Generator(device='cpu').manual_seed(0)
        rho = (torch.randn(bt, n, n, dtype=torch.complex64, generator=g) / n).to(dev)
        out = torch.empty_like(rho)
        stream = torch.cuda.current_stream(dev).cuda_stream

        def make_run(t):
            def run():
                _lib.check(lib.dqb_lindblad_rhs_dia_tiled(
                    ctypes.byref(pt), form, t, rho.data_ptr(), out.data_ptr(),
                    ws.data_ptr(), ws_bytes, stream), 'dqb_lindblad_rhs_dia_tiled')
            return run

        key = ('dia_stencil', torch.cuda.get_device_name(dev), n, prob.n_jumps, pattern,
               autotune.batch_bucket(prob.batch), form)
        self._tuned['tile'] = autotune.choose(key, list(DIA_STENCIL_SHAPES), make_run, 1)

    # kept for callers that select a path explicitly (tests)
    def _run_dense_small(self, lib) -> MESolveResult:
        return self._prepare_dense(lib, 'small').launch().result()

    def _run_dense_large(self, lib) -> MESolveResult:
        return self._prepare_dense(lib, 'large').launch().result()

    def _run_dia(self, lib) -> MESolveResult:
        return self._prepare_dia(lib).launch().result()

    def _checks(self, states, trace):
        """FP64 checks of the saved states: tr(rho) at every save point (the identity's
        expectation value, summed in FP64 by the kernels) and the hermiticity defect
        ||rho - rho^+||_F / ||rho||_F of every saved state (FP64, on the device)."""
        import torch

        st = states.to(torch.complex128)
        den = torch.linalg.norm(st.reshape(*st.shape[:-2], -1), dim=-1)
        num = torch.linalg.norm((st - st.mH).reshape(*st.shape[:-2], -1), dim=-1)
        return {'trace': trace, 'hermiticity': num / torch.clamp(den, min=1e-300)}

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
        trace = None
        if expects is not None:  # the last row is the identity's: the trace check
            trace = expects[:, self._n_user_E].to(torch.complex128)
            trace = trace.reshape(*bshape, trace.shape[-1])
            expects = expects[:, :self._n_user_E] if self._n_user_E else None
        if self._path == 'vectorized':  # vec(rho) -> rho (unvectorize, columns stacked)
            m = int(round(states.shape[-1] ** 0.5))
            states = states.reshape(*states.shape[:-1], m, m).transpose(-1, -2)
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
                             infos=info, extra=extra, checks=self._checks(states, trace))


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
    from .time_qarray import ModulatedTimeQArray, PWCTimeQArray, SummedTimeQArray, as_summed

    td_types = (PWCTimeQArray, ModulatedTimeQArray, SummedTimeQArray)
    if any(isinstance(L, td_types) for L in jump_ops):
        Hs = as_summed(H if isinstance(H, td_types) else _as_op(H))
        if _td_on_dia(Hs, jump_ops, options):
            return _mesolve_td_dia(Hs, jump_ops, rho0, tsave, exp_ops=exp_ops, method=method,
                                   gradient=gradient, options=options)
        if _td_jumps_on_large(Hs, jump_ops, options):
            return _mesolve_td(Hs, jump_ops, rho0, tsave, exp_ops=exp_ops, method=method,
                               gradient=gradient, options=options, kind='large')
        raise NotImplementedError('Time-dependent jump operators need every operator dense (the '
                                  'GEMM path) or every one in sparse-DIA storage (the DIA '
                                  'stepper), each time-dependent jump operator one dq.pwc / '
                                  'dq.modulated term with unbatched values, and at most four '
                                  'time-dependent terms in H.')
    if isinstance(H, td_types):
        Hs = as_summed(H)
        if _td_on_device(Hs, jump_ops, options):
            return _mesolve_td(Hs, jump_ops, rho0, tsave, exp_ops=exp_ops, method=method,
                               gradient=gradient, options=options)
        if _td_on_dia(Hs, jump_ops, options):
            return _mesolve_td_dia(Hs, jump_ops, rho0, tsave, exp_ops=exp_ops, method=method,
                                   gradient=gradient, options=options)
        if _td_on_large(Hs, jump_ops, options):
            return _mesolve_td(Hs, jump_ops, rho0, tsave, exp_ops=exp_ops, method=method,
                               gradient=gradient, options=options, kind='large')
        if not Hs.only_pwc:
            raise NotImplementedError('Modulated Hamiltonians run in one launch with at most four '
                                      'time-dependent terms, options.vectorized=False, and either '
                                      'every operator dense or every operator in sparse-DIA '
                                      'storage.')
        return _mesolve_piecewise(H, jump_ops, rho0, tsave, exp_ops=exp_ops, method=method,
                                  gradient=gradient, options=options, solve=mesolve)
    if getattr(H, '__class__', None).__name__.endswith('TimeQArray'):
        raise NotImplementedError('Callable time-dependent operators cannot run inside the B200 '
                                  'kernels: use dq.pwc or dq.modulated with a Wave prefactor.')
    from .autodiff import mesolve_autograd, needs_autograd

    if needs_autograd(H, jump_ops, rho0):
        tsave_np = np.asarray(tsave.detach().cpu().numpy() if hasattr(tsave, 'detach') else tsave,
                              dtype=np.float64)
        tsave_np = check_times(tsave_np, 'tsave')
        check_options(options, 'mesolve')
        options = options.initialise()
        assert_method_supported(method)
        method.assert_supports_gradient(gradient)
        return mesolve_autograd(H, jump_ops, rho0, tsave_np, exp_ops=exp_ops, method=method,
                                gradient=gradient, options=options,
                                integ_cls=MESolveB200Integrator, make_plan=make_batch_plan,
                                check=_check_mesolve_args)
    if any(isinstance(L, (PWCTimeQArray, SummedTimeQArray)) for L in jump_ops):
        raise NotImplementedError('Time-dependent jump operators are not supported on the B200 '
                                  'path.')
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


def _td_on_device(Hs, jump_ops, options) -> bool:
    """Whether a time-dependent H runs as one launch of the n <= 64 kernel."""
    n = Hs.constant.shape[-1]
    if options.vectorized or len(Hs.td_terms) > _lib.TD_MAX_TERMS:
        return False
    if any(isinstance(L, SparseDIA) or np.ndim(L) != 2 for L in jump_ops):
        return False
    return n <= _lib.load().dqb_dense_small_max_n(len(jump_ops) + 1)


def _td_on_large(Hs, jump_ops, options) -> bool:
    """Whether a time-dependent H with dense operators runs as one launch of the GEMM path
    (n beyond the n <= 64 kernel's reach)."""
    if options.vectorized or len(Hs.td_terms) > _lib.TD_MAX_TERMS or options.stepper == 'krylov':
        return False
    return not any(isinstance(L, SparseDIA) or np.ndim(L) != 2 for L in jump_ops)


def _mesolve_td(Hs, jump_ops, rho0, tsave, *, exp_ops, method, gradient, options, kind='small'):
    """``H(t) = H0 + sum_m c_m(t) H_m`` in one launch (``dqb_mesolve_dense_td`` for
    n <= 64, ``dqb_mesolve_dense_large_td`` on the GEMM path beyond): the kernels evaluate
    the PWC and Wave prefactors at every stage time, and the controller clips its steps at
    the discontinuity times as the reference's ``jump_ts`` does.  Batched PWC values
    ``(..., N)`` are the leading result dimensions (cartesian batching) and run as
    instances of the same launch."""
    import ctypes

    import torch

    from .time_qarray import PWCTimeQArray

    Ls = [_as_op(_jump_source(L)) for L in jump_ops]
    rho0 = _as_op(rho0)
    tsave = np.asarray(tsave.detach().cpu().numpy() if hasattr(tsave, 'detach') else tsave,
                       dtype=np.float64)
    if exp_ops is not None:
        exp_ops = [_as_op(E) for E in exp_ops] if len(exp_ops) > 0 else None
    n = Hs.constant.shape[-1]
    bs = tuple(Hs.batch_shape)
    if bs and not options.cartesian_batching:
        raise NotImplementedError('Batched PWC values need cartesian batching on the B200 path.')
    Hb = np.broadcast_to(Hs.constant.astype(np.complex64), (*bs, n, n))
    _check_mesolve_args(Hb, Ls, rho0, exp_ops)
    tsave = check_times(tsave, 'tsave')
    check_options(options, 'mesolve')
    options = options.initialise()
    assert_method_supported(method)
    method.assert_supports_gradient(gradient)
    plan = make_batch_plan(Hb, Ls, rho0, True)
    integ = MESolveB200Integrator(ts=tsave, y0=rho0, method=method, gradient=gradient,
                                  options=options, H=Hb, Ls=Ls, Es=exp_ops, plan=plan)
    lib = _lib.load()
    if kind == 'small':
        prep = integ._prepare_dense(lib, 'small', extra_mats=1)
    else:  # the GEMM path also keeps the constant Hnh0 in its workspace
        prep = integ._prepare_dense(lib, 'large')
        n_, K_, ntsave_, B_, nE_, _ = integ._sizes()
        wsb = lib.dqb_mesolve_dense_large_td_workspace_size(n_, K_, nE_, ntsave_, B_)
        prep.bufs['workspace'] = torch.empty(max(wsb, 1), dtype=torch.uint8, device=prep.dev)
        prep.ws_bytes = wsb
    dev = prep.dev
    nsets = int(np.prod(bs, dtype=np.int64)) if bs else 1
    terms = (_lib.TdTerm * _lib.TD_MAX_TERMS)()
    keep = []
    for m, term in enumerate(Hs.td_terms):
        T = terms[m]
        if isinstance(term, PWCTimeQArray):
            vals = np.broadcast_to(term.values, (*bs, term.values.shape[-1])).reshape(nsets, -1)
            tt = _to_dev(term.times, torch.float64, dev)
            vv = _to_dev(np.ascontiguousarray(vals, dtype=np.complex128), torch.complex128, dev)
            keep += [tt, vv]
            T.kind, T.n_times = _lib.TD_PWC, term.times.size
            T.times, T.values = tt.data_ptr(), vv.data_ptr()
            T.value_index = prep.bufs['H_index'].data_ptr() if bs else None
        else:
            f = term.f
            T.kind = _lib.TD_WAVE
            T.amp_re, T.amp_im = f.amplitude.real, f.amplitude.imag
            T.omega, T.phase, T.t_center, T.sigma = f.omega, f.phase, f.t_center, f.sigma
            T.t_start, T.t_end = f.t_start, f.t_end
    ops_d = (_to_dev(np.stack([t.qarray for t in Hs.td_terms]), torch.complex64, dev)
             if Hs.td_terms else torch.zeros(1, dtype=torch.complex64, device=dev))
    jterms, disc = _jump_prefactors(jump_ops, dev, keep)
    jts = np.unique(np.concatenate([np.asarray(Hs.discontinuity_ts, dtype=np.float64)] + disc))
    jts_d = _to_dev(jts if jts.size else np.zeros(1), torch.float64, dev)
    keep += [ops_d, jts_d]
    td = _lib.TdHamiltonian(n_terms=len(Hs.td_terms), ops=ops_d.data_ptr(),
                            terms=ctypes.cast(terms, ctypes.POINTER(_lib.TdTerm)),
                            n_jump_ts=int(jts.size), jump_ts=jts_d.data_ptr(),
                            jump_terms=(ctypes.cast(jterms, ctypes.POINTER(_lib.TdTerm))
                                        if jterms is not None else None))
    prep.bufs['td'] = (td, terms, keep)

    entry = 'dqb_mesolve_dense_td' if kind == 'small' else 'dqb_mesolve_dense_large_td'

    def fn(prob, opts, outs, ws, wsb, stream):
        return getattr(lib, entry)(prob, td, opts, outs, ws, wsb, stream)

    prep.fn, prep.name = fn, entry
    return prep.launch().result()


def _td_on_dia(Hs, jump_ops, options) -> bool:
    """Whether a time-dependent H runs as one launch of the DIA stepper: every term of H and
    every jump operator in sparse-DIA storage, at most four time-dependent terms, and their
    diagonals together within the stepper's limit."""
    if options.vectorized or len(Hs.td_terms) > _lib.TD_MAX_TERMS or not Hs.is_dia:
        return False
    if not all(isinstance(_jump_source(L), SparseDIA) for L in jump_ops):
        return False
    return len(_td_union_offsets(Hs)) <= _lib.DIA_MAX_HNH_DIAGS


def _jump_prefactors(jump_ops, dev, keep):
    """The dqb_td_term array of the jump operators' prefactors c_k(t) (constant operators:
    DQB_TD_CONST), or None when none depends on time, and their discontinuity times."""
    import torch

    from .time_qarray import ModulatedTimeQArray, PWCTimeQArray

    if not any(isinstance(L, (PWCTimeQArray, ModulatedTimeQArray)) for L in jump_ops):
        return None, []
    jterms = (_lib.TdTerm * max(len(jump_ops), 1))()
    disc = []
    for k, L in enumerate(jump_ops):
        T = jterms[k]
        if isinstance(L, PWCTimeQArray):
            tt = _to_dev(L.times, torch.float64, dev)
            vv = _to_dev(np.ascontiguousarray(L.values.reshape(1, -1), dtype=np.complex128),
                         torch.complex128, dev)
            keep += [tt, vv]
            T.kind, T.n_times = _lib.TD_PWC, L.times.size
            T.times, T.values, T.value_index = tt.data_ptr(), vv.data_ptr(), None
            disc.append(np.asarray(L.discontinuity_ts, dtype=np.float64))
        elif isinstance(L, ModulatedTimeQArray):
            f = L.f
            T.kind = _lib.TD_WAVE
            T.amp_re, T.amp_im = f.amplitude.real, f.amplitude.imag
            T.omega, T.phase, T.t_center, T.sigma = f.omega, f.phase, f.t_center, f.sigma
            T.t_start, T.t_end = f.t_start, f.t_end
            disc.append(np.asarray(L.discontinuity_ts, dtype=np.float64))
        else:
            T.kind = _lib.TD_CONST
    keep.append(jterms)
    return jterms, disc


def _td_jumps_on_large(Hs, jump_ops, options) -> bool:
    """Whether time-dependent jump operators with dense operators run on the GEMM path:
    dense H (constant part and terms) and jump operators, at most four time-dependent
    terms in H."""
    if options.vectorized or len(Hs.td_terms) > _lib.TD_MAX_TERMS or options.stepper == 'krylov':
        return False
    if any(isinstance(c, SparseDIA) for c in Hs._const_src) or \
            any(isinstance(t.source, SparseDIA) for t in Hs.td_terms):
        return False
    srcs = [_jump_source(L) for L in jump_ops]
    return all(s is not None and not isinstance(s, SparseDIA) and np.ndim(s) == 2 for s in srcs)


def _jump_source(L):
    """The operator of a jump operator that is constant or one dq.pwc / dq.modulated term with
    unbatched values (None for anything else)."""
    from .time_qarray import ModulatedTimeQArray, PWCTimeQArray

    if isinstance(L, PWCTimeQArray):
        return L.source if not L.batch_shape else None
    if isinstance(L, ModulatedTimeQArray):
        return L.source
    return L if not getattr(L, '__class__', type(None)).__name__.endswith('TimeQArray') else None


def _td_union_offsets(Hs) -> tuple:
    offs = set()
    for c in Hs._const_src:
        offs.update(c.offsets)
    for t in Hs.td_terms:
        offs.update(t.source.offsets)
    return tuple(sorted(offs))


def _on_offsets(x: SparseDIA, offsets: tuple) -> np.ndarray:
    """The diagonals of ``x`` on ``offsets`` (a superset of its own), zeros elsewhere."""
    out = np.zeros((*x.diags.shape[:-2], len(offsets), x.diags.shape[-1]), np.complex64)
    for d, k in enumerate(x.offsets):
        out[..., offsets.index(k), :] += x.diags[..., d, :]
    return out


def _mesolve_td_dia(Hs, jump_ops, rho0, tsave, *, exp_ops, method, gradient, options):
    """``H(t) = H0 + sum_m c_m(t) H_m`` with every operator in sparse-DIA storage, in one
    launch of the DIA stepper (``dqb_mesolve_dia_td``): H0 and the H_m on the union of their
    offsets, the prefactors evaluated at every stage time, the steps clipped at the
    discontinuities as the reference's ``jump_ts`` does.  Batched PWC values are leading
    result dimensions (cartesian batching), as on the n <= 64 kernel."""
    import ctypes

    import torch

    from .time_qarray import PWCTimeQArray

    Ls = [_jump_source(L) for L in jump_ops]
    rho0 = _as_op(rho0)
    tsave = np.asarray(tsave.detach().cpu().numpy() if hasattr(tsave, 'detach') else tsave,
                       dtype=np.float64)
    if exp_ops is not None:
        exp_ops = [_as_op(E) for E in exp_ops] if len(exp_ops) > 0 else None
    offs = _td_union_offsets(Hs)
    n = Hs.constant.shape[-1]
    bs = tuple(Hs.batch_shape)
    if bs and not options.cartesian_batching:
        raise NotImplementedError('Batched PWC values need cartesian batching on the B200 path.')
    h0 = sum(_on_offsets(c, offs) for c in Hs._const_src) if Hs._const_src else \
        np.zeros((len(offs), n), np.complex64)
    Hb = SparseDIA(offs, np.ascontiguousarray(np.broadcast_to(h0, (*bs, len(offs), n))))
    _check_mesolve_args(Hb, Ls, rho0, exp_ops)
    tsave = check_times(tsave, 'tsave')
    check_options(options, 'mesolve')
    options = options.initialise()
    assert_method_supported(method)
    method.assert_supports_gradient(gradient)
    if options.stepper == 'krylov':
        raise NotImplementedError('The Krylov form needs a constant Hamiltonian.')
    plan = make_batch_plan(Hb, Ls, rho0, True)
    integ = MESolveB200Integrator(ts=tsave, y0=rho0, method=method, gradient=gradient,
                                  options=options, H=Hb, Ls=Ls, Es=exp_ops, plan=plan)
    lib = _lib.load()
    prep = integ._prepare_dia(lib)
    dev = prep.dev
    nsets = int(np.prod(bs, dtype=np.int64)) if bs else 1
    terms = (_lib.TdTerm * _lib.TD_MAX_TERMS)()
    keep = []
    for m, term in enumerate(Hs.td_terms):
        T = terms[m]
        if isinstance(term, PWCTimeQArray):
            vals = np.broadcast_to(term.values, (*bs, term.values.shape[-1])).reshape(nsets, -1)
            tt = _to_dev(term.times, torch.float64, dev)
            vv = _to_dev(np.ascontiguousarray(vals, dtype=np.complex128), torch.complex128, dev)
            keep += [tt, vv]
            T.kind, T.n_times = _lib.TD_PWC, term.times.size
            T.times, T.values = tt.data_ptr(), vv.data_ptr()
            T.value_index = prep.bufs['H_index'].data_ptr() if bs else None
        else:
            f = term.f
            T.kind = _lib.TD_WAVE
            T.amp_re, T.amp_im = f.amplitude.real, f.amplitude.imag
            T.omega, T.phase, T.t_center, T.sigma = f.omega, f.phase, f.t_center, f.sigma
            T.t_start, T.t_end = f.t_start, f.t_end
    ops_d = (_to_dev(np.stack([_on_offsets(t.source, offs) for t in Hs.td_terms]), torch.complex64, dev)
             if Hs.td_terms else torch.zeros(1, dtype=torch.complex64, device=dev))
    # prefactors of the jump operators (constant ones: 1)
    jterms, disc = _jump_prefactors(jump_ops, dev, keep)
    jts = np.unique(np.concatenate([np.asarray(Hs.discontinuity_ts, dtype=np.float64)] + disc))
    jts_d = _to_dev(jts if jts.size else np.zeros(1), torch.float64, dev)
    keep += [ops_d, jts_d]
    td = _lib.TdHamiltonian(n_terms=len(Hs.td_terms), ops=ops_d.data_ptr(),
                            terms=ctypes.cast(terms, ctypes.POINTER(_lib.TdTerm)),
                            n_jump_ts=int(jts.size), jump_ts=jts_d.data_ptr(),
                            jump_terms=(ctypes.cast(jterms, ctypes.POINTER(_lib.TdTerm))
                                        if jterms is not None else None))
    prep.bufs['td'] = (td, terms, jterms, keep)

    def fn(prob, opts, outs, ws, wsb, stream):
        return lib.dqb_mesolve_dia_td(prob, td, opts, outs, ws, wsb, stream)

    prep.fn, prep.name = fn, 'dqb_mesolve_dia_td'
    return prep.launch().result()


def _mesolve_piecewise(H, jump_ops, rho0, tsave, *, exp_ops, method, gradient, options, solve):
    """Solve with a piecewise-constant H (``time_qarray``): one constant-operator ``solve``
    per piece between consecutive discontinuities, each started from the previous piece's
    final state; saved states, expectation values and step counts are stitched together
    into one result over ``tsave``.  ``solve`` has ``mesolve``'s signature (the oracle's
    stand-in in the CPU tests)."""
    import dataclasses

    from .time_qarray import as_summed, piecewise_plan

    Hs = as_summed(H)
    if Hs.batch_shape:
        if not options.cartesian_batching:
            raise NotImplementedError('Batched PWC values need cartesian batching on the B200 '
                                      'path.')
        rs = [_mesolve_piecewise(Hs.item(idx), jump_ops, rho0, tsave, exp_ops=exp_ops,
                                 method=method, gradient=gradient, options=options, solve=solve)
              for idx in np.ndindex(*Hs.batch_shape)]
        stack = _stack_like(rs[0].states)
        shape = Hs.batch_shape

        def stacked(xs):
            out = stack(xs)
            return out.reshape(*shape, *out.shape[1:])

        r0 = rs[0]
        return MESolveResult(
            tsave=r0.tsave, method=method, gradient=gradient, options=options,
            states=stacked([r.states for r in rs]),
            expects=stacked([r.expects for r in rs]) if r0.expects is not None else None,
            infos=AdaptiveStepInfos(stacked([r.infos.nsteps for r in rs]),
                                    stacked([r.infos.naccepted for r in rs]),
                                    stacked([r.infos.nrejected for r in rs])))
    tsave = check_times(np.asarray(tsave.detach().cpu().numpy() if hasattr(tsave, 'detach')
                                   else tsave, dtype=np.float64), 'tsave')
    t0 = float(tsave[0] if options.t0 is None else options.t0)
    if t0 > tsave[0]:
        # the pieces start at t0: save points before it would be dropped silently
        raise ValueError(f'Option `t0` ({t0}) must not be after the first save time '
                         f'tsave[0] ({tsave[0]}) with a piecewise-constant Hamiltonian.')
    piece_opts = dataclasses.replace(options, t0=None)
    states, expects, infos = [], [], None
    state = rho0
    for _a, _b, Hc, ts, keep in piecewise_plan(Hs, tsave, t0):
        r = solve(Hc, jump_ops, state, ts, exp_ops=exp_ops, method=method, gradient=gradient,
                  options=piece_opts)
        if options.save_states:
            states.append(r.states[..., keep, :, :])
        if r.expects is not None:
            expects.append(r.expects[..., keep])
        state = r.states[..., -1, :, :]
        i = (r.infos.nsteps, r.infos.naccepted, r.infos.nrejected)
        infos = i if infos is None else tuple(x + y for x, y in zip(infos, i))
    cat = _concatenate_like(state)
    out_states = cat(states, -3) if options.save_states else state[..., None, :, :]
    out_expects = cat(expects, -1) if expects else None
    return MESolveResult(tsave=tsave, method=method, gradient=gradient, options=options,
                         states=out_states, expects=out_expects,
                         infos=AdaptiveStepInfos(*infos))


def _stack_like(x):
    if hasattr(x, 'detach'):
        import torch

        return lambda xs: torch.stack([torch.as_tensor(v) for v in xs])
    return lambda xs: np.stack([np.asarray(v) for v in xs])


def _concatenate_like(x):
    if hasattr(x, 'detach'):
        import torch

        return lambda xs, axis: torch.cat(list(xs), dim=axis)
    return lambda xs, axis: np.concatenate(list(xs), axis=axis)


def _prod(shape) -> int:
    return int(math.prod(shape)) if shape else 1
