"""``dq.sesolve`` on the GPU: the Schroedinger equation d psi/dt = -i H psi on the same
Runge-Kutta engine as ``mesolve`` (``dynamiqs/integrators/apis/sesolve.py:35-330``;
vector field ``dynamiqs/integrators/core/diffrax_integrator.py:221-228``), through one
C-ABI call (``dqb_sesolve_dense``, ``include/dqb200.h``) for the whole batch.

Same signature, argument checks and batching semantics as the reference: ``H`` of shape
``(...H, n, n)``, ``psi0`` ``(...psi0, n, 1)``, ``tsave`` ``(ntsave,)``, ``exp_ops`` a
list of ``(n, n)``; cartesian batching gives results of shape ``(...H, ...psi0, ...)``,
flat batching broadcasts ``...H`` against ``...psi0``.  ``method`` is ``Tsit5`` (default)
or ``Dopri5``.  Three kernels, by size: n <= 128 one warp per instance
(``dqb_sesolve_dense``; sparse-DIA ``H`` is densified); n up to 8192 the batched
large-problem stepper with a dense ``H`` (``dqb_sesolve_dense_large``) or with ``H`` kept in
sparse-DIA storage (``dqb_sesolve_dia``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from .mesolve import (_as_op, _check_shape, _device, _MAX_STEPS_MSG, _shape, _to_dev,
                      assert_method_supported, check_times, make_batch_plan)
from .method import Method, Tsit5
from .options import Options, check_options
from .qarrays import SparseDIA, to_dense
from .result import AdaptiveStepInfos, MESolveResult

__all__ = ['sesolve', 'SESolveResult', 'SESolveB200Integrator']


class SESolveResult(MESolveResult):
    """``dynamiqs/result.py`` SESolveResult: ``states`` ``(..., nsave, n, 1)``,
    ``final_state`` ``(..., n, 1)``, ``expects`` ``(..., nE, ntsave)``, ``infos``."""


def _check_sesolve_args(H, psi0, exp_ops) -> None:
    """``_check_sesolve_args`` (``sesolve.py:318-330``)."""
    _check_shape(H, 'H', '(..., n, n)', subs={'...': '...H'})
    _check_shape(psi0, 'psi0', '(..., n, 1)', subs={'...': '...psi0'})
    if exp_ops is not None:
        for i, E in enumerate(exp_ops):
            _check_shape(E, f'exp_ops[{i}]', '(n, n)')


# largest n of the warp-per-instance kernel and of the large-problem stepper
WARP_MAX_N = 128
LARGE_MAX_N = 8192


@dataclass
class _Prepared:
    integ: 'SESolveB200Integrator'
    prob: object
    outs: object
    bufs: dict
    fn: str = 'dqb_sesolve_dense'
    host: tuple = ()  # host arrays the problem struct points to
    td: object = None  # the dqb_td_hamiltonian of a time-dependent H

    def launch(self, stream=None):
        import ctypes

        import torch

        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        lib = _lib.load()
        head = (ctypes.byref(self.prob),) + ((ctypes.byref(self.td),) if self.td is not None else ())
        rc = getattr(lib, self.fn)(*head, ctypes.byref(self.integ._ode_options()),
                                   ctypes.byref(self.outs), self.bufs['workspace'].data_ptr(),
                                   self.bufs['workspace'].numel(), s)
        _lib.check(rc, self.fn)
        return self

    def result(self) -> SESolveResult:
        return self.integ._result(self.bufs)


class SESolveB200Integrator:
    """Registry-compatible integrator: ``constructor(ts=, y0=, method=, gradient=,
    options=, H=, Es=)`` then ``.run() -> SESolveResult`` (``sesolve.py:289-304``)."""

    def __init__(self, *, ts, y0, method, gradient, options, H, Es, plan, td=None):
        self.td = td  # a time-dependent H (SummedTimeQArray): H is then its constant part
        self.ts = ts
        self.y0 = y0
        self.method = method
        self.gradient = gradient
        self.options = options
        self.H = H
        self.plan = plan
        # the identity's expectation value <psi|psi> (FP64 sums) is the norm check; with H
        # in DIA storage (large n) a dense identity would cost more than the solve, so the
        # norm is taken from the returned states instead
        self._n_user_E = len(Es) if Es else 0
        self._norm_from_states = self.path == 'dia'
        self.Es = list(Es or []) + ([] if self._norm_from_states
                                    else [np.eye(_shape(H)[-1], dtype=np.complex64)])

    @property
    def t0(self) -> float:
        return float(self.ts[0] if self.options.t0 is None else self.options.t0)

    def _ode_options(self) -> _lib.OdeOptions:
        m = self.method
        return _lib.OdeOptions(
            method=_lib.METHOD_TSIT5 if isinstance(m, Tsit5) else _lib.METHOD_DOPRI5,
            form=_lib.FORM_STANDARD, rtol=float(m.rtol), atol=float(m.atol),
            safety=float(m.safety_factor), factormin=float(m.min_factor),
            factormax=float(m.max_factor), max_steps=int(m.max_steps), t0=self.t0,
            save_states=int(bool(self.options.save_states)), check_hermitian=0)

    @property
    def path(self) -> str:
        """'warp' (n <= 128), 'dia' (sparse-DIA H beyond that) or 'dense_large'."""
        n = _shape(self.H)[-1]
        if n <= WARP_MAX_N and self.td is None:
            return 'warp'
        return 'dia' if isinstance(self.plan.H_items, SparseDIA) else 'dense_large'

    def prepare(self) -> _Prepared:
        import ctypes

        import torch

        dev = _device()
        plan = self.plan
        n = _shape(self.H)[-1]
        ntsave = len(self.ts)
        nE = len(self.Es) if self.Es else 0
        nsave = ntsave if self.options.save_states else 1
        B = plan.batch
        c64 = torch.complex64
        path = self.path
        lib = _lib.load()
        dia = path == 'dia'
        if path == 'warp':
            ws_bytes = lib.dqb_sesolve_dense_workspace_size()
        elif self.td is not None:
            hv = len(plan.H_items.offsets) * n if dia else n * n
            ws_bytes = lib.dqb_sesolve_large_td_workspace_size(n, hv, nE, ntsave, B)
        else:
            ws_bytes = lib.dqb_sesolve_large_workspace_size(n, nE, ntsave, B)
        if ws_bytes == 0:
            raise NotImplementedError(f'sesolve on the B200 path supports n <= {LARGE_MAX_N}.')
        bufs = {
            'H': _to_dev(plan.H_items.diags if dia else plan.H_items_dense(), c64, dev),
            'psi0': _to_dev(plan.rho_items, c64, dev),
            'E': (_to_dev(np.stack([to_dense(E) for E in self.Es]), c64, dev) if nE
                  else torch.zeros(1, dtype=c64, device=dev)),
            'tsave': _to_dev(np.asarray(self.ts, dtype=np.float64), torch.float64, dev),
            'H_index': _to_dev(plan.H_index, torch.int32, dev),
            'psi0_index': _to_dev(plan.rho_index, torch.int32, dev),
            'states': torch.empty((B, nsave, n, 1), dtype=c64, device=dev),
            'expects': torch.empty((B, max(nE, 1), ntsave), dtype=c64, device=dev),
            'infos': torch.empty((B, 3), dtype=torch.int32, device=dev),
            'status': torch.empty((B,), dtype=torch.int32, device=dev),
            'workspace': torch.empty(ws_bytes, dtype=torch.uint8, device=dev),
        }
        host = ()
        if dia:
            offs = tuple(int(k) for k in plan.H_items.offsets)
            h_off = (ctypes.c_int32 * max(len(offs), 1))(*offs)
            host = (h_off,)
            prob = _lib.DiaProblem(
                n=n, n_jumps=0, n_exp=nE, n_tsave=ntsave, batch=B, h_ndiag=len(offs),
                h_offsets=ctypes.cast(h_off, ctypes.c_void_p), h_diags=bufs['H'].data_ptr(),
                l_ndiag=None, l_offsets=None, l_diags=None, rho0=bufs['psi0'].data_ptr(),
                rho0_is_ket=1, E=bufs['E'].data_ptr(), tsave=bufs['tsave'].data_ptr(),
                H_index=bufs['H_index'].data_ptr(), L_index=None,
                rho0_index=bufs['psi0_index'].data_ptr())
        else:
            prob = _lib.DenseProblem(
                n=n, n_jumps=0, n_exp=nE, n_tsave=ntsave, batch=B, H=bufs['H'].data_ptr(), L=None,
                rho0=bufs['psi0'].data_ptr(), rho0_is_ket=1, E=bufs['E'].data_ptr(),
                tsave=bufs['tsave'].data_ptr(), H_index=bufs['H_index'].data_ptr(), L_index=None,
                rho0_index=bufs['psi0_index'].data_ptr())
        outs = _lib.Outputs(states=bufs['states'].data_ptr(), expects=bufs['expects'].data_ptr(),
                            infos=bufs['infos'].data_ptr(), status=bufs['status'].data_ptr())
        self._nE = nE
        fn = {'warp': 'dqb_sesolve_dense', 'dense_large': 'dqb_sesolve_dense_large',
              'dia': 'dqb_sesolve_dia'}[path]
        td = None
        if self.td is not None:
            td, keep = _td_struct(self.td, plan, bufs, dev, dia)
            host = host + (keep,)
            fn += '_td'
        return _Prepared(self, prob, outs, bufs, fn, host, td)

    def run(self) -> SESolveResult:
        return self.prepare().launch().result()

    def _result(self, b) -> SESolveResult:
        st = b['status'].cpu()
        if bool((st == _lib.INST_MAX_STEPS).any()):
            raise RuntimeError(_MAX_STEPS_MSG)
        if bool((st == _lib.INST_NONFINITE).any()):
            raise RuntimeError('The solution became non-finite (NaN or inf) during the '
                               'integration.')
        bshape = self.plan.bshape
        states = b['states'].reshape(*bshape, *b['states'].shape[1:])
        ex = b['expects'].reshape(*bshape, *b['expects'].shape[1:])
        expects = ex[..., :self._n_user_E, :] if self._n_user_E else None
        import torch

        if self._norm_from_states:  # (..., nsave): every saved state, or the final one
            sd = states.to(torch.complex128)
            checks = {'norm': (sd.abs() ** 2).sum(dim=(-2, -1))}
        else:
            checks = {'norm': ex[..., self._n_user_E, :].to(torch.complex128).real}
        infos = b['infos'].reshape(*bshape, 3)
        info = AdaptiveStepInfos(infos[..., 0], infos[..., 1], infos[..., 2])
        extra = None
        if self.options.save_extra is not None:  # applied to every saved state
            import torch

            if not self.options.save_states:
                raise NotImplementedError('`save_extra` needs `save_states=True` on the '
                                          'B200 path (it is applied to the saved states).')
            vals = [self.options.save_extra(x) for x in states.reshape(-1, *states.shape[-2:])]
            try:
                extra = torch.stack([torch.as_tensor(v) for v in vals]).reshape(
                    *states.shape[:-2], *torch.as_tensor(vals[0]).shape)
            except (TypeError, RuntimeError):
                extra = vals
        return SESolveResult(tsave=self.ts, method=self.method, gradient=self.gradient,
                             options=self.options, states=states, expects=expects, infos=info,
                             extra=extra, checks=checks)


def _td_struct(Hs, plan, bufs, dev, dia):
    """The dqb_td_hamiltonian of a time-dependent H: its terms' prefactors (batched PWC
    values indexed by the instance's H index) and operators in the layout of the constant
    part (dense, or diagonals on its offsets)."""
    import ctypes

    import torch

    from .mesolve import _on_offsets
    from .time_qarray import PWCTimeQArray

    bs = tuple(Hs.batch_shape)
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
            T.value_index = bufs['H_index'].data_ptr() if bs else None
        else:
            f = term.f
            T.kind = _lib.TD_WAVE
            T.amp_re, T.amp_im = f.amplitude.real, f.amplitude.imag
            T.omega, T.phase, T.t_center, T.sigma = f.omega, f.phase, f.t_center, f.sigma
            T.t_start, T.t_end = f.t_start, f.t_end
    if dia:
        offs = tuple(plan.H_items.offsets)
        ops = np.stack([_on_offsets(t.source, offs) for t in Hs.td_terms])
    else:
        ops = np.stack([t.qarray for t in Hs.td_terms])
    ops_d = _to_dev(ops, torch.complex64, dev)
    jts = np.asarray(Hs.discontinuity_ts, dtype=np.float64)
    jts_d = _to_dev(jts if jts.size else np.zeros(1), torch.float64, dev)
    keep += [ops_d, jts_d, terms]
    td = _lib.TdHamiltonian(n_terms=len(Hs.td_terms), ops=ops_d.data_ptr(),
                            terms=ctypes.cast(terms, ctypes.POINTER(_lib.TdTerm)),
                            n_jump_ts=int(jts.size), jump_ts=jts_d.data_ptr())
    return td, keep


def _sesolve_td(Hs, psi0, tsave, *, exp_ops, method, gradient, options) -> SESolveResult:
    """A time-dependent H (``dq.pwc`` / ``dq.modulated`` sums, at most four terms, every
    operator dense or every one sparse-DIA) in one launch of the large-problem stepper at
    any n: H(t) formed at every stage time, the steps clipped at the discontinuities as the
    reference's ``jump_ts`` does; batched PWC values are leading result dimensions."""
    from .mesolve import _td_union_offsets, _on_offsets
    from .time_qarray import as_summed

    Hs = as_summed(Hs)
    if len(Hs.td_terms) > _lib.TD_MAX_TERMS:
        raise NotImplementedError(f'At most {_lib.TD_MAX_TERMS} time-dependent terms on the B200 '
                                  'path.')
    psi0 = _as_op(psi0)
    tsave = np.asarray(tsave.detach().cpu().numpy() if hasattr(tsave, 'detach') else tsave,
                       dtype=np.float64)
    if exp_ops is not None:
        exp_ops = [_as_op(E) for E in exp_ops] if len(exp_ops) > 0 else None
    n = Hs.constant.shape[-1]
    bs = tuple(Hs.batch_shape)
    if bs and not options.cartesian_batching:
        raise NotImplementedError('Batched PWC values need cartesian batching on the B200 path.')
    if Hs.is_dia:
        offs = _td_union_offsets(Hs)
        h0 = sum(_on_offsets(c, offs) for c in Hs._const_src) if Hs._const_src else \
            np.zeros((len(offs), n), np.complex64)
        H = SparseDIA(offs, np.ascontiguousarray(np.broadcast_to(h0, (*bs, len(offs), n))))
    else:
        H = np.ascontiguousarray(np.broadcast_to(Hs.constant.astype(np.complex64), (*bs, n, n)))
    _check_sesolve_args(H, psi0, exp_ops)
    tsave = check_times(tsave, 'tsave')
    check_options(options, 'sesolve')
    options = options.initialise()
    assert_method_supported(method)
    method.assert_supports_gradient(gradient)
    if n > LARGE_MAX_N:
        raise NotImplementedError(f'sesolve on the B200 path supports n <= {LARGE_MAX_N}.')
    if _shape(psi0)[-2] != n:
        raise ValueError(f'Argument `psi0` must have shape (..., {n}, 1).')
    plan = make_batch_plan(H, [], psi0, True)
    integ = SESolveB200Integrator(ts=tsave, y0=psi0, method=method, gradient=gradient,
                                  options=options, H=H, Es=exp_ops, plan=plan, td=Hs)
    return integ.run()


def sesolve(H, psi0, tsave, *, exp_ops=None, method: Method = Tsit5(),  # noqa: B008
            gradient=None, options: Options = Options()) -> SESolveResult:  # noqa: B008
    r"""Solve the Schroedinger equation d psi/dt = -i H psi on the GPU (``dq.sesolve``,
    ``dynamiqs/integrators/apis/sesolve.py:35-224``).  Returns a :class:`SESolveResult`
    with ``states`` ``(..., nsave, n, 1)`` and ``expects`` ``(..., nE, ntsave)``.  ``H`` may
    be time-dependent (``dq.pwc`` / ``dq.modulated`` sums with a ``Wave`` prefactor)."""
    from .time_qarray import ModulatedTimeQArray, PWCTimeQArray, SummedTimeQArray

    if isinstance(H, (PWCTimeQArray, ModulatedTimeQArray, SummedTimeQArray)):
        return _sesolve_td(H, psi0, tsave, exp_ops=exp_ops, method=method, gradient=gradient,
                           options=options)
    if getattr(H, '__class__', None).__name__.endswith('TimeQArray'):
        raise NotImplementedError('Callable time-dependent operators cannot run inside the B200 '
                                  'kernels: use dq.pwc or dq.modulated with a Wave prefactor.')
    H = _as_op(H)
    psi0 = _as_op(psi0)
    tsave = np.asarray(tsave.detach().cpu().numpy() if hasattr(tsave, 'detach') else tsave,
                       dtype=np.float64)
    if exp_ops is not None:
        exp_ops = [_as_op(E) for E in exp_ops] if len(exp_ops) > 0 else None

    _check_sesolve_args(H, psi0, exp_ops)
    tsave = check_times(tsave, 'tsave')
    check_options(options, 'sesolve')
    options = options.initialise()
    assert_method_supported(method)
    method.assert_supports_gradient(gradient)

    n = _shape(H)[-1]
    if _shape(psi0)[-2] != n:
        raise ValueError(f'Argument `psi0` must have shape (..., {n}, 1).')
    if n > LARGE_MAX_N:
        raise NotImplementedError(f'sesolve on the B200 path supports n <= {LARGE_MAX_N}.')
    if n <= WARP_MAX_N or not isinstance(H, SparseDIA):
        H = to_dense(H) if not isinstance(H, np.ndarray) else H
    plan = make_batch_plan(H, [], psi0, options.cartesian_batching)
    integ = SESolveB200Integrator(ts=tsave, y0=psi0, method=method, gradient=gradient,
                                  options=options, H=H, Es=exp_ops, plan=plan)
    return integ.run()
