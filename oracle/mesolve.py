"""CPU restatement (test infrastructure only) of one ``dq.mesolve`` instance.

Follows ``dynamiqs/integrators/apis/mesolve.py:62-304`` (argument handling) for a single
unbatched problem, ``MESolveDiffraxIntegrator`` (``dynamiqs/integrators/core/
diffrax_integrator.py:283-352``: vector field choice and ``__post_init__``),
``DiffraxIntegrator.run`` (``:135-147``), and the saving rules of ``SolveSaveMixin``
(``dynamiqs/integrators/core/save_mixin.py:44-68``): states at every ``tsave`` (or the
final state only when ``save_states=False``), expectation values ``tr(E rho)`` stacked
as ``(nE, ntsave)``, and ``(nsteps, naccepted, nrejected)`` infos
(``diffrax_integrator.py:149-157``).  Imported by tests and bench CPU legs only.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import lindblad as lb
from .rk import solve


@dataclass
class OracleResult:
    states: np.ndarray  # (nsave, n, n)
    expects: np.ndarray | None  # (nE, ntsave)
    nsteps: int
    naccepted: int
    nrejected: int
    status: int
    final_state: np.ndarray
    errors: list  # (t, h, scaled error) of every attempted step


def _as_dense(op, n):
    if isinstance(op, tuple):
        return lb.dia_to_dense(*op)
    return np.asarray(op)


def mesolve(H, Ls, rho0, tsave, exp_ops=None, *, method='Tsit5', rtol=1e-6, atol=1e-6,
            safety=0.9, factormin=0.2, factormax=5.0, max_steps=100_000, t0=None,
            save_states=True, form='hermitian', dtype=np.complex128,
            time_dtype=np.float64, jump_ts=None) -> OracleResult:
    """Solve one Lindblad problem.  ``H`` and each ``L`` are dense arrays or DIA
    ``(offsets, diags)`` tuples; ``rho0`` is a ket ``(n, 1)`` or a density matrix.  A
    callable ``H`` is a time-dependent Hamiltonian ``t -> (n, n)`` (``TimeQArray.__call__``,
    dynamiqs/time_qarray.py:430-451), solved in the hermitian form with ``jump_ts`` handed
    to the step-size controller (``diffrax_integrator.py:59-72``)."""
    rho0 = np.asarray(rho0, dtype=dtype)
    n = rho0.shape[-2]
    if rho0.shape[-1] == 1:  # todm (dynamiqs/utils/general.py:821)
        rho0 = rho0 @ lb.dag(rho0)
    dia = isinstance(H, tuple) or any(isinstance(L, tuple) for L in Ls)
    time_dependent = callable(H) and not isinstance(H, (np.ndarray, tuple))
    Hd = None if time_dependent else _as_dense(H, n).astype(dtype)
    Lsd = [_as_dense(L, n).astype(dtype) for L in Ls]
    if time_dependent:
        if form != 'hermitian':
            raise ValueError('time-dependent H: hermitian form only')
        LsH = [lb.dag(L) for L in Lsd]

        def f(t, y):
            Hnh = lb.hnh_dense(np.asarray(H(t), dtype=dtype), Lsd)
            tmp = Hnh @ y
            for L, Lh in zip(Lsd, LsH):
                tmp = tmp + 0.5 * (L @ y @ Lh)
            return tmp + lb.dag(tmp)
        y0 = rho0
        unvec = lambda y: y  # noqa: E731
    elif form == 'hermitian':
        if dia:
            Hdia = H if isinstance(H, tuple) else lb.dense_to_dia(Hd)
            Ldia = [L if isinstance(L, tuple) else lb.dense_to_dia(Ld)
                    for L, Ld in zip(Ls, Lsd)]
            Hdia = (Hdia[0], Hdia[1].astype(dtype))
            Ldia = [(o, d.astype(dtype)) for o, d in Ldia]

            def f(t, y):
                return lb.vf_hermitian_dia(Hdia, Ldia, y)
        else:
            Hnh = lb.hnh_dense(Hd, Lsd)
            LsH = [lb.dag(L) for L in Lsd]

            def f(t, y):
                tmp = Hnh @ y
                for L, Lh in zip(Lsd, LsH):
                    tmp = tmp + 0.5 * (L @ y @ Lh)
                return tmp + lb.dag(tmp)
        y0 = rho0
        unvec = lambda y: y  # noqa: E731
    elif form == 'standard':
        def f(t, y):
            return lb.vf_standard(Hd, Lsd, y)
        y0 = rho0
        unvec = lambda y: y  # noqa: E731
    elif form == 'vectorized':
        S = lb.slindbladian(Hd, Lsd).astype(dtype)

        def f(t, y):
            return S @ y
        y0 = lb.vectorize(rho0)
        unvec = lb.unvectorize
    else:
        raise ValueError(form)

    Es = [np.asarray(_as_dense(E, n), dtype=dtype) for E in (exp_ops or [])]

    def save_fn(y):
        rho = unvec(y)
        e = np.array([lb.expect(E, rho) for E in Es]) if Es else None
        return rho, e

    out = solve(f, y0, tsave, method=method, rtol=rtol, atol=atol, safety=safety,
                factormin=factormin, factormax=factormax, max_steps=max_steps, t0=t0,
                time_dtype=time_dtype, save_fn=save_fn, jump_ts=jump_ts)
    final = unvec(out.ylast)
    if out.ysave:
        states = np.stack([s[0] for s in out.ysave])
        expects = np.stack([s[1] for s in out.ysave], axis=-1) if Es else None
    else:
        states = final[None]
        expects = None
    if not save_states:
        states = final[None]
    return OracleResult(states, expects, out.nsteps, out.naccepted, out.nrejected,
                        out.status, final, out.errors)


def sesolve(H, psi0, tsave, *, method='Tsit5', rtol=1e-6, atol=1e-6, dtype=np.complex128,
            time_dtype=np.float64, **kw):
    """Schroedinger equation d psi/dt = -i H psi (``diffrax_integrator.py:221-228``);
    used only to pin the shared RK engine against the reference docs' Dopri5 example."""
    Hd = np.asarray(H, dtype=dtype)
    out = solve(lambda t, y: -1j * (Hd @ y), np.asarray(psi0, dtype=dtype), tsave,
                method=method, rtol=rtol, atol=atol, time_dtype=time_dtype, **kw)
    return out
