"""CPU restatement (test infrastructure only) of the adaptive Runge-Kutta loop that
dynamiqs' ``mesolve`` delegates to diffrax.

This module is the ORACLE: it is imported by ``tests/``, by ``__graft_entry__.smoke()``
and by the ``cpu_baseline``/reference legs of ``bench.py`` only, always as the checker.
The product path (``dynamiqs_b200``) never imports it.

What is restated, and from where
--------------------------------
dynamiqs builds the vector field and hands the loop to ``diffrax.diffeqsolve``
(``dynamiqs/integrators/core/diffrax_integrator.py:101-133``) with

* ``PIDController(rtol, atol, safety, factormin, factormax, jump_ts)``
  (``diffrax_integrator.py:59-72``), defaults ``rtol=atol=1e-6, safety=0.9,
  factormin=0.2, factormax=5.0, max_steps=100_000`` (``dynamiqs/method.py:121-127``);
* ``dt0=None`` so the first step comes from the automatic initial-step heuristic
  (``diffrax_integrator.py:74-76``);
* ``SaveAt(subs=[SubSaveAt(ts=tsave, fn=save), SubSaveAt(t1=True)])``
  (``diffrax_integrator.py:135-147``): states at ``tsave`` through the solver's dense
  interpolant, plus the final state;
* solver ``dx.Tsit5()`` or ``dx.Dopri5()`` (``diffrax_integrator.py:361-378``).

diffrax itself (``pyproject.toml:30``: ``diffrax>=0.6.1``, unpinned, no lock file) is
not vendored in the reference. Its arithmetic is restated here from the published
methods it implements:

* Tsit5: Ch. Tsitouras, "Runge-Kutta pairs of order 5(4) satisfying only the first
  column simplifying assumption", Comput. Math. Appl. 62 (2011) 770-775 -- tableau,
  embedded 4th-order weights and the continuous extension b_i(theta).
* Dopri5: J. R. Dormand, P. J. Prince, "A family of embedded Runge-Kutta formulae",
  J. Comput. Appl. Math. 6 (1980) 19-26 -- tableau; the error estimate uses the
  alternative fourth-order embedded weights (1951/21600, 0, 22642/50085, 451/720,
  -12231/42400, 649/6300, 1/60), which satisfy every order-4 condition of the same
  tableau (checked in tests/test_oracle_tableau.py); dense output is the quartic
  through y0, y1, f0, f1 and L. F. Shampine's midpoint value ("Some practical
  Runge-Kutta formulas", Math. Comp. 46 (1986) 135-150).
* Initial step: Hairer, Norsett, Wanner, "Solving ODEs I", 2nd ed., Sec. II.4
  (the "starting step size" algorithm), with the RMS norm and the exponent 1/4 in its
  last stage, h1 = (0.01 / max(d1, d2))^(1/4).
* Step-size control: integral controller h_new = h * clip(safety * err^(-1/q),
  fmin, fmax) with q = 5 (order of the embedded pair's error estimate, min(p,q)+1 for
  a 5(4) pair), where a step is kept when err < 1, and an accepted step never shrinks
  the next step (fmin is 1 on acceptance, ``factormin`` on rejection).
* Error norm: RMS over every complex entry of e / (atol + rtol * max(|y0|, |y1|)).
* End of interval: the trial end time is clipped to t1 when it lies within 1e-10
  (float64 time) or 1e-6 (float32 time) of t1.

Parity pins (tests/test_oracle_known_answers.py): the step counts printed by the
reference's own docs (README.md:48-76 "40 steps (40 accepted, 0 rejected)";
dynamiqs/integrators/apis/mesolve.py:204-227 "9 steps (9 accepted, 0 rejected)";
docs/documentation/basics/workflow.md:50-88 Dopri5 "56 steps (48 accepted,
8 rejected)"), all three reproduced exactly, and the analytic solutions used by the
reference's tests (tests/systems/open_system.py:172-182).  The two choices above
that are not fixed by the published methods alone -- the starting-step exponent and
Dopri5's embedded weights -- are the only combination of (controller exponent 1/4
or 1/5, starting-step exponent 1/3..1/6, accepted steps allowed to shrink or not, RMS
over complex entries or over real and imaginary parts, either Dopri5 embedded set)
that reproduces all three counts, with float32 and with float64 time alike; with
exponent 1/5 and the 5179/57600 weights the counts are 39, 8 and 59 (51 accepted).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

import numpy as np

# --------------------------------------------------------------------------------------
# Butcher tableaux
# --------------------------------------------------------------------------------------


@dataclass(frozen=True)
class Tableau:
    name: str
    c: np.ndarray  # (7,)
    a: np.ndarray  # (7, 7) strictly lower triangular; row 6 == b (FSAL)
    b: np.ndarray  # (7,) 5th-order weights
    btilde: np.ndarray  # (7,) b - bhat (error weights)
    order: int = 5
    error_order: int = 5  # controller exponent 1/error_order
    start_exponent: float = 0.25  # exponent of the starting step's last stage


def _tsit5() -> Tableau:
    c = np.array([0.0, 0.161, 0.327, 0.9, 0.9800255409045097, 1.0, 1.0])
    a = np.zeros((7, 7))
    a[1, 0] = 0.161
    a[2, :2] = [-0.008480655492356989, 0.335480655492357]
    a[3, :3] = [2.897153057105493, -6.359448489975075, 4.3622954328695815]
    a[4, :4] = [5.325864828439257, -11.748883564062828, 7.4955393428898365,
                -0.09249506636175525]
    a[5, :5] = [5.86145544294642, -12.92096931784711, 8.159367898576159,
                -0.071584973281401, -0.028269050394068383]
    a[6, :6] = [0.09646076681806523, 0.01, 0.4798896504144996, 1.379008574103742,
                -3.290069515436081, 2.324710524099774]
    b = a[6].copy()
    btilde = np.array([-0.001780011052226, -0.000816434459657, 0.007880878010262,
                       -0.144711007173263, 0.582357165452555, -0.458082105929187,
                       1.0 / 66.0])
    return Tableau('Tsit5', c, a, b, btilde)


def _dopri5() -> Tableau:
    c = np.array([0.0, 1 / 5, 3 / 10, 4 / 5, 8 / 9, 1.0, 1.0])
    a = np.zeros((7, 7))
    a[1, 0] = 1 / 5
    a[2, :2] = [3 / 40, 9 / 40]
    a[3, :3] = [44 / 45, -56 / 15, 32 / 9]
    a[4, :4] = [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729]
    a[5, :5] = [9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656]
    a[6, :6] = [35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84]
    b = a[6].copy()
    bhat = np.array([1951 / 21600, 0.0, 22642 / 50085, 451 / 720, -12231 / 42400,
                     649 / 6300, 1 / 60])
    return Tableau('Dopri5', c, a, b, b - bhat)


TSIT5 = _tsit5()
DOPRI5 = _dopri5()

# Shampine's midpoint weights for Dopri5 (y(t0 + h/2) = y0 + h * sum c_mid_i k_i).
DOPRI5_C_MID = np.array([
    6025192743 / 30085553152 / 2, 0.0, 51252292925 / 65400821598 / 2,
    -2691868925 / 45128329728 / 2, 187940372067 / 1594534317056 / 2,
    -1776094331 / 19743644256 / 2, 11237099 / 235043384 / 2,
])


def tsit5_dense_weights(theta: float) -> np.ndarray:
    """Tsitouras' continuous extension b_i(theta), i = 1..7 (Tsitouras 2011)."""
    t = theta
    t2 = t * t
    return np.array([
        -1.0530884977290216 * t * (t - 1.3299890189751412)
        * (t2 - 1.4364028541716351 * t + 0.7139816917074209),
        0.1017 * t2 * (t2 - 2.1966568338249754 * t + 1.2949852507374631),
        2.490627285651252793 * t2 * (t2 - 2.38535645472061657 * t + 1.57803468208092486),
        -16.54810288924490272 * (t - 1.21712927295533244) * (t - 0.61620406037800089) * t2,
        47.37952196281928122 * (t - 1.203071208372362603) * (t - 0.658047292653547382) * t2,
        -34.87065786149660974 * (t - 1.2) * (t - 0.666666666666666667) * t2,
        2.5 * (t - 1.0) * (t - 0.6) * t2,
    ])


def dopri5_dense_weights(theta: float) -> np.ndarray:
    """Dense-output weights w_i(theta) such that y(t0 + theta h) = y0 + h sum w_i k_i.

    The interpolant is the quartic p with p(0)=y0, p(1)=y1, p'(0)=h k1, p'(1)=h k7
    and p(1/2)=y_mid (Shampine's midpoint).  Writing p(theta) = y0 + sum_m c_m theta^m
    (m = 1..4), c1 = h k1 and c2..c4 solve a 3x3 linear system in
    d = y1 - y0, dm = y_mid - y0, f0 = h k1, f1 = h k7.  Everything is linear in the
    stages, so the weights on k_i follow by linearity.
    """
    # Solve the 4x4 system for c2..c4 given c1 = f0 (basis: d, dm, f0, f1).
    # Conditions: sum_m c_m = d ; sum_m m c_m = f1 ; sum_m c_m / 2^m = dm.
    M = np.array([[1.0, 1.0, 1.0],          # c2 + c3 + c4 = d - f0
                  [2.0, 3.0, 4.0],          # 2c2 + 3c3 + 4c4 = f1 - f0
                  [1 / 4, 1 / 8, 1 / 16]])  # c2/4 + c3/8 + c4/16 = dm - f0/2
    Minv = np.linalg.inv(M)
    # right-hand sides in the basis (d, dm, f0, f1)
    rhs = np.array([[1.0, 0.0, -1.0, 0.0],
                    [0.0, 0.0, -1.0, 1.0],
                    [0.0, 1.0, -0.5, 0.0]])
    C = Minv @ rhs  # rows: c2, c3, c4 in basis (d, dm, f0, f1)
    powers = np.array([theta ** 2, theta ** 3, theta ** 4])
    coef = powers @ C  # coefficients on (d, dm, f0, f1)
    coef[2] += theta  # c1 theta with c1 = f0
    # d = h sum b_i k_i, dm = h sum c_mid_i k_i, f0 = h k1, f1 = h k7
    w = coef[0] * DOPRI5.b + coef[1] * DOPRI5_C_MID
    w = w.copy()
    w[0] += coef[2]
    w[6] += coef[3]
    return w


def dense_weights(tab: Tableau, theta: float) -> np.ndarray:
    return tsit5_dense_weights(theta) if tab.name == 'Tsit5' else dopri5_dense_weights(theta)


# --------------------------------------------------------------------------------------
# Norm, initial step, controller
# --------------------------------------------------------------------------------------


def rms_norm(x: np.ndarray) -> float:
    """Root mean square over every (complex) entry: sqrt(mean |x|^2)."""
    x = np.asarray(x)
    if x.size == 0:
        return 0.0
    return float(np.sqrt(np.mean(np.abs(x.astype(np.complex128)) ** 2)))


def select_initial_step(f: Callable, t0: float, y0: np.ndarray, rtol: float,
                        atol: float, exponent: float = 0.25) -> float:
    """Hairer-Norsett-Wanner starting step (Solving ODEs I, Sec. II.4), RMS norm,
    last stage h1 = (0.01 / max(d1, d2))**exponent."""
    f0 = f(t0, y0)
    scale = atol + np.abs(y0) * rtol
    d0 = rms_norm(y0 / scale)
    d1 = rms_norm(f0 / scale)
    if d0 < 1e-5 or d1 < 1e-5:
        h0 = 1e-6
    else:
        h0 = 0.01 * d0 / d1
    y1 = y0 + h0 * f0
    f1 = f(t0 + h0, y1)
    d2 = rms_norm((f1 - f0) / scale) / h0
    max_d = max(d1, d2)
    if max_d <= 1e-15:
        h1 = max(1e-6, h0 * 1e-3)
    else:
        h1 = (0.01 / max_d) ** exponent
    return min(100 * h0, h1)


# --------------------------------------------------------------------------------------
# Solve loop
# --------------------------------------------------------------------------------------

STATUS_OK = 0
STATUS_MAX_STEPS = 1
STATUS_NONFINITE = 2


@dataclass
class SolveOutput:
    ts: np.ndarray
    ysave: list = field(default_factory=list)  # interpolated states at tsave
    ylast: np.ndarray | None = None
    nsteps: int = 0
    naccepted: int = 0
    nrejected: int = 0
    status: int = STATUS_OK
    accepted_times: list = field(default_factory=list)
    errors: list = field(default_factory=list)  # (t, h, scaled error) of every attempt


def solve(f: Callable, y0: np.ndarray, tsave: np.ndarray, *, method: str = 'Tsit5',
          rtol: float = 1e-6, atol: float = 1e-6, safety: float = 0.9,
          factormin: float = 0.2, factormax: float = 5.0, max_steps: int = 100_000,
          t0: float | None = None, time_dtype=np.float64,
          save_fn: Callable | None = None, dt0: float | None = None,
          jump_ts=None) -> SolveOutput:
    """Adaptive explicit RK (Tsit5 or Dopri5) from t0 to tsave[-1].

    ``f(t, y)`` is the vector field; ``y`` keeps its dtype (complex64 to mimic the
    reference's default precision, complex128 for the FP64 oracle).  Time arithmetic is
    done in ``time_dtype`` (float32 mimics JAX's default, float64 is the GPU design).
    ``save_fn(y)`` is applied to every interpolated save.

    ``jump_ts``: discontinuity times of the vector field, handled as the reference's
    ``PIDController(jump_ts=...)`` does (``dynamiqs/integrators/core/
    diffrax_integrator.py:59-72``): a trial step that would cross the next discontinuity J
    is clipped to end just before it (the largest time below J), the step after it starts
    at J itself with its first stage re-evaluated (no first-same-as-last across the jump),
    and the controller scales the step it had proposed -- not the clipped one -- to
    propose the next.
    """
    tab = TSIT5 if method == 'Tsit5' else DOPRI5
    td = np.dtype(time_dtype).type
    tsave = np.asarray(tsave, dtype=time_dtype)
    t_start = td(tsave[0] if t0 is None else t0)
    t_end = td(tsave[-1])
    clip_tol = td(1e-10) if np.dtype(time_dtype) == np.float64 else td(1e-6)
    ydt = y0.dtype
    out = SolveOutput(ts=tsave)
    save_fn = save_fn or (lambda y: y)

    def fe(t, y):
        return np.asarray(f(t, y), dtype=ydt)

    jumps = np.unique(np.asarray([] if jump_ts is None else jump_ts, dtype=time_dtype))

    def clip_jump(ta, tb):
        """(tb clipped before the first discontinuity after ta, whether it was)."""
        k = int(np.searchsorted(jumps, ta, side='right'))
        if k < jumps.size and tb >= jumps[k]:
            return np.nextafter(jumps[k], td(-np.inf)), True
        return tb, False

    y = y0.copy()
    t = t_start
    if dt0 is None:
        dt = td(select_initial_step(fe, float(t), y, rtol, atol, tab.start_exponent))
    else:
        dt = td(dt0)
    dt_prop = dt  # the controller's last proposal (before any clipping)
    tnext, made_jump = clip_jump(t, td(t + dt))
    tnext = min(tnext, t_end)
    if tnext > t_end - clip_tol:
        tnext = t_end
    k1 = fe(t, y)
    save_idx = 0
    # save points before or at t_start that are not crossed by any step
    while save_idx < len(tsave) and tsave[save_idx] <= t and t >= t_end:
        out.ysave.append(save_fn(y.copy()))
        save_idx += 1

    n_iter = 0
    while t < t_end:
        if n_iter >= max_steps:
            out.status = STATUS_MAX_STEPS
            break
        n_iter += 1
        h = td(tnext - t)
        hf = float(h)
        ks = [k1]
        for i in range(1, 6):
            yi = y.copy()
            for j in range(i):
                if tab.a[i, j] != 0.0:
                    yi = yi + (hf * tab.a[i, j]) * ks[j]
            ks.append(fe(float(t + td(tab.c[i] * hf)), yi.astype(ydt)))
        # y1 is the FSAL stage input (row 6 of a equals b)
        y1 = y.copy()
        for j in range(6):
            if tab.b[j] != 0.0:
                y1 = y1 + (hf * tab.b[j]) * ks[j]
        y1 = y1.astype(ydt)
        ks.append(fe(float(tnext), y1))
        yerr = np.zeros_like(y)
        for j in range(7):
            yerr = yerr + (hf * tab.btilde[j]) * ks[j]
        if not np.all(np.isfinite(y1)):
            y1_for_scale = y
        else:
            y1_for_scale = y1
        scale = atol + rtol * np.maximum(np.abs(y), np.abs(y1_for_scale))
        err = rms_norm(yerr / scale)
        if not np.isfinite(err):
            # a non-finite error estimate ends the solve (reported, never retried)
            out.nrejected += 1
            out.status = STATUS_NONFINITE
            break
        keep = err < 1.0
        out.errors.append((float(t), float(h), float(err)))
        # integral controller
        inv = np.inf if err == 0.0 else 1.0 / err
        fmin = 1.0 if keep else factormin
        factor = safety * (inv ** (1.0 / tab.error_order)) if np.isfinite(inv) else np.inf
        factor = float(np.clip(factor, fmin, factormax))
        dt_new = td((dt_prop if made_jump else h) * td(factor))
        if keep:
            out.naccepted += 1
            out.accepted_times.append(float(tnext))
            # dense output for every save time in (t, tnext]
            while save_idx < len(tsave) and tsave[save_idx] <= tnext:
                ts_ = tsave[save_idx]
                theta = float((ts_ - t) / h) if h > 0 else 1.0
                w = dense_weights(tab, theta)
                ys = y.copy()
                for j in range(7):
                    if w[j] != 0.0:
                        ys = ys + (hf * w[j]) * ks[j]
                out.ysave.append(save_fn(ys.astype(ydt)))
                save_idx += 1
            y = y1
            if made_jump:  # step ended just before a discontinuity: restart at it
                t = np.nextafter(tnext, td(np.inf))
                k1 = fe(float(t), y)
            else:
                t = tnext
                k1 = ks[6]
            if not np.all(np.isfinite(y)):
                out.status = STATUS_NONFINITE
                break
        else:
            out.nrejected += 1
        dt_prop = dt_new
        tn, made_jump = clip_jump(t, td(t + dt_new))
        if tn > t_end - clip_tol:
            # close to the end: an accepted step lands on t1, a rejected one retries
            # with half of what is left
            tn = t_end if keep else td(t + td(0.5) * td(t_end - t))
        tnext = min(tn, t_end)
    out.nsteps = n_iter
    out.ylast = y
    return out
