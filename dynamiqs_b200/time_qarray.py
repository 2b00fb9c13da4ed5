"""Time-dependent operators for ``mesolve``.

Mirrors the reference's ``dq.pwc`` / ``PWCTimeQArray`` and ``dq.modulated`` /
``ModulatedTimeQArray`` (``dynamiqs/time_qarray.py:53-170,572-754``):
``pwc(times, values, qarray)`` is ``O(t) = c_k O_0`` for ``t`` in ``[t_k, t_{k+1})`` and
``0`` outside ``[t_0, t_N)``; ``modulated(f, qarray)`` is ``O(t) = f(t) O_0``; a constant
operator plus such terms (``H0 + pwc(...) + modulated(...)``) is a summed time-dependent
operator whose discontinuity times (the PWC times and the ``discontinuity_ts`` of modulated
terms) reach the step-size controller as ``jump_ts`` (``dynamiqs/integrators/core/
diffrax_integrator.py:59-72``).

On the GPU the prefactors are evaluated by the kernels at every stage time, so ``f`` must
be one they can evaluate: a :class:`Wave` (amplitude, angular frequency, phase, optional
Gaussian envelope and support) -- a Python callable cannot run inside a kernel.  Problems
with n <= 64 and at most four time-dependent terms run in one persistent launch with the
reference's discontinuity handling; larger PWC problems are split at the discontinuities
(one constant-operator solve per piece, each started with a fresh starting step).
"""

from __future__ import annotations

import numpy as np

from .qarrays import SparseDIA

__all__ = ['PWCTimeQArray', 'ModulatedTimeQArray', 'SummedTimeQArray', 'Wave', 'pwc',
           'modulated']


def _dense_op(x) -> np.ndarray:
    if isinstance(x, SparseDIA):
        return np.asarray(x.to_dense(), dtype=np.complex64)
    if hasattr(x, 'detach'):
        x = x.detach().cpu().numpy()
    return np.asarray(x, dtype=np.complex64)


class PWCTimeQArray:
    """``O(t) = values[k] * qarray`` for ``times[k] <= t < times[k+1]``, ``0`` elsewhere."""

    __array_ufunc__ = None  # ``ndarray + PWCTimeQArray`` defers to __radd__

    def __init__(self, times, values, qarray):
        times = np.asarray(times, dtype=np.float64)
        values = np.asarray(values)
        if times.ndim != 1 or times.size < 2:
            raise ValueError('Argument `times` must be a 1-D array of at least 2 time points.')
        if np.any(np.diff(times) < 0):
            raise ValueError('Argument `times` must be sorted in ascending order.')
        if values.shape[-1:] != (times.size - 1,):
            raise ValueError(f'Argument `values` must have shape (..., {times.size - 1}), got '
                             f'{values.shape}.')
        self.times = times
        self.values = values.astype(np.complex128)
        self.source = qarray  # as given (a SparseDIA stays sparse in the piecewise path)
        self.qarray = _dense_op(qarray)
        if self.qarray.ndim != 2 or self.qarray.shape[0] != self.qarray.shape[1]:
            raise ValueError('Argument `qarray` must be a square (n, n) operator.')

    @property
    def shape(self) -> tuple[int, ...]:
        return (*self.values.shape[:-1], *self.qarray.shape)

    @property
    def batch_shape(self) -> tuple[int, ...]:
        return self.values.shape[:-1]

    def item(self, idx: tuple) -> PWCTimeQArray:
        """The unbatched term at index ``idx`` of a batch shape that this term's value batch
        broadcasts to (dimensions aligned on the right, size-1 dimensions broadcast)."""
        bs = self.batch_shape
        if not bs:
            return self
        tail = idx[len(idx) - len(bs):]
        sub = self.values[tuple(0 if size == 1 else i for i, size in zip(tail, bs))]
        return PWCTimeQArray(self.times, sub, self.source)

    @property
    def discontinuity_ts(self) -> np.ndarray:
        return self.times

    def prefactor(self, t: float) -> complex:
        k = int(np.searchsorted(self.times, t, side='right')) - 1
        return complex(self.values[k]) if 0 <= k < self.values.size else 0.0

    def __call__(self, t: float) -> np.ndarray:
        return (self.prefactor(t) * self.qarray).astype(np.complex64)

    def __add__(self, other) -> SummedTimeQArray:
        return SummedTimeQArray([self, other])

    __radd__ = __add__


class Wave:
    """A prefactor the kernels evaluate: ``f(t) = amplitude * cos(omega t + phase) * env(t)``
    for ``t_start <= t < t_end`` and ``0`` elsewhere, with ``env(t) = exp(-(t - t_center)^2
    / (2 sigma^2))`` when ``sigma > 0`` and ``1`` otherwise.  ``amplitude`` may be complex;
    ``omega = 0`` gives a constant, ``phase = -pi/2`` a sine."""

    def __init__(self, omega: float = 0.0, phase: float = 0.0, amplitude: complex = 1.0, *,
                 t_center: float = 0.0, sigma: float = 0.0, t_start: float = -np.inf,
                 t_end: float = np.inf):
        self.omega = float(omega)
        self.phase = float(phase)
        self.amplitude = complex(amplitude)
        self.t_center = float(t_center)
        self.sigma = float(sigma)
        self.t_start = float(t_start)
        self.t_end = float(t_end)
        if self.sigma < 0:
            raise ValueError('Argument `sigma` must be >= 0.')

    def __call__(self, t: float) -> complex:
        if not (self.t_start <= t < self.t_end):
            return 0.0
        f = np.cos(self.omega * t + self.phase)
        if self.sigma > 0:
            f *= np.exp(-0.5 * ((t - self.t_center) / self.sigma) ** 2)
        return self.amplitude * f

    @property
    def discontinuity_ts(self) -> np.ndarray:
        return np.asarray([t for t in (self.t_start, self.t_end) if np.isfinite(t)])


class ModulatedTimeQArray:
    """``O(t) = f(t) * qarray`` with ``f`` a :class:`Wave` (``ModulatedTimeQArray``,
    ``dynamiqs/time_qarray.py:669-754``)."""

    __array_ufunc__ = None

    def __init__(self, f, qarray, discontinuity_ts=None):
        if not isinstance(f, Wave):
            raise NotImplementedError(
                'dynamiqs_b200.modulated needs a prefactor the GPU kernels can evaluate: a '
                '`Wave` (amplitude, omega, phase, optional Gaussian envelope and support); an '
                'arbitrary Python callable cannot run inside a kernel.')
        self.f = f
        self.source = qarray
        self.qarray = _dense_op(qarray)
        if self.qarray.ndim != 2 or self.qarray.shape[0] != self.qarray.shape[1]:
            raise ValueError('Argument `qarray` must be a square (n, n) operator.')
        extra = np.asarray([] if discontinuity_ts is None else discontinuity_ts, dtype=np.float64)
        self._disc = np.unique(np.concatenate([extra, f.discontinuity_ts]))

    @property
    def shape(self) -> tuple[int, ...]:
        return self.qarray.shape

    @property
    def batch_shape(self) -> tuple[int, ...]:
        return ()

    def item(self, idx: tuple) -> ModulatedTimeQArray:
        return self

    @property
    def discontinuity_ts(self) -> np.ndarray:
        return self._disc

    def prefactor(self, t: float) -> complex:
        return complex(self.f(t))

    def __call__(self, t: float) -> np.ndarray:
        return (self.prefactor(t) * self.qarray).astype(np.complex64)

    def __add__(self, other) -> SummedTimeQArray:
        return SummedTimeQArray([self, other])

    __radd__ = __add__


_TD_TYPES = (PWCTimeQArray, ModulatedTimeQArray)


class SummedTimeQArray:
    """A sum of constant operators and :class:`PWCTimeQArray` / :class:`ModulatedTimeQArray`
    terms."""

    __array_ufunc__ = None

    def __init__(self, terms):
        flat = []
        for t in terms:
            flat.extend(t.terms if isinstance(t, SummedTimeQArray) else [t])
        self.pwc_terms = [t for t in flat if isinstance(t, _TD_TYPES)]
        self._const_src = [t for t in flat if not isinstance(t, _TD_TYPES)]
        const = [_dense_op(t) for t in self._const_src]
        n = (self.pwc_terms[0].shape if self.pwc_terms else const[0].shape)[-1]
        for c in const:
            if c.ndim != 2:
                raise NotImplementedError('A batched constant part of a time-dependent H is not '
                                          'supported on the B200 path.')
        self.constant = sum(const) if const else np.zeros((n, n), np.complex64)
        self.terms = flat
        for t in self.pwc_terms:
            if t.qarray.shape != self.constant.shape:
                raise ValueError('All terms of a time-dependent operator must have the same shape.')
        try:
            self.batch_shape
        except ValueError:
            raise ValueError('The batch shapes of the PWC values do not broadcast together.') from None

    @property
    def shape(self) -> tuple[int, ...]:
        return (*self.batch_shape, *self.constant.shape)

    @property
    def batch_shape(self) -> tuple[int, ...]:
        return np.broadcast_shapes(*[t.batch_shape for t in self.pwc_terms]) if self.pwc_terms else ()

    def item(self, idx: tuple) -> SummedTimeQArray:
        """The unbatched operator at index ``idx`` of :attr:`batch_shape`."""
        const = self._const_src if self.is_dia else [self.constant]
        return SummedTimeQArray(list(const) + [t.item(idx) for t in self.pwc_terms])

    @property
    def is_dia(self) -> bool:
        """Every term (constant or time-dependent) is a SparseDIA operator."""
        return (all(isinstance(c, SparseDIA) for c in self._const_src)
                and all(isinstance(t.source, SparseDIA) for t in self.pwc_terms))

    def piece(self, t: float):
        """The constant operator at time ``t``: a SparseDIA (diagonals summed over the
        terms) when every term is one, so that a piece's solve stays on the DIA path, else
        a dense array."""
        if not self.is_dia:
            return self(t)
        out = None
        for c in self._const_src:
            out = c if out is None else out + c
        for term in self.pwc_terms:
            x = term.source * np.complex64(term.prefactor(t))
            out = x if out is None else out + x
        return out.astype(np.complex64)

    @property
    def td_terms(self) -> list:
        return self.pwc_terms

    @property
    def only_pwc(self) -> bool:
        return all(isinstance(t, PWCTimeQArray) for t in self.pwc_terms)

    @property
    def discontinuity_ts(self) -> np.ndarray:
        ts = [t.discontinuity_ts for t in self.pwc_terms]
        return np.unique(np.concatenate(ts)) if ts else np.zeros(0)

    def __call__(self, t: float) -> np.ndarray:
        out = self.constant.astype(np.complex128)
        for term in self.pwc_terms:
            out = out + term.prefactor(t) * term.qarray
        return out.astype(np.complex64)

    def __add__(self, other) -> SummedTimeQArray:
        return SummedTimeQArray([self, other])

    __radd__ = __add__


def pwc(times, values, qarray) -> PWCTimeQArray:
    """Piecewise-constant operator ``O(t) = sum_k c_k 1_[t_k, t_{k+1})(t) O_0``
    (``dq.pwc``, ``dynamiqs/time_qarray.py:53-120``)."""
    return PWCTimeQArray(times, values, qarray)


def modulated(f, qarray, *, discontinuity_ts=None) -> ModulatedTimeQArray:
    """Modulated operator ``O(t) = f(t) O_0`` (``dq.modulated``,
    ``dynamiqs/time_qarray.py:123-170``); ``f`` must be a :class:`Wave`."""
    return ModulatedTimeQArray(f, qarray, discontinuity_ts)


def as_summed(H) -> SummedTimeQArray:
    return H if isinstance(H, SummedTimeQArray) else SummedTimeQArray([H])


def piecewise_plan(H: SummedTimeQArray, tsave: np.ndarray, t0: float):
    """The constant pieces of a solve from ``t0`` to ``tsave[-1]``: a list of
    ``(a, b, H_piece, ts_piece, keep)`` where ``ts_piece`` is the save grid handed to the
    constant-operator solve of ``[a, b]`` (it starts at ``a`` and ends at ``b``) and
    ``keep`` the indices of ``ts_piece`` that are points of ``tsave``, in order.  Every
    point of ``tsave`` is kept exactly once (a point on a discontinuity belongs to the piece
    that ends there; ``tsave[0] == t0`` to the first piece)."""
    t1 = float(tsave[-1])
    bps = [float(t) for t in H.discontinuity_ts if t0 < t < t1]
    edges = [t0] + sorted(set(bps)) + [t1]
    plan = []
    for i, (a, b) in enumerate(zip(edges[:-1], edges[1:])):
        inside = [float(t) for t in tsave if (a < t <= b) or (i == 0 and t == a)]
        ts = sorted(set([a, b] + inside))
        keep = [ts.index(t) for t in inside]
        plan.append((a, b, H.piece(0.5 * (a + b)), np.asarray(ts), keep))
    return plan
