"""Integration methods accepted by ``dynamiqs_b200.mesolve``.

Same names, fields and defaults as the reference's adaptive ODE methods
(``dynamiqs/method.py:121-127`` ``_DEAdaptiveStep``; ``Dopri5`` ``:356-394``;
``Tsit5`` ``:438-476``): ``rtol=1e-6, atol=1e-6, safety_factor=0.9, min_factor=0.2,
max_factor=5.0, max_steps=100_000``.  The reference's other methods (Euler, Dopri8,
Kvaerno, Rouchon, Expm, Monte-Carlo, LowRank) are not part of this hot path;
``mesolve`` rejects them with the reference's ``TypeError`` message.
"""

from __future__ import annotations

from dataclasses import dataclass

__all__ = ['Method', 'Tsit5', 'Dopri5']


class Method:
    pass


@dataclass(frozen=True)
class _DEAdaptiveStep(Method):
    rtol: float = 1e-6
    atol: float = 1e-6
    safety_factor: float = 0.9
    min_factor: float = 0.2
    max_factor: float = 5.0
    max_steps: int = 100_000

    def assert_supports_gradient(self, gradient) -> None:
        """``Method.assert_supports_gradient`` (``dynamiqs/method.py:44-60``): Tsit5 and
        Dopri5 take ``Direct``, ``BackwardCheckpointed`` and ``Forward``."""
        from .gradient import BackwardCheckpointed, Direct, Forward

        supported = (Direct, BackwardCheckpointed, Forward)
        if gradient is not None and not isinstance(gradient, supported):
            support_str = ', '.join(f'`{x.__name__}`' for x in supported)
            raise ValueError(f'Method `{type(self).__name__}` does not support gradient '
                             f'`{type(gradient).__name__}` (supported gradient types: '
                             f'{support_str}).')


@dataclass(frozen=True)
class Tsit5(_DEAdaptiveStep):
    """Tsitouras method of order 5 (adaptive step size ODE method)."""


@dataclass(frozen=True)
class Dopri5(_DEAdaptiveStep):
    """Dormand-Prince method of order 5 (adaptive step size ODE method)."""
