"""Gradient options (``dynamiqs/gradient.py:10-110``): ``Direct``, ``BackwardCheckpointed``
and ``Forward``.

On the B200 path every one of them gives the same numbers: the exact reverse-mode
derivative of the discrete solve (the Runge-Kutta steps it took, step sizes held
constant as the reference's controller is not differentiated), computed by the adjoint
kernel (``dqb_mesolve_dense_adjoint``) from a tape of the accepted steps, and delivered
through ``torch.autograd``: pass ``H``, ``jump_ops`` or ``rho0`` as torch tensors with
``requires_grad=True`` and call ``backward()`` on a loss built from the result's
``states`` / ``expects``.  ``BackwardCheckpointed(ncheckpoints)`` keeps its argument for
the reference's signature: the tape holds every accepted step (n^2 complex64 each), which
is what the checkpointing of the reference trades memory against.
"""

from __future__ import annotations

from dataclasses import dataclass

__all__ = ['Gradient', 'Direct', 'BackwardCheckpointed', 'Forward']


class Gradient:
    pass


@dataclass(frozen=True)
class Direct(Gradient):
    """Differentiation through the solver's internals."""


@dataclass(frozen=True)
class BackwardCheckpointed(Gradient):
    """Reverse mode through the solver's steps (the reference's default for Tsit5)."""

    ncheckpoints: int | None = None


@dataclass(frozen=True)
class Forward(Gradient):
    """Forward mode in the reference; here the same derivatives, through the adjoint."""
