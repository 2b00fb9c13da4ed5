"""Result objects, mirroring ``dynamiqs/result.py:78-194`` and ``AdaptiveStepInfos``
(``dynamiqs/integrators/core/diffrax_integrator.py:35-50``).

Arrays are torch tensors on the device that ran the solve (``.cpu().numpy()`` for
numpy), with the reference's shapes: ``states`` ``(..., nsave, n, n)``, ``expects``
``(..., nE, ntsave)``, ``infos.nsteps`` ``(...)``.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

__all__ = ['AdaptiveStepInfos', 'MESolveResult']


@dataclass
class AdaptiveStepInfos:
    nsteps: Any
    naccepted: Any
    nrejected: Any

    def __str__(self) -> str:
        if self.nsteps.ndim >= 1:
            return (f'avg. {self.nsteps.float().mean():.1f} steps '
                    f'({self.naccepted.float().mean():.1f} accepted, '
                    f'{self.nrejected.float().mean():.1f} rejected) | infos shape '
                    f'{tuple(self.nsteps.shape)}')
        return (f'{int(self.nsteps)} steps ({int(self.naccepted)} accepted, '
                f'{int(self.nrejected)} rejected)')


def _array_str(x) -> str | None:
    if x is None:
        return None
    nbytes = x.numel() * x.element_size()
    return f'Array {str(x.dtype).replace("torch.", "")} {tuple(x.shape)} | {nbytes / 1024:.1f} Kb'


@dataclass
class MESolveResult:
    tsave: Any
    method: Any
    gradient: Any
    options: Any
    states: Any
    expects: Any
    infos: AdaptiveStepInfos
    extra: Any = None
    # FP64 checks of the saved states (an addition of this library): 'trace' tr(rho) at
    # every save point (..., ntsave) and 'hermiticity' ||rho - rho^+||_F / ||rho||_F of
    # every saved state (..., nsave)
    checks: Any = None

    @property
    def final_state(self):
        return self.states[..., -1, :, :]

    def block_until_ready(self) -> MESolveResult:
        import torch

        if self.states.is_cuda:
            torch.cuda.synchronize(self.states.device)
        return self

    def __str__(self) -> str:
        parts = {
            'Method': type(self.method).__name__,
            'Gradient': type(self.gradient).__name__ if self.gradient is not None else None,
            'Infos': self.infos,
            'States': _array_str(self.states),
            'Expects': _array_str(self.expects),
        }
        parts = {k: v for k, v in parts.items() if v is not None}
        pad = max(len(k) for k in parts) + 1
        body = '\n'.join(f'{k:<{pad}}: {v}' for k, v in parts.items())
        return f'==== {self.__class__.__name__} ====\n' + body
