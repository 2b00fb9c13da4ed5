"""dynamiqs_b200 -- dynamiqs' ``mesolve`` hot path (Lindblad right-hand side inside the
Tsit5 / Dopri5 adaptive Runge-Kutta loop) as hand-written sm_100a CUDA kernels behind a
C ABI (``include/dqb200.h``), with the reference's Python API on top.
"""

from . import gradient, method, operators
from .mesolve import MESolveB200Integrator, mesolve
from .method import Dopri5, Tsit5
from .options import Options
from .qarrays import SparseDIA, dense, dia
from .result import AdaptiveStepInfos, MESolveResult
from .sesolve import SESolveResult, sesolve
from .time_qarray import Wave, modulated, pwc

__all__ = ['mesolve', 'sesolve', 'MESolveB200Integrator', 'Options', 'Tsit5', 'Dopri5',
           'MESolveResult', 'SESolveResult', 'AdaptiveStepInfos', 'SparseDIA', 'dense', 'dia',
           'method', 'gradient', 'operators', 'pwc', 'modulated', 'Wave']
