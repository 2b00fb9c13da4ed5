"""``Options`` and the per-solver option check, as in ``dynamiqs/options.py:17-123``."""

from __future__ import annotations

from dataclasses import dataclass, fields
from typing import Any, Callable

__all__ = ['Options', 'check_options']


@dataclass(frozen=True)
class Options:
    save_states: bool = True
    save_propagators: bool = True
    cartesian_batching: bool = True
    progress_meter: Any = None
    t0: float | None = None
    save_extra: Callable | None = None
    nmaxclick: int = 10_000
    vectorized: bool = False
    assume_hermitian: bool = True
    # Arithmetic of the complex products (an addition of this library): 'fp32' (CUDA
    # cores, default); on the dense GEMM path (n > 64) 'tf32x3' or 'bf16x3' (tcgen05
    # tensor cores on hi + lo operand splits, FP32 accumulation) or 'tf32' (one TF32 pass,
    # ~1e-3: error studies only); on the n <= 64 kernel 'f16x3' (tcgen05 on FP16 hi + lo
    # splits of power-of-two-scaled operands, for 32 < n <= 64, at most two jumps; other
    # problems run FP32), ~1.4x faster on the batched-Kerr workload but with ~38 bits of
    # dynamic range: entries below ~2^-38 of a matrix's largest are flushed, so the error
    # control no longer sees a density matrix's far tail and takes fewer, larger steps
    # than the reference (states stay as accurate against an FP64 solution).  'auto' lets
    # the autotuner pick the faster of 'fp32' and 'tf32x3' on the GEMM path and means
    # 'fp32' elsewhere.  The sparse-DIA kernels always run FP32.
    precision: str = 'fp32'
    # How the sparse-DIA and dense GEMM (n > 64) paths form an RK step (an addition of
    # this library): 'stages' (stage by stage, as diffrax does), 'krylov' (every stage, y1,
    # the error estimate and the dense output as polynomials in hL applied to y, from the
    # basis (hL)^q y, q <= 7: the same method in exact arithmetic, 22 instead of 54 passes
    # over the state per step, and a rejected step reuses its basis; 1.8x faster on the
    # coupled-Kerr DIA workload, 1.2x on transmon x cavity, but in FP32 the expanded
    # polynomial rounds up to ~5x worse than the stages on stiff problems, still inside
    # the solve's tolerance), or 'auto' (= 'stages').  The n <= 64 kernel, sesolve and
    # the vectorized form run 'stages'.
    stepper: str = 'auto'

    def initialise(self) -> Options:
        return self


_SUPPORTED = {
    'sesolve': ('save_states', 'cartesian_batching', 'progress_meter', 't0', 'save_extra'),
    'mesolve': ('save_states', 'cartesian_batching', 'progress_meter', 't0', 'save_extra',
                'vectorized', 'assume_hermitian', 'precision', 'stepper'),
}


def check_options(options: Options, solver_name: str) -> None:
    """Raise if an option that ``solver_name`` ignores differs from its default
    (``dynamiqs/options.py:80-123``)."""
    valid = _SUPPORTED[solver_name]
    default = Options()
    for f in fields(options):
        value = getattr(options, f.name)
        if f.name not in valid and value != getattr(default, f.name):
            valid_str = ', '.join(f'`{x}`' for x in valid)
            raise ValueError(
                f'Option `{f.name}` was set to `{value}` but is not used by '
                f'the solver `dq.{solver_name}()` (valid options: {valid_str}).')
