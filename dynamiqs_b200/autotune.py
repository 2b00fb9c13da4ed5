"""Launch-shape autotuner for the large-problem paths.

Some launch choices have no single best value: the fastest depends on the Hilbert
dimension, the number of jump operators, the sparsity pattern and how many instances run
together.  The first solve with a new combination times every candidate on the problem at
hand -- one right-hand-side evaluation per candidate through the library's own
``dqb_lindblad_rhs_*`` entry points, CUDA events on the current stream, median of a few
runs -- and caches the fastest under a key of (GPU name, path, n, n_jumps, sparsity
signature, batch bucket, form).  Later solves with the same key reuse the choice.

Choices tuned:

* sparse DIA (``dqb_mesolve_dia``): the stencil kernel and its rows -- the generic kernel,
  the tiled one (coefficient tables) with 4, 8 or 16 rows per thread, the staged one
  (rows of X in shared memory) with 8 or 16 rows per CTA, the wide one (4 or 2 columns
  per thread, column factors in registers) with 8 or 16 rows per CTA, two rows in flight
  or registers capped for more resident CTAs, or the bulk-staged one
  (``dqb_ode_options.tile``); timed on the instances that run together and in the form
  the solve's stencils write (the stage slots' upper tiles in the hermitian stage form).
* dense GEMM path (n > 64) with ``Options(precision='auto')``: FP32 CUDA-core products or
  3xTF32 tensor-core products, the two arithmetic modes that meet the 1e-5 relative error
  bar; the tensor-core mode needs the hermitian form and an even n, else FP32 is used.

The cache lives in memory and in a JSON file, ``$DQB_AUTOTUNE_CACHE`` or
``~/.cache/dynamiqs_b200/autotune.json`` (not written when the location is read-only).
``DQB_AUTOTUNE=0`` turns tuning off: every choice is then its default (generic DIA
stencil, FP32 products).
"""

from __future__ import annotations

import json
import os
import threading

__all__ = ['enabled', 'cache_file', 'lookup', 'choose', 'clear_memory_cache']

_LOCK = threading.Lock()
_MEM: dict[str, dict] = {}
_LOADED = False


def enabled() -> bool:
    return os.environ.get('DQB_AUTOTUNE', '1') != '0'


def cache_file() -> str:
    return os.environ.get('DQB_AUTOTUNE_CACHE') or os.path.join(
        os.path.expanduser('~'), '.cache', 'dynamiqs_b200', 'autotune.json')


def key_string(parts: tuple) -> str:
    return '|'.join(str(p) for p in parts)


def batch_bucket(batch: int) -> int:
    """Largest power of two <= batch (capped at 4096): instances that run together."""
    b = 1
    while b * 2 <= min(max(batch, 1), 4096):
        b *= 2
    return b


def _load() -> None:
    global _LOADED
    if _LOADED:
        return
    _LOADED = True
    try:
        with open(cache_file()) as f:
            data = json.load(f)
        if isinstance(data, dict):
            for k, v in data.items():
                if isinstance(v, dict) and 'choice' in v:
                    _MEM.setdefault(k, v)
    except (OSError, ValueError):
        pass


def _save() -> None:
    path = cache_file()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = f'{path}.{os.getpid()}.tmp'
        with open(tmp, 'w') as f:
            json.dump(_MEM, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def lookup(key: str):
    with _LOCK:
        _load()
        ent = _MEM.get(key)
        return None if ent is None else ent['choice']


def clear_memory_cache() -> None:
    global _LOADED
    with _LOCK:
        _MEM.clear()
        _LOADED = True  # do not reload the file: callers want fresh measurements


def _time_ms(run, stream, reps: int) -> float:
    import torch

    run()  # warm-up (module load, first-touch)
    times = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        run()
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    times.sort()
    return times[len(times) // 2]


def choose(key_parts: tuple, candidates: list, make_run, default, reps: int = 3):
    """Return the cached choice for ``key_parts``, or time ``make_run(candidate)()`` for
    every candidate (CUDA events on the current stream), cache and return the fastest.
    With tuning disabled, or a single candidate, return ``default`` untimed."""
    import torch

    if not enabled() or len(candidates) <= 1:
        return default
    key = key_string(key_parts)
    hit = lookup(key)
    if hit is not None and hit in candidates:
        return hit
    stream = torch.cuda.current_stream()
    times = {}
    for c in candidates:
        times[c] = _time_ms(make_run(c), stream, reps)
    best = min(candidates, key=lambda c: times[c])
    with _LOCK:
        _MEM[key] = {'choice': best, 'times_ms': {str(c): t for c, t in times.items()}}
        _save()
    return best
