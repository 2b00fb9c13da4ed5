"""Continuous-batching mesolve server.

Requests (single problems, any of the sizes the kernels support) arrive at any time
through :meth:`MESolveServer.submit`.  A dispatcher thread groups the waiting requests by
size class -- Hilbert dimension padded to 16, 32 or 64 for the shared-memory kernel, or
the exact n for the GEMM path above 64 -- and launches a *wave* for a class as soon as a
stream and memory are free:

* n <= 64: one ``dqb_mesolve_ragged`` launch per wave (n padded to the class size).
* n > 64: one ``dqb_mesolve_dense_large_ragged`` launch per wave of requests of that n.

Every request in a wave keeps its own jump operators, exp_ops, tsave grid, start time and
outputs (and, below 64, its own n); each is solved exactly as it would be alone, with no
dependence on the other instances of the wave.

Waves run on a pool of CUDA streams, so requests that arrive while others are on the GPU
start right away on another stream and their work overlaps on the device.  Admission is
bounded by a byte budget for the device memory a wave holds (inputs, outputs and
scratch), 150 GB by default; a finished wave releases its budget.  Results stay on the
device (as ``dq.mesolve`` returns them).  The kernels write each request's step counts and
then, after a system-scope fence, its status word straight into page-locked host memory;
the dispatcher hands a request out as soon as its status word appears, without waiting for
the rest of its wave (a quick request does not wait for a slow one launched with it).

Tickets record submit, launch and completion times, from which :meth:`stats` reports
solves/s and p50 / p99 latency.

:meth:`Ticket.cancel` stops a request: a waiting one leaves the queue, a running one gets
its cancel word (page-locked host memory, one per request, named in its kernel
descriptor) set; the kernels read the word between RK steps and end the request with the
cancelled status, which the dispatcher hands out like any other end.  The other requests
of its wave are not affected (each instance is independent).

CUDA maps streams onto ``CUDA_DEVICE_MAX_CONNECTIONS`` hardware queues (8 by default);
streams that share a queue run one after the other.  Set it to at least the number of
server streams (32 at most) before CUDA is initialised in the process, or a wave can
wait behind an unrelated long wave on the same queue.
"""

from __future__ import annotations

import contextlib
import ctypes
import dataclasses
import threading
import time
from collections import deque
from concurrent.futures import CancelledError, ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .mesolve import (_as_op, _check_mesolve_args, _MAX_STEPS_MSG, _precision_code,
                      _stepper_code, assert_method_supported, check_times)
from .method import Tsit5
from .options import Options, check_options
from .qarrays import to_dense
from .result import AdaptiveStepInfos, MESolveResult

__all__ = ['MESolveServer', 'Ticket']


def _align(x: int) -> int:
    return (x + 255) & ~255


# Per request, page-locked: step counts (3 int32), status word, cancel word, padding.
_INFO = 32


class _Arena:
    """First-fit sub-allocator over one buffer allocated at start-up, so that serving never
    calls the CUDA allocators (device and page-locked allocations synchronise with work
    in flight on other streams)."""

    def __init__(self, nbytes: int):
        self.size = nbytes
        self.free = [(0, nbytes)]  # sorted (offset, size)
        self.lock = threading.Lock()

    def alloc(self, nbytes: int) -> int | None:
        nbytes = _align(max(nbytes, 1))
        with self.lock:
            for i, (o, sz) in enumerate(self.free):
                if sz >= nbytes:
                    if sz == nbytes:
                        self.free.pop(i)
                    else:
                        self.free[i] = (o + nbytes, sz - nbytes)
                    return o
        return None

    def release(self, off: int, nbytes: int) -> None:
        nbytes = _align(max(nbytes, 1))
        with self.lock:
            self.free.append((off, nbytes))
            self.free.sort()
            merged = []
            for o, sz in self.free:
                if merged and merged[-1][0] + merged[-1][1] == o:
                    merged[-1] = (merged[-1][0], merged[-1][1] + sz)
                else:
                    merged.append((o, sz))
            self.free = merged

    def used(self) -> int:
        with self.lock:
            return self.size - sum(sz for _, sz in self.free)


@dataclass
class Ticket:
    """Handle of one submitted request."""

    id: int
    n: int
    H: np.ndarray
    Ls: list
    rho0: np.ndarray
    tsave: np.ndarray
    Es: list | None
    method: object
    options: Options
    t_submit: float = 0.0
    t_launch: float = 0.0
    t_done: float = 0.0
    _event: threading.Event = field(default_factory=threading.Event)
    _result: MESolveResult | None = None
    _error: BaseException | None = None
    _out: tuple | None = None  # (arena, offset, nbytes) of the result buffers
    _server: object = None
    _cancel_word: int | None = None  # index of the cancel word in the pinned int32 view
    _cancel_requested: bool = False
    # the ticket's wave has ended (its kernels no longer write the result buffers), and a
    # release() that came before that, carried out when it ends
    _wave_done: bool = False
    _release_pending: bool = False
    _release_lock: threading.Lock = field(default_factory=threading.Lock)

    def done(self) -> bool:
        return self._event.is_set()

    def cancel(self) -> bool:
        """Stop the request.  A waiting request leaves the queue at once; a running one
        stops at its next check (between RK steps) and its ticket then ends.  Either way
        :meth:`result` raises ``concurrent.futures.CancelledError``.  Returns False when
        the request had already finished."""
        return self._server._cancel(self) if self._server is not None else False

    def result(self, timeout: float | None = None) -> MESolveResult:
        if not self._event.wait(timeout):
            raise TimeoutError(f'request {self.id} not finished after {timeout} s')
        if self._error is not None:
            raise self._error
        return self._result

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit

    def release(self) -> None:
        """Give the result's device memory back to the server (the result's tensors must
        not be used afterwards).  A ticket handed out before the rest of its wave finished
        is released when the wave ends: until then the wave's kernels may still write its
        buffers (the large-problem path writes every instance's outputs once more at the
        end of the wave)."""
        with self._release_lock:
            if not self._wave_done:
                self._release_pending = True
                return
            self._release_now()

    def _release_now(self) -> None:
        if self._out is not None:
            arena, off, nb = self._out
            self._out = None
            arena.release(off, nb)

    def _wave_ended(self) -> None:
        with self._release_lock:
            self._wave_done = True
            if self._release_pending:
                self._release_now()


class _Wave:
    def __init__(self, kind, tickets, stream, event, keep, nbytes, outputs):
        self.kind = kind
        self.tickets = tickets
        self.stream = stream
        self.event = event
        self.keep = keep  # device / pinned buffers alive until the wave retires
        self.nbytes = nbytes
        self.outputs = outputs  # per ticket: (states, expects) device views into the arena


class MESolveServer:
    # bounds of a request on the GEMM path (they size the per-stream graph slots)
    LARGE_MAX_JUMPS = 8
    LARGE_MAX_EXP = 8
    LARGE_MAX_TSAVE = 1024

    def __init__(self, budget_bytes: float = 150e9, max_wave: int = 4096, n_streams: int = 16,
                 poll_s: float = 50e-6, max_large_wave: int = 64, staging_bytes: float = 2e9,
                 history: int = 100_000):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError('MESolveServer needs a CUDA device; there is no CPU fallback.')
        import os
        import warnings

        if int(os.environ.get('CUDA_DEVICE_MAX_CONNECTIONS', '8')) < n_streams:
            warnings.warn(f'CUDA_DEVICE_MAX_CONNECTIONS < {n_streams}: server streams will share '
                          'hardware queues and waves may wait behind one another.', stacklevel=2)
        self._torch = torch
        self.lib = _lib.load()
        self.dev = torch.device('cuda', torch.cuda.current_device())
        free, _total = torch.cuda.mem_get_info(self.dev)
        self.budget = int(min(budget_bytes, 0.85 * free))
        # the memory budget is a device arena allocated once; waves and results live in it
        self._dev_buf = torch.empty(self.budget, dtype=torch.uint8, device=self.dev)
        self._dev = _Arena(self.budget)
        staging = int(staging_bytes) // 256 * 256
        self._host_buf = torch.empty(staging, dtype=torch.uint8, pin_memory=True)
        self._host_i32 = self._host_buf.numpy().view(np.int32)
        self._host = _Arena(staging)
        self.max_wave = max_wave
        self.poll_s = poll_s
        # separate stream pools, so that long GEMM-path waves never hold up small requests;
        # small waves also get the higher stream priority, so their blocks are scheduled
        # ahead of the wide GEMM grids that a large wave keeps launching
        n_small = max(1, n_streams // 2)
        hi = torch.cuda.Stream.priority_range()[1]
        self._free_streams = {
            'small': deque(torch.cuda.Stream(self.dev, priority=hi) for _ in range(n_small)),
            'large': deque(torch.cuda.Stream(self.dev) for _ in range(max(1, n_streams - n_small))),
        }
        self.max_large_wave = max_large_wave
        self._large_slots: dict = {}  # (stream id, n) -> (desc_off, count_off, ws_off, ws_bytes)
        self._pending: dict[tuple, deque] = {}
        self._inflight: list[_Wave] = []
        self._lock = threading.Lock()
        self._cancel_lock = threading.Lock()
        self._wake = threading.Condition(self._lock)
        self._closing = False
        self._paused = False
        self._next_id = 0
        # finished tickets and per-wave launch records, the latest `history` of each (a
        # long-running server keeps a bounded window for stats())
        self.finished: deque[Ticket] = deque(maxlen=history)
        self.waves_launched = 0
        self.launch_seconds: deque = deque(maxlen=history)  # (class, instances, host s in the launch)
        self.launch_profile: deque = deque(maxlen=history)  # (class, {step: host seconds}) per wave
        # waves are launched from worker threads: a driver call that waits (for instance a
        # graph instantiation while another conditional graph runs) holds up only its class
        self._launcher = ThreadPoolExecutor(max_workers=n_streams, thread_name_prefix='mesolve-launch')
        self._launching = 0
        self._thread = threading.Thread(target=self._loop, name='mesolve-dispatch', daemon=True)
        self._thread.start()

    # ---- client side ----------------------------------------------------------------
    def submit(self, H, jump_ops, rho0, tsave, *, exp_ops=None, method=Tsit5(),  # noqa: B008
               options: Options = Options()) -> Ticket:  # noqa: B008
        """Queue one problem (no batch dimensions); returns a :class:`Ticket`."""
        H = _as_op(H)
        Ls = [_as_op(L) for L in jump_ops]
        rho0 = _as_op(rho0)
        tsave = check_times(np.asarray(tsave, dtype=np.float64), 'tsave')
        Es = [_as_op(E) for E in exp_ops] if exp_ops else None
        _check_mesolve_args(H, Ls, rho0, Es)
        check_options(options, 'mesolve')
        assert_method_supported(method)
        if len(H.shape) != 2 or any(len(L.shape) != 2 for L in Ls) or len(rho0.shape) != 2:
            raise ValueError('MESolveServer.submit takes one problem without batch dimensions.')
        n = H.shape[-1]
        form = (_lib.FORM_STANDARD if (options.vectorized or not options.assume_hermitian)
                else _lib.FORM_HERMITIAN)
        if n > 64 and (_precision_code(options, form) != _lib.PREC_FP32 and n % 2):
            raise ValueError('Option `precision` other than "fp32" needs an even n.')
        t = Ticket(id=-1, n=n, H=to_dense(H).astype(np.complex64),
                   Ls=[to_dense(L).astype(np.complex64) for L in Ls],
                   rho0=np.asarray(rho0, np.complex64), tsave=tsave,
                   Es=[to_dense(E).astype(np.complex64) for E in Es] if Es else None,
                   method=method, options=options)
        key = self._class_of(t)
        t._server = self
        with self._lock:
            if self._closing:
                raise RuntimeError('server is closed')
            t.id = self._next_id
            self._next_id += 1
            t.t_submit = time.perf_counter()
            self._pending.setdefault(key, deque()).append(t)
            self._wake.notify()
        return t

    def pause(self) -> None:
        """Stop launching new waves (running ones continue and retire); the requests
        submitted meanwhile wait, so that :meth:`resume` launches them together, a class's
        queue as one wave (up to the wave size) per free stream."""
        with self._lock:
            self._paused = True

    def resume(self) -> None:
        with self._lock:
            self._paused = False
            self._wake.notify()

    @contextlib.contextmanager
    def paused(self):
        """``with server.paused(): submit(...)`` -- the requests submitted in the block
        are launched together when it ends."""
        self.pause()
        try:
            yield self
        finally:
            self.resume()

    def _cancel(self, t: Ticket) -> bool:
        with self._lock:
            if t._event.is_set():
                return False
            for q in self._pending.values():
                if t in q:  # still waiting: leave the queue
                    q.remove(t)
                    self._fail([t], CancelledError(f'request {t.id} cancelled'))
                    return True
        with self._cancel_lock:  # launched, or being launched: the kernel stops it
            t._cancel_requested = True
            if t._cancel_word is not None:
                self._host_i32[t._cancel_word] = 1
        return True

    def close(self, wait: bool = True) -> None:
        with self._lock:
            self._closing = True
            self._paused = False  # a paused server still finishes what it was given
            self._wake.notify()
        if wait:
            self._thread.join()

    def stats(self) -> dict:
        done = [t for t in self.finished if t._error is None]
        if not done:
            return {'solves': 0}
        lat = np.array([t.latency for t in done]) * 1e3
        t0 = min(t.t_submit for t in done)
        t1 = max(t.t_done for t in done)
        return {'solves': len(done), 'errors': len(self.finished) - len(done),
                'makespan_s': t1 - t0, 'solves_per_s': len(done) / (t1 - t0),
                'p50_ms': float(np.percentile(lat, 50)), 'p99_ms': float(np.percentile(lat, 99)),
                'mean_ms': float(lat.mean()), 'waves': self.waves_launched}

    # ---- dispatcher ---------------------------------------------------------------------
    def _class_of(self, t: Ticket) -> tuple:
        K = len(t.Ls)
        if t.n <= 64:
            np_ = 16 if t.n <= 16 else (32 if t.n <= 32 else 64)
            if self.lib.dqb_dense_small_max_n(K) >= np_:
                return ('small', np_)
        return ('large', t.n)

    def _loop(self) -> None:
        torch = self._torch
        torch.cuda.set_device(self.dev)
        while True:
            with self._lock:
                if (self._closing and not self._inflight and not self._launching
                        and not any(self._pending.values())):
                    self._launcher.shutdown(wait=False)
                    return
            progressed = self._retire()
            progressed |= self._admit()
            if not progressed:
                with self._lock:
                    if (not self._closing and not any(self._pending.values())
                            and not self._inflight and not self._launching):
                        self._wake.wait(timeout=0.05)
                time.sleep(self.poll_s)

    def _retire(self) -> bool:
        with self._lock:
            inflight = list(self._inflight)
        progressed = False
        for w in inflight:  # requests whose status word is written: hand them out now
            progressed |= self._retire_early(w)
        done = [w for w in inflight if w.event.query()]
        for w in done:
            self._finish(w)
            with self._lock:
                self._inflight.remove(w)
                self._free_streams[w.kind].append(w.stream)
        return bool(done) or progressed

    def _retire_early(self, w: _Wave) -> bool:
        """Finish the tickets of a running wave whose status word the kernel has written
        (it writes it last, after the request's outputs and a system-scope fence), without
        waiting for the rest of the wave."""
        if not w.pending:
            return False
        words = self._host_i32[w.status_words]
        ready = np.nonzero(words != -1)[0]
        if ready.size == 0:
            return False
        keep = np.ones(len(w.pending), bool)
        keep[ready] = False
        for i in ready:
            self._finish_ticket(w, w.pending[i])
        w.pending = [t for t, k in zip(w.pending, keep) if k]
        w.status_words = w.status_words[keep]
        return True

    def _admit(self) -> bool:
        launched = False
        with self._lock:
            if self._paused:
                return False
            keys = [k for k, q in self._pending.items() if q]
        for key in keys:
            while True:
                with self._lock:
                    q = self._pending[key]
                    pool = self._free_streams[key[0]]
                    if not q or not pool:
                        break
                    cap = self.max_wave if key[0] == 'small' else self.max_large_wave
                    take = [q.popleft() for _ in range(min(cap, len(q)))]
                    stream = pool.popleft()
                    self._launching += 1
                self._launcher.submit(self._launch_job, take, key, stream)
                launched = True
        return launched

    def _launch_job(self, take, key, stream) -> None:
        """Worker thread: launch a wave (shrinking it if the arena is short), then hand it to
        the dispatcher for retirement."""
        self._torch.cuda.set_device(self.dev)
        wave = None
        t0 = time.perf_counter()
        try:
            while take:
                try:
                    wave = self._launch_wave(take, key, stream)
                except BaseException as e:  # report to the tickets, keep serving
                    self._fail(take, e)
                    take = []
                    break
                if wave is not None:
                    break
                # not enough memory for all of them: retry with fewer, requeue the rest
                with self._lock:
                    idle = not self._inflight
                if len(take) == 1 and idle:
                    self._fail(take, MemoryError(
                        'request needs more device memory than the server budget has free'))
                    take = []
                    break
                keep = max(len(take) // 2, 0)
                with self._lock:
                    self._pending[key].extendleft(reversed(take[keep:]))
                take = take[:keep]
        finally:
            with self._lock:
                self._launching -= 1
                if wave is None:
                    self._free_streams[key[0]].append(stream)
                else:
                    self._inflight.append(wave)
                    self.waves_launched += 1
                    self.launch_seconds.append((key, len(wave.tickets), time.perf_counter() - t0))
                self._wake.notify()

    def _fail(self, tickets, err) -> None:
        now = time.perf_counter()
        for t in tickets:
            t._error = err
            t.t_done = now
            self.finished.append(t)
            t._event.set()

    # ---- waves --------------------------------------------------------------------------
    def _precision_of(self, t: Ticket, form: int, count: int) -> int:
        """GEMM-path arithmetic of a wave.  ``precision='auto'``: 3xTF32 tensor cores
        whenever the form and n allow them (hermitian form, even n), else FP32 CUDA cores.
        Measured on the serving workload, the tensor cores were also the faster choice for
        waves of one or two stiff requests, where their 128x128 tiles leave most SMs idle."""
        o = t.options
        if t.n <= 64:
            return _lib.PREC_FP32
        if o.precision == 'auto':
            ok = form == _lib.FORM_HERMITIAN and t.n % 2 == 0
            return _lib.PREC_TF32X3 if ok else _lib.PREC_FP32
        return _precision_code(o, form)

    def _ode_options(self, t: Ticket, count: int = 1) -> _lib.OdeOptions:
        m, o = t.method, t.options
        form = (_lib.FORM_STANDARD if (o.vectorized or not o.assume_hermitian)
                else _lib.FORM_HERMITIAN)
        return _lib.OdeOptions(
            method=_lib.METHOD_TSIT5 if isinstance(m, Tsit5) else _lib.METHOD_DOPRI5, form=form,
            rtol=float(m.rtol), atol=float(m.atol), safety=float(m.safety_factor),
            factormin=float(m.min_factor), factormax=float(m.max_factor),
            max_steps=int(m.max_steps), t0=0.0, save_states=1,
            check_hermitian=int(bool(o.assume_hermitian)),
            precision=self._precision_of(t, form, count), stepper=_stepper_code(o))

    def _launch_wave(self, tickets, key, stream) -> _Wave | None:
        """Pack the wave's inputs into pinned staging (one host-to-device copy), give every
        request its own output region in the device arena, and launch dqb_mesolve_ragged
        (n <= 64) or dqb_mesolve_dense_large_ragged (one n above 64).  Returns None when the
        arenas cannot hold the wave (nothing is launched then)."""
        torch = self._torch
        groups: dict = {}
        for t in tickets:  # different methods or tolerances go to different launches
            groups.setdefault((type(t.method), t.method.rtol, t.method.atol,
                               t.method.safety_factor, t.method.min_factor, t.method.max_factor,
                               t.method.max_steps, t.options.assume_hermitian,
                               t.options.vectorized, t.options.precision,
                               t.options.stepper), []).append(t)
        held = []  # (arena, offset, nbytes) released when the wave retires
        outs_held = {}  # per ticket output region
        plans = []

        def grab(arena, nb):
            off = arena.alloc(nb)
            if off is None:
                raise MemoryError
            held.append((arena, off, nb))
            return off

        try:
            for group in groups.values():
                layout, off = [], 0

                def put(nb):
                    nonlocal off
                    o = off
                    off = _align(off + nb)
                    return o

                for t in group:
                    layout.append({'H': put(t.H.nbytes),
                                   'L': put(max(sum(L.nbytes for L in t.Ls), 8)),
                                   'rho0': put(t.rho0.nbytes),
                                   'E': put(max(sum(E.nbytes for E in t.Es), 8) if t.Es else 8),
                                   'tsave': put(t.tsave.nbytes)})
                desc_off = put(ctypes.sizeof(_lib.RaggedInstance) * len(group))
                info_off = put(_INFO * len(group))
                in_bytes = off
                maxK = max(len(t.Ls) for t in group)
                count = len(group)
                maxE = maxT = 0
                h_in = grab(self._host, in_bytes)
                d_in = grab(self._dev, in_bytes)
                if key[0] == 'small':
                    ws_bytes = self.lib.dqb_mesolve_ragged_workspace_size(key[1], maxK, count)
                    d_ws = grab(self._dev, ws_bytes)
                else:
                    for t in group:
                        if (len(t.Ls) > self.LARGE_MAX_JUMPS or len(t.tsave) > self.LARGE_MAX_TSAVE
                                or (len(t.Es) if t.Es else 0) > self.LARGE_MAX_EXP):
                            raise ValueError('request outside the GEMM-path bounds of the server '
                                             f'(jumps <= {self.LARGE_MAX_JUMPS}, exp_ops <= '
                                             f'{self.LARGE_MAX_EXP}, tsave <= {self.LARGE_MAX_TSAVE})')
                    d_ws, ws_bytes = self._large_slot(stream, key[1])
                o_offs = []
                for t in group:
                    nE = len(t.Es) if t.Es else 0
                    nsave = len(t.tsave) if t.options.save_states else 1
                    sb = _align(nsave * t.n * t.n * 8)
                    nb = sb + _align(max(nE * len(t.tsave) * 8, 8))
                    o = self._dev.alloc(nb)
                    if o is None:
                        raise MemoryError
                    outs_held[t.id] = (o, nb, sb)
                    o_offs.append(o)
                plans.append((group, layout, desc_off, info_off, in_bytes, h_in, d_in, d_ws,
                              ws_bytes, maxK, maxE, maxT))
        except MemoryError:
            for arena, o, nb in held:
                arena.release(o, nb)
            for o, nb, _ in outs_held.values():
                self._dev.release(o, nb)
            return None

        dev_base = self._dev_buf.data_ptr()
        host_base = self._host_buf.data_ptr()
        host_np = self._host_buf.numpy()
        now = time.perf_counter()
        outputs, infos_host = {}, {}
        prof = {}

        def mark(name, t0):
            prof[name] = prof.get(name, 0.0) + time.perf_counter() - t0

        t_ctx = time.perf_counter()
        with torch.cuda.stream(stream):
            mark('enter_stream', t_ctx)
            for (group, layout, desc_off, info_off, in_bytes, h_in, d_in, d_ws, ws_bytes, maxK,
                 maxE, maxT) in plans:
                sv = host_np[h_in:h_in + in_bytes]
                base_in = dev_base + d_in
                host_in = host_base + h_in
                descs = (_lib.RaggedInstance * len(group))()
                for i, t in enumerate(group):
                    ent = layout[i]
                    o, nb, sb = outs_held[t.id]

                    def copy_in(at, arrs):
                        p = at
                        for a in arrs:
                            b = np.ascontiguousarray(a).view(np.uint8).ravel()
                            sv[p:p + b.size] = b
                            p += b.size

                    copy_in(ent['H'], [t.H])
                    copy_in(ent['L'], t.Ls)
                    copy_in(ent['rho0'], [t.rho0])
                    if t.Es:
                        copy_in(ent['E'], t.Es)
                    copy_in(ent['tsave'], [t.tsave])
                    d = descs[i]
                    d.n, d.n_jumps = t.n, len(t.Ls)
                    d.n_exp, d.n_tsave = (len(t.Es) if t.Es else 0), len(t.tsave)
                    d.rho0_is_ket = int(t.rho0.shape[-1] == 1 and t.n > 1)
                    d.save_states = int(bool(t.options.save_states))
                    d.t0 = float(t.tsave[0] if t.options.t0 is None else t.options.t0)
                    d.H, d.L = base_in + ent['H'], base_in + ent['L']
                    d.rho0, d.E, d.tsave = base_in + ent['rho0'], base_in + ent['E'], base_in + ent['tsave']
                    d.states, d.expects = dev_base + o, dev_base + o + sb
                    # step counts and status go straight to page-locked host memory, which
                    # the device reaches through unified addressing: the dispatcher polls
                    # the status word and hands a result out as soon as it is written
                    d.infos = host_in + info_off + _INFO * i
                    d.status = host_in + info_off + _INFO * i + 12
                    d.cancel = host_in + info_off + _INFO * i + 16
                    t.t_launch = now
                raw = np.frombuffer(bytes(descs), dtype=np.uint8)
                sv[desc_off:desc_off + raw.size] = raw
                words = sv[info_off:info_off + _INFO * len(group)].view(np.int32).reshape(-1, _INFO // 4)
                words[:, 3] = -1  # status: not yet written
                words[:, 4] = 0   # cancel word
                with self._cancel_lock:  # a cancel() that came during the launch
                    for i, t in enumerate(group):
                        t._cancel_word = (h_in + info_off + _INFO * i + 16) // 4
                        if t._cancel_requested:
                            words[i, 4] = 1
                count = len(group)
                if key[0] == 'large':  # descriptors and live count go to the stream's slot
                    sv[info_off:info_off + 4] = np.array([count], np.int32).view(np.uint8)
                t1 = time.perf_counter()
                self._dev_buf[d_in:d_in + in_bytes].copy_(self._host_buf[h_in:h_in + in_bytes],
                                                         non_blocking=True)
                mark('h2d', t1)
                opts = self._ode_options(group[0], len(group))
                t1 = time.perf_counter()
                if key[0] == 'small':
                    rc = self.lib.dqb_mesolve_ragged(base_in + desc_off, count, key[1], maxK, opts,
                                                     dev_base + d_ws, ws_bytes, stream.cuda_stream)
                    _lib.check(rc, 'dqb_mesolve_ragged')
                else:  # host-to-device straight into the slot (no device-to-device copy)
                    slot_desc, slot_count = self._large_slot_tables(stream, key[1])
                    self._dev_buf[slot_desc:slot_desc + raw.size].copy_(
                        self._host_buf[h_in + desc_off:h_in + desc_off + raw.size], non_blocking=True)
                    self._dev_buf[slot_count:slot_count + 4].copy_(
                        self._host_buf[h_in + info_off:h_in + info_off + 4], non_blocking=True)
                    rc = self.lib.dqb_mesolve_dense_large_ragged(
                        dev_base + slot_desc, self.max_large_wave, dev_base + slot_count, key[1],
                        self.LARGE_MAX_JUMPS, self.LARGE_MAX_EXP, self.LARGE_MAX_TSAVE, opts,
                        dev_base + d_ws, ws_bytes, stream.cuda_stream)
                    _lib.check(rc, 'dqb_mesolve_dense_large_ragged')
                mark('launch', t1)
                t1 = time.perf_counter()
                for i, t in enumerate(group):
                    o, nb, sb = outs_held[t.id]
                    nE = len(t.Es) if t.Es else 0
                    nsave = len(t.tsave) if t.options.save_states else 1
                    st = self._dev_buf[o:o + nsave * t.n * t.n * 8]
                    ex = self._dev_buf[o + sb:o + sb + nE * len(t.tsave) * 8]
                    outputs[t.id] = (st.view(torch.complex64).view(nsave, t.n, t.n),
                                     ex.view(torch.complex64).view(nE, len(t.tsave)) if nE else None)
                    infos_host[t.id] = (h_in + info_off + _INFO * i)
                    t._out = (self._dev, o, nb)
            t1 = time.perf_counter()
            ev = torch.cuda.Event()
            ev.record(stream)
            mark('event', t1)
        t1 = time.perf_counter()
        w = _Wave(key[0], tickets, stream, ev, held, 0, outputs)
        w.infos_host = infos_host
        w.pending = list(tickets)
        w.status_words = np.array([(infos_host[t.id] + 12) // 4 for t in tickets], np.int64)
        mark('exit', t1)
        self.launch_profile.append((key, prof))
        return w

    def _large_slot(self, stream, n):
        """Fixed workspace, descriptor table and live-count word of (stream, n): waves
        through the same slot keep every launch parameter, so the RK-loop graph captured for
        the first wave is reused by all later ones."""
        key = (id(stream), n)
        with self._lock:
            slot = self._large_slots.get(key)
        if slot is None:
            ws_bytes = self.lib.dqb_mesolve_dense_large_ragged_workspace_size(
                n, self.LARGE_MAX_JUMPS, self.LARGE_MAX_EXP, self.LARGE_MAX_TSAVE,
                self.max_large_wave)
            tables = ctypes.sizeof(_lib.RaggedInstance) * self.max_large_wave + 256
            ws_off = self._dev.alloc(ws_bytes)
            tab_off = self._dev.alloc(tables)
            if ws_off is None or tab_off is None:
                if ws_off is not None:
                    self._dev.release(ws_off, ws_bytes)
                if tab_off is not None:
                    self._dev.release(tab_off, tables)
                raise MemoryError
            slot = (ws_off, ws_bytes, tab_off, tab_off + tables - 256)
            with self._lock:
                self._large_slots[key] = slot
        return slot[0], slot[1]

    def _large_slot_tables(self, stream, n):
        slot = self._large_slots[(id(stream), n)]
        return slot[2], slot[3]

    def warmup(self, large_dims=(128, 256), method=Tsit5(), options: Options = Options()) -> None:  # noqa: B008
        """Run a trivial request through every stream of every class, one at a time (free
        streams are used round-robin): this loads every kernel and captures every
        large-path graph before serving starts.

        A large-path graph is specific to the method's tolerances and to
        ``options.precision``: warm up with those of the requests to come.  A request with
        other values makes its wave capture a new graph while it is being served, and graph
        instantiation can wait for the conditional graphs already running on the device,
        holding up every stream meanwhile."""
        torch = self._torch
        # 'auto' serves large waves in either arithmetic: capture both
        large_opts = ([dataclasses.replace(options, precision=p) for p in ('fp32', 'tf32x3')]
                      if options.precision == 'auto' else [options])
        plan = [(n, len(self._free_streams['small']), Options()) for n in (8, 24, 48)]
        plan += [(n, len(self._free_streams['large']), o) for n in large_dims for o in large_opts]
        done = []
        for n, reps, opt in plan:
            a = np.diag(np.sqrt(np.arange(1, n)), 1).astype(np.complex64)
            for _ in range(reps):
                t = self.submit(np.zeros((n, n), np.complex64), [a],
                                np.eye(n, 1, dtype=np.complex64), [0.0, 0.1], method=method,
                                options=opt)
                t.result()
                t.release()
                done.append(t)
        torch.cuda.synchronize(self.dev)
        with self._lock:
            for t in done:
                self.finished.remove(t)

    def _finish_ticket(self, w: _Wave, t: Ticket) -> None:
        torch = self._torch
        st, ex = w.outputs[t.id]
        o = w.infos_host[t.id]
        # status first, then the step counts (written before it on the device)
        status = int(self._host_i32[(o + 12) // 4])
        nsteps, nacc, nrej = (int(v) for v in self._host_i32[o // 4:o // 4 + 3])
        t.t_done = time.perf_counter()
        if status == _lib.INST_MAX_STEPS:
            t._error = RuntimeError(_MAX_STEPS_MSG)
        elif status == _lib.INST_NONFINITE:
            t._error = RuntimeError('The solution became non-finite (NaN or inf) during '
                                    'the integration.')
        elif status == _lib.INST_NOT_HERMITIAN:
            t._error = RuntimeError('Argument y0 is not hermitian.')
        elif status == _lib.INST_CANCELLED:
            t._error = CancelledError(f'request {t.id} cancelled')
        elif status != _lib.INST_OK:
            t._error = RuntimeError(f'request ended with status {status}')
        if t._error is not None:
            t.release()
        else:
            t._result = MESolveResult(
                tsave=t.tsave, method=t.method, gradient=None, options=t.options,
                states=st, expects=ex,
                infos=AdaptiveStepInfos(torch.tensor(nsteps), torch.tensor(nacc),
                                        torch.tensor(nrej)))
        self.finished.append(t)
        t._event.set()

    def _finish(self, w: _Wave) -> None:
        for t in w.pending:  # the whole wave is done: every status word is final
            self._finish_ticket(w, t)
        w.pending = []
        for t in w.tickets:  # releases asked for while the wave was still running
            t._wave_ended()
        for arena, off, nb in w.keep:
            arena.release(off, nb)
