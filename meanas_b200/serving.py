"""Continuous-batching FDFD server: many solves of different sizes in flight at once.

Requests (``omega``, ``dxes``, ``J``, ``epsilon``) are submitted as they arrive and
return futures.  The server keeps **slots**: device-resident solver state for one grid
size (a ``GridOperator`` with its plan, the solve workspace with the Krylov vectors,
the field buffer and a CUDA stream).  A slot serves request after request of its size:
a new request is copied into the slot's buffers and the plan is refilled in place
(``fdfd_plan_update``), so the iteration bodies captured as CUDA graphs for that size
are replayed, not re-captured.

Admission: a worker picks the oldest waiting request whose slot (idle, or new within
the HBM budget) is available; idle slots of other sizes are released when the budget
needs room.  Up to ``max_active`` solves run at once, each on its own stream and
host thread (the C call releases the GIL), so requests that arrive while others are
on the GPU start as soon as a slot and memory free up and their kernels overlap on
the device.  Every solve is deterministic (fixed-order reductions, fixed tiling per
slot), so a request's result does not depend on what else is in flight.
"""
from __future__ import annotations

import collections
import concurrent.futures
import dataclasses
import threading
import time
from typing import Any

import numpy
import torch

from . import operators
from .operators import GridOperator, SolveInfo

# one autotuning run per (device, grid size, precision) at a time; later slots of that
# size take its result, so every slot of a size has the same tiling
_TUNE_LOCKS: dict[tuple, threading.Lock] = collections.defaultdict(threading.Lock)
_TUNE_GUARD = threading.Lock()


@dataclasses.dataclass
class Request:
    omega: complex
    dxes: Any
    J: Any
    epsilon: Any
    arrival: float = 0.0          # host time (perf_counter) the request arrived
    tag: Any = None

    @property
    def shape(self) -> tuple[int, int, int]:
        return tuple(int(numpy.size(d)) for d in self.dxes[0])


@dataclasses.dataclass
class Result:
    E: numpy.ndarray
    info: SolveInfo
    arrival: float
    start: float
    finish: float
    tag: Any = None

    @property
    def latency(self) -> float:
        return self.finish - self.arrival


def slot_bytes(shape: tuple[int, int, int], precision: str) -> int:
    """Device bytes one slot holds for a grid: inputs, field, plan and solve workspace."""
    n = 3 * int(numpy.prod(shape))
    s = sum(shape)
    inputs = n * 8 + n * 16 + n * 16              # epsilon, J, E
    tables = 2 * 4 * s * 16 + 256 * 1024          # dx tables (host copies + plan) and slack
    fp32 = n * 4 if precision == 'mixed' else 0
    ws = 2 * n * 16 + 8 * n * (8 if precision == 'mixed' else 16) + (4 * n * 16 if precision != 'mixed' else 0)
    return inputs + tables + fp32 + ws


class _Slot:
    def __init__(self, shape, req: Request, device: torch.device, precision: str, xchunk: int | None,
                 autotune: bool = True):
        self.shape = shape
        self.precision = precision
        self.stream = torch.cuda.Stream(device=device)
        prec = 'c64' if precision == 'mixed' else 'c128'
        with torch.cuda.device(device), torch.cuda.stream(self.stream):
            self.op = GridOperator(req.omega, req.dxes, req.epsilon, device=device, fp32=(precision == 'mixed'))
            if xchunk:
                self.op.set_xchunk(prec, xchunk)
                self.xchunk = xchunk
            elif autotune:
                # the first slot of a size times the x-chunk candidates on its own stream
                key = (self.op.device.index, tuple(shape), prec)
                with _TUNE_GUARD:
                    lock = _TUNE_LOCKS[key]
                with lock:
                    tuned = operators._TUNED.get(key)
                    if tuned is None:
                        self.op.autotune(methods=('mixed' if precision == 'mixed' else 'cocg',))
                    else:
                        self.op.set_xchunk(prec, tuned)
                    self.xchunk = operators._TUNED.get(key)
            self.J = torch.empty(self.op.n, dtype=torch.complex128, device=device)
            self.E = torch.empty(self.op.n, dtype=torch.complex128, device=device)
            self.E_host = torch.empty(self.op.n, dtype=torch.complex128).pin_memory()
        self.fresh = True
        self.bytes = slot_bytes(shape, precision)

    xchunk: int | None = None

    def close(self):
        self.op.close()


class FDFDServer:
    """Continuous-batching server (see the module docstring).

    ``max_active``: solves in flight at once.  ``hbm_budget``: bytes of device memory
    the slots may hold (default: 80 % of free memory at start-up).  ``precision``:
    ``'mixed'`` (complex64 BiCGSTAB + complex128 refinement) or ``'fp64'`` (COCG).
    ``rtol``: true FP64 residual target.  ``xchunk``: optional fixed x planes per CTA;
    otherwise (``autotune=True``) the first slot of each grid size times the candidates
    (``GridOperator.autotune``) and every later slot of that size reuses the choice, or
    (``autotune=False``) the library's default.
    """

    def __init__(self, device: Any | None = None, *, max_active: int = 8, hbm_budget: int | None = None,
                 precision: str = 'mixed', rtol: float = 1e-8, maxiter: int | None = 200000,
                 xchunk: int | None = None, autotune: bool = True):
        self.device = torch.device(device) if device is not None else torch.device('cuda', 0)
        self._slot_factory = _Slot
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(0.8 * free)
        self.budget = int(hbm_budget)
        self.precision = precision
        self.rtol = rtol
        self.maxiter = maxiter
        self.xchunk = xchunk
        self.autotune = autotune
        self._method = 'mixed' if precision == 'mixed' else 'cocg'
        self._cv = threading.Condition()
        self._waiting: collections.deque[tuple[Request, concurrent.futures.Future]] = collections.deque()
        self._idle: dict[tuple, list[_Slot]] = collections.defaultdict(list)
        self._used = 0                      # bytes held by all slots (idle + busy)
        self._closed = False
        self.stats = collections.Counter()
        self._threads = [threading.Thread(target=self._worker, daemon=True, name=f'fdfd-worker-{i}')
                         for i in range(max_active)]
        for t in self._threads:
            t.start()

    # ------------------------------------------------------------------ public API
    def submit(self, req: Request) -> concurrent.futures.Future:
        if not req.arrival:
            req.arrival = time.perf_counter()
        fut: concurrent.futures.Future = concurrent.futures.Future()
        need = slot_bytes(req.shape, self.precision)
        if need > self.budget:
            fut.set_exception(MemoryError(f'request needs {need} bytes, budget is {self.budget}'))
            return fut
        with self._cv:
            if self._closed:
                raise RuntimeError('server is shut down')
            self._waiting.append((req, fut))
            self._cv.notify()
        return fut

    def shutdown(self) -> None:
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        for slots in self._idle.values():
            for s in slots:
                s.close()
        self._idle.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.shutdown()

    # ------------------------------------------------------------------ scheduling
    def _take(self) -> tuple[Request, concurrent.futures.Future, _Slot | None] | None:
        """Under the lock: the oldest waiting request that can start now, with its slot
        (None = create one; its bytes are already reserved)."""
        for pos, (req, fut) in enumerate(self._waiting):
            shape = req.shape
            if self._idle[shape]:
                del self._waiting[pos]
                self.stats['slot_reuse'] += 1
                return req, fut, self._idle[shape].pop()
            need = slot_bytes(shape, self.precision)
            # free idle slots of other sizes until the new one fits
            while self._used + need > self.budget:
                victim = next((v[0] for v in self._idle.values() if v), None)
                if victim is None:
                    break
                self._idle[victim.shape].remove(victim)
                self._used -= victim.bytes
                victim.close()
                self.stats['slot_evict'] += 1
            if self._used + need <= self.budget:
                del self._waiting[pos]
                self._used += need
                self.stats['slot_new'] += 1
                return req, fut, None
            # this request must wait for memory; let a smaller one behind it start
        return None

    def _worker(self) -> None:
        if self.device.type == 'cuda':
            torch.cuda.set_device(self.device)
        while True:
            with self._cv:
                item = None
                while item is None:
                    if self._closed and not self._waiting:
                        return
                    item = self._take()
                    if item is None:
                        self._cv.wait()
            req, fut, slot = item
            try:
                if slot is None:
                    slot = self._slot_factory(req.shape, req, self.device, self.precision, self.xchunk,
                                              self.autotune)
                    self.stats['slot_tuned'] += int(getattr(slot, 'xchunk', None) is not None)
                fut.set_result(self._run(slot, req))
            except BaseException as exc:  # the error goes to the caller
                fut.set_exception(exc)
            finally:
                with self._cv:
                    if slot is not None:
                        self._idle[slot.shape].append(slot)
                    else:  # slot creation failed: give its reservation back
                        self._used -= slot_bytes(req.shape, self.precision)
                    self._cv.notify_all()

    def _run(self, slot: _Slot, req: Request) -> Result:
        start = time.perf_counter()
        with torch.cuda.device(self.device), torch.cuda.stream(slot.stream):
            if not slot.fresh:
                slot.op.update(req.omega, req.dxes, req.epsilon)
            slot.fresh = False
            J = req.J if isinstance(req.J, torch.Tensor) else torch.from_numpy(numpy.asarray(req.J, dtype=complex))
            slot.J.copy_(J.reshape(-1).to(torch.complex128), non_blocking=J.is_pinned())
            E, info = slot.op.solve(slot.J, out=slot.E, method=self._method, rtol=self.rtol,
                                    criterion='true', maxiter=self.maxiter)
            slot.E_host.copy_(E, non_blocking=True)
            slot.stream.synchronize()
            out = slot.E_host.numpy().copy()
        finish = time.perf_counter()
        return Result(E=out, info=info, arrival=req.arrival, start=start, finish=finish, tag=req.tag)


def poisson_stream(n: int, rate: float, seed: int = 0, shapes=None) -> list[tuple[float, Any]]:
    """``n`` seeded serving requests with exponential inter-arrival times (mean 1/rate s):
    ``[(offset_seconds, Problem), ...]`` with problems from ``workloads.serving_request``."""
    from . import workloads
    rng = numpy.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate))
        shape = None if shapes is None else shapes[int(rng.integers(len(shapes)))]
        out.append((t, workloads.serving_request(rng, shape=shape)))
    return out


def replay(server: FDFDServer, stream: list[tuple[float, Any]]) -> list[Result]:
    """Submit each request at its arrival offset (real time) and wait for all results."""
    t0 = time.perf_counter()
    futs = []
    for k, (offset, p) in enumerate(stream):
        delay = t0 + offset - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        futs.append(server.submit(Request(p.omega, p.dxes, p.J, p.epsilon, arrival=t0 + offset, tag=k)))
    return [f.result() for f in futs]
