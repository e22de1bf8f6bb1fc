"""Serving scheduler logic on the CPU (slots and solves replaced by fakes): admission by
memory footprint, slot reuse per grid size, eviction of idle slots, and concurrency."""
from __future__ import annotations

import threading
import time

import numpy
import torch

from meanas_b200 import serving


class FakeSlot:
    created = []

    def __init__(self, shape, req, device, precision, xchunk, autotune=True):
        self.shape = shape
        self.bytes = serving.slot_bytes(shape, precision)
        self.closed = False
        FakeSlot.created.append(self)

    def close(self):
        self.closed = True


def _req(shape, tag):
    dxes = [[numpy.ones(s) for s in shape] for _ in range(2)]
    return serving.Request(0.3, dxes, numpy.zeros(3 * int(numpy.prod(shape)), complex), None, tag=tag)


def _server(budget, max_active, run_time=0.02):
    """A server whose workers run on the CPU with fake slots and a sleeping solve."""
    srv = serving.FDFDServer.__new__(serving.FDFDServer)
    srv.device = torch.device('cpu')
    srv.budget = budget
    srv.precision = 'mixed'
    srv.rtol = 1e-8
    srv.maxiter = None
    srv.xchunk = None
    srv.autotune = False
    srv._method = 'mixed'
    srv._cv = threading.Condition()
    srv._waiting = serving.collections.deque()
    srv._idle = serving.collections.defaultdict(list)
    srv._used = 0
    srv._closed = False
    srv.stats = serving.collections.Counter()
    srv._slot_factory = FakeSlot
    srv.active = 0
    srv.max_seen = 0
    lock = threading.Lock()

    def fake_run(slot, req):
        with lock:
            srv.active += 1
            srv.max_seen = max(srv.max_seen, srv.active)
        time.sleep(run_time)
        with lock:
            srv.active -= 1
        return serving.Result(E=None, info=None, arrival=req.arrival, start=0, finish=time.perf_counter(),
                              tag=(req.tag, id(slot)))
    srv._run = fake_run
    srv._threads = [threading.Thread(target=srv._worker, daemon=True) for _ in range(max_active)]
    for t in srv._threads:
        t.start()
    return srv


def test_slots_are_reused_per_size_and_solves_overlap():
    FakeSlot.created.clear()
    srv = _server(budget=10 ** 12, max_active=4)
    futs = [srv.submit(_req((16, 16, 1), k)) for k in range(12)]
    res = [f.result(timeout=10) for f in futs]
    srv.shutdown()
    assert len(res) == 12
    assert srv.max_seen == 4                       # four solves in flight at once
    assert len(FakeSlot.created) == 4              # one slot per concurrent solve, then reused
    assert srv.stats['slot_reuse'] == 8


def test_admission_respects_the_memory_budget_and_evicts_idle_slots():
    FakeSlot.created.clear()
    small, big = (32, 32, 1), (64, 64, 64)
    b_small = serving.slot_bytes(small, 'mixed')
    b_big = serving.slot_bytes(big, 'mixed')
    srv = _server(budget=b_big + b_small, max_active=4)
    futs = [srv.submit(_req(small, k)) for k in range(3)]
    [f.result(timeout=10) for f in futs]
    # a big request needs the idle small slots released first
    srv.submit(_req(big, 'big')).result(timeout=10)
    srv.shutdown()
    assert srv.stats['slot_evict'] >= 1
    assert srv._used <= srv.budget


def test_oversized_request_is_refused():
    srv = _server(budget=1000, max_active=1)
    f = srv.submit(_req((64, 64, 64), 0))
    try:
        f.result(timeout=5)
        raise AssertionError('expected MemoryError')
    except MemoryError:
        pass
    srv.shutdown()
