"""Host logic of the serving loop (continuous batching under a memory
budget), with stand-in workers in place of the device pipeline:

* no batch exceeds the read cap or, with what is in flight, the budget;
* every request is answered with its own reads' results, in order;
* a request waits while the budget is full and runs once memory frees;
* a failing batch fails every request in it, and only those; the budget
  and the worker come back after it.
"""

from __future__ import annotations

import queue
import threading
import time

import numpy as np
import pytest

from graphmambaformer_b200.chaining import AnchorCSR, ChainingConfig
from graphmambaformer_b200.config import ExtensionConfig
from graphmambaformer_b200.serving import AlignServer, estimate_bytes


class _Worker:
    """Stands in for BatchAligner: answers each read with its length."""

    def __init__(self, log, delay=0.002, fail_on=None):
        self.log, self.delay, self.fail_on = log, delay, fail_on

    def align(self, reads, anchors):
        assert anchors is not None and len(anchors) == len(reads)
        self.log.append((len(reads), sum(len(r) for r in reads)))
        time.sleep(self.delay)
        if self.fail_on is not None and any(len(r) == self.fail_on for r in reads):
            raise RuntimeError("device step failed")
        return [len(r) for r in reads]


def _server(workers, budget, max_reads):
    """An AlignServer without a device: the dispatcher and the workers'
    threads as in production, the device pipeline replaced."""
    s = AlignServer.__new__(AlignServer)
    s.ccfg, s.ecfg = ChainingConfig(), ExtensionConfig()
    s.budget, s.max_batch_reads, s.index = int(budget), int(max_reads), None
    s.workers = workers
    s.free = queue.Queue()
    for w in workers:
        s.free.put(w)
    s.pending = queue.Queue()
    s.in_flight_bytes, s.lock = 0, threading.Lock()
    s.completed, s.batches, s._next = [], 0, 0
    s._stop = threading.Event()
    s._dispatcher = threading.Thread(target=s._dispatch, daemon=True)
    s._threads = []
    return s


def _anchors(lens):
    counts = np.array([3] * len(lens), np.int64)
    off = np.concatenate([[0], np.cumsum(counts)])
    n = int(off[-1])
    return AnchorCSR(off, np.zeros(n, np.int32), np.zeros(n, np.int32), np.full(n, 15, np.int32),
                     np.ones(n, np.int8))


def _reads(rng, k):
    return [np.zeros(int(x), np.int8) for x in rng.integers(100, 2000, k)]


def test_batches_respect_the_read_cap_and_answer_every_request():
    log = []
    s = _server([_Worker(log), _Worker(log)], budget=8 << 30, max_reads=40).start()
    rng = np.random.default_rng(0)
    reqs = [_reads(rng, int(rng.integers(1, 30))) for _ in range(120)]
    futs = [s.submit(r, _anchors([len(x) for x in r])) for r in reqs]
    for r, f in zip(reqs, futs):
        assert f.result(timeout=60) == [len(x) for x in r]
    s.stop()
    assert max(n for n, _ in log) <= 40
    assert sum(n for n, _ in log) == sum(len(r) for r in reqs)
    assert s.in_flight_bytes == 0 and s.free.qsize() == 2
    assert s.latency_stats()["requests"] == 120


def test_budget_holds_requests_until_memory_frees():
    log = []
    one = estimate_bytes(np.array([1000]), 3, ExtensionConfig(), ChainingConfig().max_chains)
    # room for two one-read requests at a time, four workers
    s = _server([_Worker(log, delay=0.02) for _ in range(4)], budget=2 * one + 1, max_reads=1).start()
    peak = [0]

    def watch():
        while not s._stop.is_set():
            with s.lock:
                peak[0] = max(peak[0], s.in_flight_bytes)
            time.sleep(0.0005)

    t = threading.Thread(target=watch, daemon=True)
    t.start()
    futs = [s.submit([np.zeros(1000, np.int8)], _anchors([1000])) for _ in range(12)]
    assert all(f.result(timeout=60) == [1000] for f in futs)
    s.stop()
    t.join(timeout=5)
    assert 0 < peak[0] <= 2 * one + 1
    assert s.in_flight_bytes == 0
    with pytest.raises(ValueError, match="budget"):
        s.submit([np.zeros(10**7, np.int8)], _anchors([10**7]))


def test_a_failing_batch_fails_only_its_requests():
    log = []
    s = _server([_Worker(log, fail_on=777)], budget=8 << 30, max_reads=1).start()
    ok1 = s.submit([np.zeros(500, np.int8)], _anchors([500]))
    bad = s.submit([np.zeros(777, np.int8)], _anchors([777]))
    ok2 = s.submit([np.zeros(600, np.int8)], _anchors([600]))
    assert ok1.result(timeout=30) == [500]
    with pytest.raises(RuntimeError, match="device step failed"):
        bad.result(timeout=30)
    assert ok2.result(timeout=30) == [600]
    s.stop()
    assert s.in_flight_bytes == 0 and s.free.qsize() == 1


def test_requests_need_anchors_without_an_index():
    s = _server([_Worker([])], budget=8 << 30, max_reads=8)
    with pytest.raises(ValueError, match="anchors are required"):
        s.submit([np.zeros(100, np.int8)])
