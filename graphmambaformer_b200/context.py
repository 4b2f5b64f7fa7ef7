"""Asynchronous banded SW on host buffers through the C ABI's contexts
(``gmf_ctx_create`` / ``gmf_batch_submit`` / ``gmf_batch_poll`` /
``gmf_batch_wait``).

The context owns the device side: per slot a stream, pinned staging memory
and a device arena.  A submitted batch goes to the device in one copy, runs
the batched SW, and comes back in one copy; with several slots, consecutive
batches overlap their copies with each other's kernels.  Results land in
numpy arrays owned by the :class:`Ticket`.  This is the serving form of the
extension stage for callers that hold their data on the host (the reference
has no counterpart: its GPU wrappers run synchronously on tensors).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _native
from .extension import SWResult
from .synth import PairSet


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class Ticket:
    """A submitted batch: its id and the host arrays its results land in."""

    id: int
    n: int
    traceback: bool
    out: dict
    keep: tuple  # the inputs, alive until the batch is complete

    def result(self) -> SWResult:
        o = self.out
        r = SWResult(o["score"], o["qe"], o["te"], error_flags=int(o["err"][0]))
        if self.traceback:
            r.query_start, r.target_start = o["qs"], o["ts"]
            r.op_counts = o["counts"].reshape(self.n, 4)
            r.cigar_start, r.cigar_len = o["cstart"], o["clen"]
            r.cigar_words = o["cigar"][: int(o["used"][0])]
        return r


class AlignContext:
    """One gmf_ctx on ``device`` with ``slots`` batches in flight and
    ``memory_budget`` bytes of device memory (0: no limit)."""

    def __init__(self, device: int = 0, slots: int = 3, memory_budget: int = 0):
        self._lib = _native.lib()
        h = ctypes.c_void_p()
        _native.check("gmf_ctx_create", self._lib.gmf_ctx_create(int(device), int(slots), int(memory_budget),
                                                                 ctypes.byref(h)))
        self._h = h
        self.device = int(device)

    def close(self) -> None:
        if self._h is not None and self._h.value:
            _native.check("gmf_ctx_destroy", self._lib.gmf_ctx_destroy(self._h))
        self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, pairs: PairSet, params: _native.GmfSwParams, traceback: bool = True) -> Ticket:
        n = len(pairs)
        q = np.ascontiguousarray(pairs.query, np.int8)
        t = np.ascontiguousarray(pairs.target, np.int8)
        qo = np.ascontiguousarray(pairs.query_off, np.int64)
        to = np.ascontiguousarray(pairs.target_off, np.int64)
        hb = np.ascontiguousarray(np.broadcast_to(np.asarray(pairs.half_band, np.int32), (n,)))
        off = np.ascontiguousarray(np.broadcast_to(np.asarray(pairs.band_offset, np.int32), (n,)))
        go = None if pairs.xdrop_group_off is None else np.ascontiguousarray(pairs.xdrop_group_off, np.int32)
        hp = _native.GmfHostPairs(n, _p(q), _p(qo), _p(t), _p(to), _p(hb), _p(off), _p(go),
                                  0 if go is None else len(go) - 1)
        cap = int(qo[-1] + to[-1] + n) if traceback else 0
        m = max(n, 1)
        # every output is written by the library (only the CIGAR words it used are touched)
        out = dict(score=np.empty(m, np.int32), qe=np.empty(m, np.int32), te=np.empty(m, np.int32),
                   used=np.zeros(1, np.int64), err=np.zeros(1, np.int32))
        if traceback:
            out.update(qs=np.empty(m, np.int32), ts=np.empty(m, np.int32), counts=np.empty(4 * m, np.int32),
                       cigar=np.empty(max(cap, 1), np.uint32), cstart=np.empty(m, np.int64),
                       clen=np.empty(m, np.int32))
        g = out.get
        res = _native.GmfHostSwResults(_p(out["score"]), _p(out["qe"]), _p(out["te"]), _p(g("qs")), _p(g("ts")),
                                       _p(g("counts")), _p(g("cigar")), cap, _p(g("cstart")), _p(g("clen")),
                                       _p(out["used"]), _p(out["err"]))
        tid = ctypes.c_int64(0)
        _native.check("gmf_batch_submit", self._lib.gmf_batch_submit(self._h, ctypes.byref(hp), ctypes.byref(params),
                                                                     ctypes.byref(res), ctypes.byref(tid)))
        for k in list(out):
            if k not in ("used", "err"):
                out[k] = out[k][:n] if k != "cigar" and k != "counts" else out[k]
        if traceback:
            out["counts"] = out["counts"][: 4 * n]
        return Ticket(int(tid.value), n, traceback, out, (q, t, qo, to, hb, off, go, res))

    def poll(self, ticket: Ticket) -> Optional[SWResult]:
        """The batch's results when it is complete, else None."""
        st = self._lib.gmf_batch_poll(self._h, ticket.id)
        if st == _native.GMF_ERR_NOT_READY:
            return None
        _native.check("gmf_batch_poll", st)
        return ticket.result()

    def wait(self, ticket: Ticket) -> SWResult:
        _native.check("gmf_batch_wait", self._lib.gmf_batch_wait(self._h, ticket.id))
        return ticket.result()

    def align(self, pairs: PairSet, params: _native.GmfSwParams, traceback: bool = True) -> SWResult:
        """submit + wait: one synchronous batch through the C ABI."""
        return self.wait(self.submit(pairs, params, traceback))
