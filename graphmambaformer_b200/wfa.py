"""Unit-cost global wavefront alignment (WFA) on the device.

Drop-in for the reference's wavefront pieces:

* :class:`WavefrontAligner` -- ``alignment/extension.py`` L308-463
  (``align(query, target) -> (edit_distance, cigar)``, raising
  ``RuntimeError`` beyond ``cfg.wfa_max_distance``), plus ``align_batch``;
* :func:`wfa_distance` -- ``accel/cuda_kernels.py`` L569-600 (padded
  ``(B, L)`` code tensors in, int32 distances out, ``-1`` beyond the bound).

A batch runs in two device passes: ``gmf_wfa_distance`` finds every pair's
distance (one warp per pair, the live wavefronts in shared memory), then
``gmf_wfa_align`` recomputes each pair's wavefronts to exactly that distance,
keeping the history ((d+1)^2 offsets, carved from the workspace), and walks
it back to the CIGAR with the reference's tie order.  Pairs whose histories
together exceed the budget are split over several calls.  Every computation
runs in the gmf CUDA library; without a GPU the calls raise.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import _native
from .config import ExtensionConfig
from .device import WORKSPACE, bind, np_ptr, ptr, require_cuda, stream_handle, to_device
from .types import words_to_cigar

# history entries (int32) one gmf_wfa_align call may hold: 2 GiB
HISTORY_BUDGET = 1 << 29


@dataclass
class DeviceWfaPairs:
    """Pairs resident on the device (CSR layout) with the host values the
    entry points take."""

    n: int
    query: torch.Tensor
    query_off: torch.Tensor
    target: torch.Tensor
    target_off: torch.Tensor
    h_qlen: np.ndarray
    h_tlen: np.ndarray
    device: torch.device

    @property
    def max_len(self) -> int:
        return int(max(self.h_qlen.max(initial=0), self.h_tlen.max(initial=0)))

    def c(self, order: Optional[torch.Tensor] = None) -> _native.GmfWfaPairs:
        return _native.GmfWfaPairs(self.n, ptr(self.query), ptr(self.query_off), ptr(self.target),
                                   ptr(self.target_off), ptr(order), int(self.h_qlen.sum()),
                                   int(self.h_tlen.sum()), self.max_len)


# Grow-only pinned staging of the concatenated codes, per (device, side): the
# sequences are concatenated straight into it, so one host copy and one
# host-to-device copy move a batch.
_STAGE: dict = {}


def _stage_codes(seqs: Sequence[np.ndarray], side: str, dev: torch.device) -> tuple:
    """CSR of the sequences on the device: (codes, offsets on the device,
    host offsets, host lengths).  The copy is enqueued on the current
    stream; the next call waits for it before it reuses the buffer."""
    lens = np.fromiter((len(x) for x in seqs), np.int64, len(seqs))
    off = np.zeros(len(seqs) + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    total = int(off[-1])
    key = (dev.index, side)
    h, done = _STAGE.get(key, (None, None))
    if done is not None:
        done.synchronize()  # the previous batch's copy out of this buffer has finished
    if h is None or h.numel() < max(total, 1):
        h = torch.empty(max(total, 1, int(h.numel() * 1.25) if h is not None else 0), dtype=torch.int8,
                        pin_memory=True)
    if total:
        np.concatenate(seqs, out=h.numpy()[:total], casting="unsafe")
    d = torch.empty(max(total, 1), dtype=torch.int8, device=dev)
    done = torch.cuda.Event()
    if total:
        d.copy_(h[:total], non_blocking=True)
    done.record(torch.cuda.current_stream(dev))
    _STAGE[key] = (h, done)
    return d, to_device(off, dev), off, lens.astype(np.int32)


def upload_wfa_pairs(queries: Sequence[np.ndarray], targets: Sequence[np.ndarray], device=None) -> DeviceWfaPairs:
    if len(queries) != len(targets):
        raise ValueError("queries and targets differ in number")
    dev = require_cuda(device)
    q, qo, _, ql = _stage_codes(queries, "q", dev)
    t, to, _, tl = _stage_codes(targets, "t", dev)
    if len(queries) and max(ql.max(), tl.max()) > (1 << 28):
        raise ValueError("sequence longer than the library's limit (2^28 codes)")
    return DeviceWfaPairs(len(queries), q, qo, t, to, ql, tl, dev)


@dataclass
class WfaBatch:
    """Host pairs as CSR code arrays: pair b is ``query[query_off[b]:
    query_off[b+1]]`` against ``target[target_off[b]: target_off[b+1]]``
    (int8 codes, int64 offsets).  Code arrays in page-locked memory (see
    :meth:`pinned`) go to the device without a host copy."""

    query: np.ndarray
    query_off: np.ndarray
    target: np.ndarray
    target_off: np.ndarray

    def __len__(self) -> int:
        return len(self.query_off) - 1

    @staticmethod
    def of(queries: Sequence[np.ndarray], targets: Sequence[np.ndarray]) -> "WfaBatch":
        if len(queries) != len(targets):
            raise ValueError("queries and targets differ in number")

        def csr(seqs):
            off = np.zeros(len(seqs) + 1, np.int64)
            np.cumsum(np.fromiter((len(x) for x in seqs), np.int64, len(seqs)), out=off[1:])
            codes = np.empty(int(off[-1]), np.int8)
            if len(codes):
                np.concatenate(seqs, out=codes, casting="unsafe")
            return codes, off

        q, qo = csr(queries)
        t, to = csr(targets)
        return WfaBatch(q, qo, t, to)

    def pinned(self) -> "WfaBatch":
        """A copy whose code arrays live in page-locked host memory."""

        def pin(a):
            h = torch.empty(max(len(a), 1), dtype=torch.int8, pin_memory=True)
            h[: len(a)].copy_(torch.from_numpy(np.ascontiguousarray(a, np.int8)))
            return h.numpy()[: len(a)]

        return WfaBatch(pin(self.query), self.query_off.copy(), pin(self.target), self.target_off.copy())


def upload_wfa_batch(batch: WfaBatch, device=None) -> DeviceWfaPairs:
    """The CSR pairs on the device (copies enqueued on the current stream; a
    page-locked code array must stay unchanged until they have run)."""
    dev = require_cuda(device)
    qo, to = np.asarray(batch.query_off, np.int64), np.asarray(batch.target_off, np.int64)
    if len(qo) != len(to) or len(qo) < 1 or qo[0] != 0 or to[0] != 0:
        raise ValueError("query_off and target_off must be offset arrays of the same batch, starting at 0")
    ql, tl = np.diff(qo), np.diff(to)
    if len(ql) and (ql.min() < 0 or tl.min() < 0):
        raise ValueError("offsets must not decrease")
    if len(ql) and max(ql.max(), tl.max()) > (1 << 28):
        raise ValueError("sequence longer than the library's limit (2^28 codes)")
    if len(batch.query) < qo[-1] or len(batch.target) < to[-1]:
        raise ValueError("offsets run past the code arrays")

    def codes(a, n):
        a = np.asarray(a)[:n]
        if a.dtype != np.int8:
            a = a.astype(np.int8)
        return to_device(a, dev) if n else torch.zeros(1, dtype=torch.int8, device=dev)

    return DeviceWfaPairs(len(ql), codes(batch.query, int(qo[-1])), to_device(qo, dev),
                          codes(batch.target, int(to[-1])), to_device(to, dev), ql.astype(np.int32),
                          tl.astype(np.int32), dev)


def _check_bound(max_distance: int, max_len: int) -> int:
    """The bound the device call takes.  No distance exceeds the longer side,
    so a bound above it changes nothing, and a negative bound acts like 0
    (only a pair complete at score 0 succeeds)."""
    md = max(0, min(int(max_distance), int(max_len)))
    if md > _native.MAX_WFA_DISTANCE:
        raise ValueError(f"a distance bound above {_native.MAX_WFA_DISTANCE} on sequences that long is "
                         "beyond the library's limit")
    return md


def _ws(workspace, device: torch.device, nbytes: int) -> torch.Tensor:
    """The caller's workspace (a callable: bytes -> uint8 device tensor) or
    the shared grow-only one."""
    return workspace(nbytes) if workspace is not None else WORKSPACE.get(device, nbytes)


def wfa_distances(dp: DeviceWfaPairs, max_distance: int, stream: Optional[torch.cuda.Stream] = None,
                  out: Optional[torch.Tensor] = None, workspace=None) -> torch.Tensor:
    """Enqueue gmf_wfa_distance; returns the device int32 distances."""
    md = _check_bound(max_distance, dp.max_len)
    out = out if out is not None else torch.empty(max(dp.n, 1), dtype=torch.int32, device=dp.device)
    if dp.n == 0:
        return out[:0]
    order = to_device(np.argsort(-(dp.h_qlen.astype(np.int64) + dp.h_tlen), kind="stable").astype(np.int32),
                      dp.device)
    need = int(_native.lib().gmf_wfa_workspace_bytes(dp.n, dp.max_len, md, 0))
    ws = _ws(workspace, dp.device, need)
    sp = stream_handle(stream, dp.device)
    bind(dp.device, sp)
    pairs = dp.c(order)
    st = _native.lib().gmf_wfa_distance(ctypes.byref(pairs), md, ctypes.c_void_p(out.data_ptr()),
                                        ctypes.c_void_p(ws.data_ptr()), ws.numel(), ctypes.c_void_p(sp))
    _native.check("gmf_wfa_distance", st)
    return out[: dp.n]


@dataclass
class WfaResult:
    """Host copy of a batch's wavefront alignments."""

    distance: np.ndarray                 # int32, -1 beyond the bound
    op_counts: Optional[np.ndarray] = None   # (n, 4): = X I D
    cigar_words: Optional[np.ndarray] = None
    cigar_start: Optional[np.ndarray] = None
    cigar_len: Optional[np.ndarray] = None

    def __len__(self) -> int:
        return len(self.distance)

    def cigar(self, b: int) -> list:
        n = int(self.cigar_len[b])
        if n < 0:
            raise RuntimeError(f"pair {b} has no alignment (distance beyond the bound)")
        s = int(self.cigar_start[b])
        return words_to_cigar(self.cigar_words[s: s + n])


def _sub_batch(dp: DeviceWfaPairs, dist_d: torch.Tensor, h_dist: np.ndarray, idx: np.ndarray) -> tuple:
    """The pairs `idx` of dp as their own device batch (codes copied on the
    device; offsets from the host lengths)."""
    qo = np.zeros(dp.n + 1, np.int64)
    np.cumsum(dp.h_qlen, out=qo[1:])
    to = np.zeros(dp.n + 1, np.int64)
    np.cumsum(dp.h_tlen, out=to[1:])
    ql, tl = dp.h_qlen[idx], dp.h_tlen[idx]
    sqo = np.zeros(len(idx) + 1, np.int64)
    np.cumsum(ql, out=sqo[1:])
    sto = np.zeros(len(idx) + 1, np.int64)
    np.cumsum(tl, out=sto[1:])
    dev = dp.device
    gq = torch.cat([dp.query[qo[p]: qo[p + 1]] for p in idx]) if sqo[-1] else torch.zeros(1, dtype=torch.int8,
                                                                                         device=dev)
    gt = torch.cat([dp.target[to[p]: to[p + 1]] for p in idx]) if sto[-1] else torch.zeros(1, dtype=torch.int8,
                                                                                          device=dev)
    sub = DeviceWfaPairs(len(idx), gq, to_device(sqo, dev), gt, to_device(sto, dev), ql, tl, dev)
    d_sub = dist_d[torch.as_tensor(idx, dtype=torch.long, device=dev)].contiguous()
    return sub, d_sub, h_dist[idx]


def _run_align(sub: DeviceWfaPairs, d_sub: torch.Tensor, h_d: np.ndarray, sp: int, workspace=None) -> dict:
    dev = sub.device
    n = sub.n
    entries = int(_native.lib().gmf_wfa_history_entries(n, np_ptr(sub.h_qlen), np_ptr(sub.h_tlen), np_ptr(h_d)))
    md = int(max(h_d.max(initial=0), 0))
    need = int(_native.lib().gmf_wfa_workspace_bytes(n, sub.max_len, md, entries))
    ws = _ws(workspace, dev, need)
    cap = int(sub.h_qlen.astype(np.int64).sum() + sub.h_tlen.astype(np.int64).sum() + n)
    i32 = dict(dtype=torch.int32, device=dev)
    out = dict(counts=torch.empty((n, 4), **i32), cigar=torch.empty(max(cap, 1), **i32),
               cstart=torch.empty(n, dtype=torch.int64, device=dev), clen=torch.empty(n, **i32),
               used=torch.zeros(1, dtype=torch.int64, device=dev), err=torch.zeros(1, **i32))
    res = _native.GmfWfaResults(ptr(out["counts"]), ptr(out["cigar"]), out["cigar"].numel(), ptr(out["cstart"]),
                                ptr(out["clen"]), ptr(out["used"]), ptr(out["err"]))
    order = to_device(np.argsort(-((h_d.astype(np.int64) + 1) * (sub.h_qlen.astype(np.int64) + sub.h_tlen)),
                                 kind="stable").astype(np.int32), dev)
    pairs = sub.c(order)
    bind(dev, sp)
    st = _native.lib().gmf_wfa_align(ctypes.byref(pairs), ctypes.c_void_p(d_sub.data_ptr()), md,
                                     ctypes.byref(res), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
                                     ctypes.c_void_p(sp))
    _native.check("gmf_wfa_align", st)
    return out


def align_wfa_pairs(queries: Sequence[np.ndarray], targets: Sequence[np.ndarray], max_distance: int = 4096,
                    traceback: bool = True, device=None, history_budget: int = HISTORY_BUDGET) -> WfaResult:
    """Host pairs in, host wavefront alignments out."""
    dp = upload_wfa_pairs(queries, targets, device)
    return align_device_pairs(dp, max_distance, traceback=traceback, history_budget=history_budget)


def align_wfa_batch(batch: WfaBatch, max_distance: int = 4096, traceback: bool = True, device=None,
                    history_budget: int = HISTORY_BUDGET) -> WfaResult:
    """:func:`align_wfa_pairs` for pairs already laid out as CSR arrays."""
    dev = require_cuda(device)
    stream = torch.cuda.current_stream(dev)
    with torch.cuda.stream(stream):
        dp = upload_wfa_batch(batch, dev)
    return align_device_pairs(dp, max_distance, stream=stream, traceback=traceback, history_budget=history_budget)


def history_chunks(hist: np.ndarray, budget: int) -> list:
    """Consecutive ranges [s, e) of pairs whose history entries sum to at
    most ``budget`` each, taken greedily in order; a pair above the budget
    forms a range of its own."""
    n = len(hist)
    cum = np.zeros(n + 1, np.int64)
    np.cumsum(hist, out=cum[1:])
    bounds = [0]
    while bounds[-1] < n:
        s = bounds[-1]
        e = int(np.searchsorted(cum, cum[s] + budget, side="right")) - 1
        bounds.append(max(e, s + 1))
    return [(bounds[k], bounds[k + 1]) for k in range(len(bounds) - 1)]


def align_device_pairs(dp: DeviceWfaPairs, max_distance: int = 4096, stream: Optional[torch.cuda.Stream] = None,
                       traceback: bool = True, history_budget: int = HISTORY_BUDGET, workspace=None) -> WfaResult:
    """Pairs already on the device in, host wavefront alignments out (on
    ``stream``, default the current one; ``workspace``: a callable giving a
    device uint8 tensor of at least the bytes asked, default the shared
    grow-only workspace)."""
    if dp.n == 0:
        z = np.zeros(0, np.int32)
        return WfaResult(z, np.zeros((0, 4), np.int32), np.zeros(0, np.uint32), np.zeros(0, np.int64), z)
    stream = stream or torch.cuda.current_stream(dp.device)
    sp = int(stream.cuda_stream)
    with torch.cuda.stream(stream):
        return _align_device(dp, max_distance, stream, sp, traceback, history_budget, workspace)


def _align_device(dp, max_distance, stream, sp, traceback, history_budget, workspace) -> WfaResult:
    dist_d = wfa_distances(dp, max_distance, stream, workspace=workspace)
    h_dist = dist_d.to("cpu", non_blocking=True)
    stream.synchronize()
    h_dist = h_dist.numpy().copy()
    if not traceback:
        return WfaResult(h_dist)
    counts = np.zeros((dp.n, 4), np.int32)
    cstart = np.zeros(dp.n, np.int64)
    clen = np.full(dp.n, -1, np.int32)
    words_all: list = []
    base = 0
    # chunks whose histories fit the budget (a pair above it alone)
    hist = np.where((h_dist >= 0) & (dp.h_qlen > 0) & (dp.h_tlen > 0),
                    (h_dist.astype(np.int64) + 1) ** 2, 0)
    chunks = history_chunks(hist, history_budget)
    for c0, c1 in chunks:
        idx = np.arange(c0, c1, dtype=np.int64)
        if len(chunks) == 1:
            sub, d_sub, h_d = dp, dist_d, h_dist
        else:
            sub, d_sub, h_d = _sub_batch(dp, dist_d, h_dist, idx)
        out = _run_align(sub, d_sub, h_d, sp, workspace)
        host = {k: v.to("cpu", non_blocking=True) for k, v in out.items() if k != "cigar"}
        stream.synchronize()
        if int(host["err"][0]) & _native.GMF_SWF_CAPACITY:
            raise RuntimeError("gmf_wfa_align: CIGAR output capacity exhausted")
        if int(host["err"][0]) & _native.GMF_SWF_WORKSPACE:
            raise RuntimeError("gmf_wfa_align: history workspace exhausted")
        if int(host["err"][0]) & _native.GMF_SWF_INTERNAL:
            raise RuntimeError("gmf_wfa_align: a distance does not belong to its pair")
        used = int(host["used"][0])
        words = np.zeros(0, np.uint32)
        if used:
            hw = out["cigar"][:used].to("cpu", non_blocking=True)
            stream.synchronize()
            words = hw.numpy().view(np.uint32).copy()
        counts[idx] = host["counts"].numpy()
        cstart[idx] = host["cstart"].numpy() + base
        clen[idx] = host["clen"].numpy()
        words_all.append(words)
        base += used
    words = np.concatenate(words_all) if words_all else np.zeros(0, np.uint32)
    return WfaResult(h_dist, counts, words, cstart, clen)


def wfa_distance(query: torch.Tensor, target: torch.Tensor, query_len: torch.Tensor, target_len: torch.Tensor,
                 max_distance: int) -> torch.Tensor:
    """Batched unit-cost WFA distance of padded ``(B, M)`` / ``(B, N)`` code
    tensors (cuda_kernels.py L569-600); ``-1`` means the bound was exceeded.
    Returns int32 on the query's device."""
    dev = require_cuda(query.device if query.is_cuda else None)
    q = query.detach().to(device=dev, dtype=torch.int8)
    t = target.detach().to(device=dev, dtype=torch.int8)
    ql = torch.as_tensor(query_len).to(dev).long().reshape(-1)
    tl = torch.as_tensor(target_len).to(dev).long().reshape(-1)
    B = q.shape[0]
    qmask = torch.arange(q.shape[1], device=dev)[None, :] < ql[:, None]
    tmask = torch.arange(t.shape[1], device=dev)[None, :] < tl[:, None]
    h_ql = torch.minimum(ql, torch.tensor(q.shape[1], device=dev)).to("cpu").numpy().astype(np.int32)
    h_tl = torch.minimum(tl, torch.tensor(t.shape[1], device=dev)).to("cpu").numpy().astype(np.int32)
    qo = np.zeros(B + 1, np.int64)
    np.cumsum(h_ql, out=qo[1:])
    to = np.zeros(B + 1, np.int64)
    np.cumsum(h_tl, out=to[1:])
    qf = q[qmask] if qo[-1] else torch.zeros(1, dtype=torch.int8, device=dev)
    tf = t[tmask] if to[-1] else torch.zeros(1, dtype=torch.int8, device=dev)
    dp = DeviceWfaPairs(B, qf.contiguous(), to_device(qo, dev), tf.contiguous(), to_device(to, dev), h_ql, h_tl, dev)
    return wfa_distances(dp, max_distance)


class WavefrontAligner:
    """Global wavefront alignment under unit edit costs (extension.py
    L308-463), on the device."""

    def __init__(self, cfg: Optional[ExtensionConfig] = None, device=None):
        self.cfg = cfg or ExtensionConfig()
        self.device = require_cuda(device)

    def align(self, query: np.ndarray, target: np.ndarray) -> tuple:
        """``(edit_distance, cigar)``; raises RuntimeError when the distance
        exceeds ``cfg.wfa_max_distance`` (the caller's cue to fall back to
        banded DP)."""
        r = align_wfa_pairs([np.asarray(query)], [np.asarray(target)], self.cfg.wfa_max_distance,
                            device=self.device)
        if int(r.distance[0]) < 0:
            raise RuntimeError(f"WFA exceeded wfa_max_distance={self.cfg.wfa_max_distance}")
        return int(r.distance[0]), r.cigar(0)

    def align_batch(self, queries: Sequence[np.ndarray], targets: Sequence[np.ndarray]) -> list:
        """``align`` for many pairs in one pass; ``None`` for a pair beyond
        the bound."""
        r = align_wfa_pairs(queries, targets, self.cfg.wfa_max_distance, device=self.device)
        return [(int(r.distance[b]), r.cigar(b)) if r.distance[b] >= 0 else None for b in range(len(r))]
