"""Stage 3 -- banded affine-gap Smith-Waterman extension with CIGAR traceback.

Drop-in for the reference's extension stage:

* :func:`banded_sw` -- ``accel/cuda_kernels.py`` L504-566 (score + ends of
  padded ``(B, M)`` / ``(B, N)`` code tensors);
* :func:`banded_affine_sw_batch` + :func:`traceback_banded` --
  ``alignment/extension.py`` L78-302 (the traceback runs on the GPU inside
  the same launch; ``return_matrices=True`` requests it, no matrices are
  materialised);
* :class:`ExtensionEngine` -- ``alignment/extension.py`` L469-641
  (``_window`` + ``extend_chains``), the object the pipeline holds as
  ``pipeline.extender``.

Semantics are the reference's.  At the primitive level each pair carries its
own band (the reference's scalar band is the special case), and x-drop stops
a batch's row loop only after every member dropped: ``banded_affine_sw_batch``
treats its whole batch as one x-drop group, ``ExtensionEngine`` one read's
chains (which also share the widest band of the read, extension.py L534), and
``align_pairs`` takes the groups a caller gives (``PairSet.xdrop_group_off``;
none = each pair alone).  Scores are integers
(float32 in the reference, exact below 2**24) and scoring parameters must be
integral.  Every computation runs in the gmf CUDA library; without a GPU the
calls raise.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np
import torch

from . import _native
from .config import ExtensionConfig
from .device import WORKSPACE, bind, np_ptr, ptr, require_cuda, stream_handle, to_device
from .synth import PairSet, encode_bases, reverse_complement
from .types import AnchorSet, Chain, ExtensionResult, add_soft_clips, decode_words

N_CODE = 5


def _int_param(name: str, v) -> int:
    f = float(v)
    if not f.is_integer():
        raise ValueError(f"{name}={v!r}: the B200 kernels score in exact integers; "
                         "use an integral value")
    return int(f)


def sw_params(match_score=2.0, mismatch_penalty=4.0, gap_open=6.0, gap_extend=2.0,
              x_drop=0.0) -> _native.GmfSwParams:
    """Integer scoring parameters.  ``x_drop > 0`` enables x-drop with the
    reference's ``(max row max) - row max > x_drop`` test; for integral scores
    that test equals ``> floor(x_drop)``."""
    xd = float(x_drop)
    return _native.GmfSwParams(
        _int_param("match_score", match_score),
        _int_param("mismatch_penalty", mismatch_penalty),
        _int_param("gap_open", gap_open),
        _int_param("gap_extend", gap_extend),
        int(math.floor(xd)) if xd > 0 else 0,
    )


def params_from_config(cfg: ExtensionConfig, x_drop: Optional[float] = None) -> _native.GmfSwParams:
    return sw_params(cfg.match_score, cfg.mismatch_penalty, cfg.gap_open, cfg.gap_extend,
                     cfg.x_drop if x_drop is None else x_drop)


# --------------------------------------------------------------------------- #
# Device batches
# --------------------------------------------------------------------------- #
@dataclass
class DevicePairs:
    """A pair batch resident on the device (CSR layout)."""

    n: int
    query: torch.Tensor
    query_off: torch.Tensor
    target: torch.Tensor
    target_off: torch.Tensor
    half_band: torch.Tensor
    band_offset: torch.Tensor
    order: Optional[torch.Tensor]
    max_half_band: int
    # host copies used to size workspace / outputs
    h_qlen: np.ndarray
    h_tlen: np.ndarray
    h_hb: np.ndarray
    device: torch.device
    xdrop_group_off: Optional[torch.Tensor] = None  # n_groups+1 offsets, or None
    n_groups: int = 0

    @property
    def h2d_bytes(self) -> int:
        ts = (self.query, self.query_off, self.target, self.target_off, self.half_band,
              self.band_offset) + ((self.order,) if self.order is not None else ())
        return int(sum(t.numel() * t.element_size() for t in ts))


def longest_first(qlen: np.ndarray, hb: np.ndarray) -> np.ndarray:
    """Processing order by decreasing DP area (longest-processing-time first);
    it changes scheduling only, never results."""
    area = qlen.astype(np.int64) * (2 * hb.astype(np.int64) + 1)
    return np.argsort(-area, kind="stable").astype(np.int32)


def upload_pairs(pairs: PairSet, device=None, order: Optional[np.ndarray] = None,
                 lpt: bool = True) -> DevicePairs:
    dev = require_cuda(device)
    qlen = np.diff(pairs.query_off).astype(np.int32)
    tlen = np.diff(pairs.target_off).astype(np.int32)
    hb = np.asarray(pairs.half_band, dtype=np.int32)
    if len(hb) and (hb.min() < 0 or hb.max() > _native.MAX_HALF_BAND):
        raise ValueError(f"half_band must be within [0, {_native.MAX_HALF_BAND}]")
    if order is None and lpt and len(hb):
        order = longest_first(qlen, hb)
    q = pairs.query if len(pairs.query) else np.zeros(1, np.int8)
    t = pairs.target if len(pairs.target) else np.zeros(1, np.int8)
    goff = None
    if pairs.xdrop_group_off is not None:
        goff = np.asarray(pairs.xdrop_group_off, np.int32)
        if goff.ndim != 1 or len(goff) < 1 or goff[0] != 0 or goff[-1] != len(hb) or np.any(np.diff(goff) < 0):
            raise ValueError("xdrop_group_off must rise from 0 to the number of pairs")
    return DevicePairs(
        n=len(hb),
        query=to_device(q.astype(np.int8, copy=False), dev),
        query_off=to_device(pairs.query_off.astype(np.int64, copy=False), dev),
        target=to_device(t.astype(np.int8, copy=False), dev),
        target_off=to_device(pairs.target_off.astype(np.int64, copy=False), dev),
        half_band=to_device(hb, dev),
        band_offset=to_device(np.asarray(pairs.band_offset, dtype=np.int32), dev),
        order=None if order is None else to_device(np.asarray(order, dtype=np.int32), dev),
        max_half_band=int(hb.max()) if len(hb) else 0,
        h_qlen=qlen, h_tlen=tlen, h_hb=hb, device=dev,
        xdrop_group_off=None if goff is None else to_device(goff, dev),
        n_groups=0 if goff is None else len(goff) - 1)


@dataclass
class SWOutputs:
    """Device-side results of one gmf_banded_sw call."""

    score: torch.Tensor
    query_end: torch.Tensor
    target_end: torch.Tensor
    query_start: Optional[torch.Tensor]
    target_start: Optional[torch.Tensor]
    op_counts: Optional[torch.Tensor]
    cigar: Optional[torch.Tensor]
    cigar_start: Optional[torch.Tensor]
    cigar_len: Optional[torch.Tensor]
    cigar_used: torch.Tensor
    error_flags: torch.Tensor

    @staticmethod
    def allocate(dp: DevicePairs, traceback: bool) -> "SWOutputs":
        dev, n = dp.device, max(dp.n, 1)
        i32 = dict(dtype=torch.int32, device=dev)
        cap = int(dp.h_qlen.astype(np.int64).sum() + dp.h_tlen.astype(np.int64).sum() + dp.n) if traceback else 0
        return SWOutputs(
            score=torch.empty(n, **i32), query_end=torch.empty(n, **i32),
            target_end=torch.empty(n, **i32),
            query_start=torch.empty(n, **i32) if traceback else None,
            target_start=torch.empty(n, **i32) if traceback else None,
            op_counts=torch.empty((n, 4), **i32) if traceback else None,
            cigar=torch.empty(max(cap, 1), dtype=torch.int32, device=dev) if traceback else None,
            cigar_start=torch.empty(n, dtype=torch.int64, device=dev) if traceback else None,
            cigar_len=torch.empty(n, **i32) if traceback else None,
            cigar_used=torch.zeros(1, dtype=torch.int64, device=dev),
            error_flags=torch.zeros(1, **i32))


def workspace_bytes(dp: DevicePairs, traceback: bool) -> int:
    return int(_native.lib().gmf_banded_sw_workspace_bytes(
        dp.n, np_ptr(dp.h_qlen), np_ptr(dp.h_tlen), np_ptr(dp.h_hb), 1 if traceback else 0))


FORMS = ("batched", "plain")


def launch_banded_sw(dp: DevicePairs, params: _native.GmfSwParams, traceback: bool = True,
                     out: Optional[SWOutputs] = None, workspace: Optional[torch.Tensor] = None,
                     stream: Optional[torch.cuda.Stream] = None, form: str = "batched") -> SWOutputs:
    """Enqueue the banded SW on ``stream`` (default: the current stream).

    ``form="batched"`` (default) is gmf_banded_sw: device classifier, int16x2
    cells where scores fit, persistent work-queue kernels.  ``form="plain"``
    is gmf_banded_sw_plain: one warp per pair, int32 cells.  Both give
    identical results."""
    if form not in FORMS:
        raise ValueError(f"form must be one of {FORMS}")
    out = out or SWOutputs.allocate(dp, traceback)
    need = workspace_bytes(dp, traceback)
    ws = workspace if workspace is not None and workspace.numel() >= need else WORKSPACE.get(dp.device, need)
    sp = stream_handle(stream, dp.device)
    bind(dp.device, sp)
    pairs = _native.GmfPairs(dp.n, ptr(dp.query), ptr(dp.query_off), ptr(dp.target), ptr(dp.target_off),
                             ptr(dp.half_band), ptr(dp.band_offset), ptr(dp.order), dp.max_half_band,
                             ptr(dp.xdrop_group_off), dp.n_groups)
    res = _native.GmfSwResults(
        ptr(out.score), ptr(out.query_end), ptr(out.target_end), ptr(out.query_start),
        ptr(out.target_start), ptr(out.op_counts), ptr(out.cigar),
        out.cigar.numel() if out.cigar is not None else 0, ptr(out.cigar_start), ptr(out.cigar_len),
        ptr(out.cigar_used), ptr(out.error_flags))
    fn = _native.lib().gmf_banded_sw if form == "batched" else _native.lib().gmf_banded_sw_plain
    st = fn(ctypes.byref(pairs), ctypes.byref(params), ctypes.byref(res),
            ctypes.c_void_p(ws.data_ptr()), ws.numel(), ctypes.c_void_p(sp))
    _native.check("gmf_banded_sw" if form == "batched" else "gmf_banded_sw_plain", st)
    return out


@dataclass
class SWResult:
    """Host copy of a batch's alignments."""

    score: np.ndarray
    query_end: np.ndarray
    target_end: np.ndarray
    query_start: Optional[np.ndarray] = None
    target_start: Optional[np.ndarray] = None
    op_counts: Optional[np.ndarray] = None
    cigar_words: Optional[np.ndarray] = None
    cigar_start: Optional[np.ndarray] = None
    cigar_len: Optional[np.ndarray] = None
    error_flags: int = 0
    d2h_bytes: int = 0

    def __len__(self) -> int:
        return len(self.score)

    def cigar(self, b: int) -> list:
        s, n = int(self.cigar_start[b]), int(self.cigar_len[b])
        if n < 0:
            raise RuntimeError(f"pair {b}: CIGAR did not fit its output buffer")
        dec = self.__dict__.get("_decoded")
        if dec is None:  # every word of the batch decoded once
            dec = self.__dict__["_decoded"] = decode_words(self.cigar_words)
        return list(zip(dec[0][s: s + n], dec[1][s: s + n]))


def fetch(out: SWOutputs, n: int) -> SWResult:
    """Copy a batch's results to the host (synchronises the device)."""
    small = [out.score, out.query_end, out.target_end, out.cigar_used, out.error_flags]
    if out.cigar is not None:
        small += [out.query_start, out.target_start, out.op_counts, out.cigar_start, out.cigar_len]
    host = [t.to("cpu", non_blocking=True) for t in small]
    torch.cuda.current_stream(out.score.device).synchronize()
    nbytes = sum(t.numel() * t.element_size() for t in host)
    r = SWResult(host[0].numpy()[:n], host[1].numpy()[:n], host[2].numpy()[:n],
                 error_flags=int(host[4][0]))
    if out.cigar is not None:
        used = int(host[3][0])
        words = out.cigar[:used].to("cpu").numpy().view(np.uint32) if used else np.zeros(0, np.uint32)
        nbytes += used * 4
        r.query_start = host[5].numpy()[:n]
        r.target_start = host[6].numpy()[:n]
        r.op_counts = host[7].numpy()[:n]
        r.cigar_start = host[8].numpy()[:n]
        r.cigar_len = host[9].numpy()[:n]
        r.cigar_words = words
    r.d2h_bytes = nbytes
    if r.error_flags & _native.GMF_SWF_WORKSPACE:
        raise RuntimeError("gmf_banded_sw: traceback workspace exhausted")
    if r.error_flags & _native.GMF_SWF_CAPACITY:
        raise RuntimeError("gmf_banded_sw: CIGAR output capacity exhausted")
    if r.error_flags & _native.GMF_SWF_TIMEOUT:
        raise RuntimeError("gmf_banded_sw: a bounded wait between cooperating warps gave up")
    return r


def align_pairs(pairs: PairSet, params: Optional[_native.GmfSwParams] = None, traceback: bool = True,
                device=None, order: Optional[np.ndarray] = None, form: str = "batched") -> SWResult:
    """Host pairs in, host alignments out (upload, one launch, download)."""
    params = params or sw_params()
    dp = upload_pairs(pairs, device, order=order)
    out = launch_banded_sw(dp, params, traceback, form=form)
    return fetch(out, dp.n)


# --------------------------------------------------------------------------- #
# Reference-shaped primitives
# --------------------------------------------------------------------------- #
def _padded_to_pairs(query: torch.Tensor, target: torch.Tensor, query_len, target_len,
                     half_band, band_offset) -> PairSet:
    q = query.detach().to("cpu").numpy().astype(np.int8)
    t = target.detach().to("cpu").numpy().astype(np.int8)
    ql = np.asarray(torch.as_tensor(query_len).to("cpu"), dtype=np.int64).reshape(-1)
    tl = np.asarray(torch.as_tensor(target_len).to("cpu"), dtype=np.int64).reshape(-1)
    B = q.shape[0]
    hb = np.broadcast_to(np.asarray(torch.as_tensor(half_band).to("cpu"), dtype=np.int32), (B,))
    off = (np.zeros(B, np.int32) if band_offset is None else
           np.broadcast_to(np.asarray(torch.as_tensor(band_offset).to("cpu"), dtype=np.int32), (B,)))
    qs = [q[b, : min(int(ql[b]), q.shape[1])] for b in range(B)]
    ts = [t[b, : min(int(tl[b]), t.shape[1])] for b in range(B)]
    return PairSet.from_lists(qs, ts, hb, off)


def banded_sw(query: torch.Tensor, target: torch.Tensor, query_len: torch.Tensor,
              target_len: torch.Tensor, half_band: int, match_score: float,
              mismatch_penalty: float, gap_open: float, gap_extend: float,
              band_offset: Optional[torch.Tensor] = None):
    """Batched banded affine SW scores and end points (cuda_kernels.py
    L504-566): ``(score float32, query_end int64, target_end int64)`` on the
    query's device.  No x-drop, like the reference kernel; unlike it, the
    band is not limited to 1024 and ties follow the torch reference."""
    dev = require_cuda(query.device if query.is_cuda else None)
    ps = _padded_to_pairs(query, target, query_len, target_len, half_band, band_offset)
    dp = upload_pairs(ps, dev)
    out = launch_banded_sw(dp, sw_params(match_score, mismatch_penalty, gap_open, gap_extend, 0), False)
    return out.score[: dp.n].float(), out.query_end[: dp.n].long(), out.target_end[: dp.n].long()


@dataclass
class BandedSWResult:
    """Counterpart of the reference's BandedDPResult (extension.py L59-75)."""

    score: torch.Tensor
    query_end: torch.Tensor
    target_end: torch.Tensor
    half_band: object
    band_offset: torch.Tensor
    alignments: Optional[SWResult] = None


def banded_affine_sw_batch(query: torch.Tensor, target: torch.Tensor, query_len, target_len,
                           cfg: ExtensionConfig, half_band=None, band_offset=None,
                           return_matrices: bool = False) -> BandedSWResult:
    """extension.py L78-204 on the GPU.  ``half_band`` may be an int (the
    reference) or a per-pair tensor; ``return_matrices=True`` runs the
    device traceback so :func:`traceback_banded` can report CIGARs."""
    dev = require_cuda(query.device if query.is_cuda else None)
    hb = cfg.half_band if half_band is None else half_band
    ps = _padded_to_pairs(query, target, query_len, target_len, hb, band_offset)
    ps.xdrop_group_off = np.array([0, len(ps)], np.int32)  # one row loop for the whole batch
    dp = upload_pairs(ps, dev)
    res = fetch(launch_banded_sw(dp, params_from_config(cfg), bool(return_matrices)), dp.n)
    return BandedSWResult(
        score=torch.as_tensor(res.score.astype(np.float32)),
        query_end=torch.as_tensor(res.query_end.astype(np.int64)),
        target_end=torch.as_tensor(res.target_end.astype(np.int64)),
        half_band=hb, band_offset=torch.as_tensor(ps.band_offset.astype(np.int64)),
        alignments=res if return_matrices else None)


def _result(res: SWResult, b: int) -> ExtensionResult:
    c = res.op_counts[b]
    return ExtensionResult(
        score=float(res.score[b]), cigar=res.cigar(b),
        read_start=int(res.query_start[b]), read_end=int(res.query_end[b]),
        ref_start=int(res.target_start[b]), ref_end=int(res.target_end[b]),
        n_match=int(c[0]), n_mismatch=int(c[1]), n_insertion=int(c[2]), n_deletion=int(c[3]))


def traceback_banded(result: BandedSWResult, index: int, query=None, target=None,
                     cfg: Optional[ExtensionConfig] = None, tolerance: float = 1e-3) -> ExtensionResult:
    """extension.py L207-302: the alignment of batch element ``index`` (traced
    on the device by :func:`banded_affine_sw_batch`)."""
    if result.alignments is None:
        raise ValueError("traceback needs banded_affine_sw_batch(return_matrices=True)")
    return _result(result.alignments, index)


# --------------------------------------------------------------------------- #
# Stage entry point
# --------------------------------------------------------------------------- #
class _RefCodes:
    """Encoded reference, cached by string identity (re-encoding a 10 Mb
    reference per call would dominate small calls)."""

    def __init__(self):
        self._key = None
        self._codes = None

    def get(self, ref_seq: str) -> np.ndarray:
        key = (id(ref_seq), len(ref_seq))
        if self._key != key:
            self._codes = encode_bases(ref_seq)
            self._key = key
        return self._codes


def wfa_extension_result(cigar: list, start: int, window_len: int, read_len: int,
                         cfg: ExtensionConfig) -> ExtensionResult:
    """A WFA-mode chain's result (extension.py L702-730): the whole read
    against reference [start, start + window_len), op tallies from the CIGAR,
    and the affine score recomputed from it in the reference's order of
    operations."""
    counts = {op: 0 for op in ("=", "X", "I", "D")}
    for op, n in cigar:
        counts[op] = counts.get(op, 0) + n
    gap_cost = sum(cfg.gap_open + max(n - 1, 0) * cfg.gap_extend for op, n in cigar if op in ("I", "D"))
    score = counts["="] * cfg.match_score - counts["X"] * cfg.mismatch_penalty - gap_cost
    return ExtensionResult(score=float(score), cigar=cigar, read_start=0, read_end=read_len, ref_start=start,
                           ref_end=start + window_len, n_match=counts["="], n_mismatch=counts["X"],
                           n_insertion=counts["I"], n_deletion=counts["D"])


class ExtensionEngine:
    """Stage 3 entry point (extension.py L469-641): chains -> alignments."""

    def __init__(self, cfg: Optional[ExtensionConfig] = None, device=None, backend: str = "b200"):
        self.cfg = cfg or ExtensionConfig()
        self.device = require_cuda(device)
        self.backend = backend
        self._ref = _RefCodes()

    def _window(self, chain: Chain, anchors: AnchorSet, read_len: int, ref_len: int):
        """DP window and band of one chain (extension.py L489-509)."""
        diagonal = chain.ref_start - chain.read_start
        start = max(0, diagonal - self.cfg.flank)
        end = min(ref_len, diagonal + read_len + self.cfg.flank)
        if end - start > self.cfg.max_window:
            end = start + self.cfg.max_window
        idx = chain.anchor_idx
        spread = 0
        if len(idx):
            diagonals = anchors.ref_pos[idx].astype(np.int64) - anchors.read_pos[idx].astype(np.int64)
            spread = int(diagonals.max() - diagonals.min())
        half_band = min(self.cfg.half_band + spread, self.cfg.max_half_band)
        return start, end, half_band

    def _pairs(self, items):
        """items: (forward codes, chains, anchors, ref codes) per read ->
        PairSet + per-pair (read index, window start, read_len)."""
        qs, ts, hbs, offs, meta = [], [], [], [], []
        groups = [0]
        for r, (forward, chains, anchors, ref_codes) in enumerate(items):
            if not chains:
                continue
            groups.append(groups[-1] + len(chains))
            reverse = reverse_complement(forward)
            read_len, ref_len = len(forward), len(ref_codes)
            windows = [self._window(chain, anchors, read_len, ref_len) for chain in chains]
            # one band for every chain of the read: the widest (extension.py L534)
            hb = max(w[2] for w in windows)
            for chain, (start, end, _) in zip(chains, windows):
                codes = forward if chain.strand > 0 else reverse
                qs.append(codes)
                ts.append(ref_codes[start:end])
                hbs.append(hb)
                offs.append((chain.ref_start - chain.read_start) - start)
                meta.append((r, start, read_len))
        ps = PairSet.from_lists(qs, ts, np.array(hbs, np.int32), np.array(offs, np.int32))
        # the chains of a read share the x-drop stop, as in the reference's batch (extension.py L190-193)
        ps.xdrop_group_off = np.array(groups, np.int32)
        return ps, meta

    def _finish(self, res: SWResult, meta) -> list:
        out = []
        for b, (_, start, read_len) in enumerate(meta):
            ext = _result(res, b)
            ext.ref_start += start
            ext.ref_end += start
            ext.cigar = add_soft_clips(ext.cigar, ext.read_start, read_len - ext.read_end)
            out.append(ext)
        return out

    def extend_chains(self, read_seq: str, chains: Sequence[Chain], anchors: AnchorSet,
                      ref_seq: str) -> list:
        """Extend every chain of one read; one result per chain."""
        return self.extend_batch([read_seq], [chains], [anchors], ref_seq)[0]

    def extend_batch(self, reads: Sequence[str], chains_per_read, anchor_sets, ref_seq: str) -> list:
        """``extend_chains`` for many reads in one device launch."""
        ref_codes = self._ref.get(ref_seq)
        items = [(encode_bases(r), c, a, ref_codes) for r, c, a in zip(reads, chains_per_read, anchor_sets)]
        if self.cfg.algorithm == "wfa":
            return self._extend_wfa(items)
        return self._extend_sw(items)

    def _extend_sw(self, items) -> list:
        ps, meta = self._pairs(items)
        results: list = [[] for _ in items]
        if len(ps) == 0:
            return results
        res = align_pairs(ps, params_from_config(self.cfg), traceback=True, device=self.device)
        for (r, _, _), ext in zip(meta, self._finish(res, meta)):
            results[r].append(ext)
        return results

    @staticmethod
    def _wfa_windows(items):
        """WFA-mode pairs (extension.py L654-663): the read (reverse
        complemented for strand -1) against the reference from the chain's
        read-zero diagonal, as long as the read plus the chain's net indel.
        Returns queries, targets and (read index, chain index, window start,
        read length) per pair."""
        qs, ts, meta = [], [], []
        for r, (forward, chains, anchors, ref_codes) in enumerate(items):
            if not chains:
                continue
            reverse = reverse_complement(forward)
            read_len, ref_len = len(forward), len(ref_codes)
            for ci, chain in enumerate(chains):
                codes = forward if chain.strand > 0 else reverse
                start = int(np.clip(chain.ref_start - chain.read_start, 0, max(ref_len - 1, 0)))
                net_indel = chain.ref_span - chain.read_span
                end = min(ref_len, start + max(1, read_len + net_indel))
                qs.append(codes)
                ts.append(ref_codes[start:end])
                meta.append((r, ci, start, read_len))
        return qs, ts, meta

    def _extend_wfa(self, items) -> list:
        """WFA mode (extension.py L643-730): each chain is aligned end to end
        against the reference stretch its read-zero diagonal and net indel
        imply; a chain beyond ``wfa_max_distance`` falls back to banded SW of
        that chain alone.  The score is recomputed from the CIGAR with the
        affine parameters."""
        from .wfa import align_wfa_pairs

        cfg = self.cfg
        qs, ts, meta = self._wfa_windows(items)
        results: list = [[None] * len(it[1]) for it in items]
        if not meta:
            return [[] for _ in items]
        res = align_wfa_pairs(qs, ts, cfg.wfa_max_distance, device=self.device)
        fallback = []
        for b, (r, ci, start, read_len) in enumerate(meta):
            if res.distance[b] < 0:
                forward, chains, anchors, ref_codes = items[r]
                fallback.append(((r, ci), (forward, [chains[ci]], anchors, ref_codes)))
                continue
            results[r][ci] = wfa_extension_result(res.cigar(b), start, len(ts[b]), read_len, cfg)
        if fallback:  # banded SW, one chain per call as the reference re-enters extend_chains
            for (r, ci), ext in zip((k for k, _ in fallback), self._extend_sw([it for _, it in fallback])):
                results[r][ci] = ext[0]
        return results
