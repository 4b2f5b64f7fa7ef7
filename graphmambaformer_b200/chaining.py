"""Stage 2 -- minimap2-style anchor chaining on the B200.

Drop-in for the reference's chaining stage:

* :func:`chain_dp` -- ``accel/cuda_kernels.py`` L440-501 (padded ``(B, A, 3)``
  anchors -> ``(f, predecessor)``), but float64 and bit-exact;
* :func:`chain_dp_rows` -- ``alignment/chaining.py`` L129-180
  (``chain_dp_numpy`` signature, computed on the GPU);
* :class:`AffineChainer` -- ``alignment/chaining.py`` L292-745: ``chain`` and
  ``chain_batch`` run strand split, sort, DP, chain peeling and selection in
  the gmf CUDA library; ``pipeline.chainer`` can be replaced by it.

Scores are float64 like ``chain_dp_numpy``: the device evaluates
``((f[j] + min(min(dq, dr), w_i)) - pen[gap]) [+ bonus]`` with IEEE adds in
that order and takes the gap penalty from a table that numpy computes with
the reference's own expression, so scores, predecessors and chains are
bit-identical.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import _native
from .config import ChainingConfig
from .device import WORKSPACE, bind, ptr, require_cuda, stream_handle, to_device
from .types import AnchorSet, Chain

NO_PREDECESSOR = -1


def penalty_lut(max_gap: int, gap_open: float, gap_extend: float, log_coeff: float) -> np.ndarray:
    """The reference's ``_penalty`` (chaining.py L120-126) for every gap
    ``0..max_gap``, evaluated by numpy with the same expression, so entry
    ``g`` is bit-identical to the reference's penalty of a gap of ``g``."""
    gap = np.arange(int(max_gap) + 1, dtype=np.int64)
    return np.where(gap > 0, gap_open + gap_extend * gap + log_coeff * np.log2(gap + 1.0), 0.0)


class _LutCache:
    def __init__(self):
        self._c: dict = {}

    def get(self, device: torch.device, max_gap, gap_open, gap_extend, log_coeff) -> torch.Tensor:
        key = (device.index, int(max_gap), float(gap_open), float(gap_extend), float(log_coeff))
        t = self._c.get(key)
        if t is None:
            t = torch.from_numpy(penalty_lut(max_gap, gap_open, gap_extend, log_coeff)).to(device)
            self._c[key] = t
        return t


LUTS = _LutCache()


def chain_params(cfg: ChainingConfig) -> _native.GmfChainParams:
    if int(cfg.max_lookback) > _native.MAX_LOOKBACK:
        raise ValueError(f"max_lookback > {_native.MAX_LOOKBACK} is not supported")
    if not 1 <= int(cfg.max_chains) <= 64:
        raise ValueError("max_chains must be within [1, 64]")
    return _native.GmfChainParams(
        max(1, int(cfg.max_lookback)), int(cfg.max_gap), int(cfg.min_chain_anchors),
        int(cfg.max_chains), float(cfg.min_chain_score), float(cfg.secondary_overlap),
        float(cfg.secondary_score_ratio))


# --------------------------------------------------------------------------- #
# Batched anchors
# --------------------------------------------------------------------------- #
@dataclass
class AnchorCSR:
    """Anchors of many reads, concatenated (per-read original order)."""

    read_off: np.ndarray  # int64 (R+1,)
    read_pos: np.ndarray  # int32
    ref_pos: np.ndarray
    length: np.ndarray
    strand: np.ndarray  # int8

    def __len__(self) -> int:
        return len(self.read_off) - 1

    @staticmethod
    def from_sets(anchor_sets: Sequence) -> "AnchorCSR":
        counts = np.array([len(a) for a in anchor_sets], dtype=np.int64)
        off = np.zeros(len(anchor_sets) + 1, dtype=np.int64)
        np.cumsum(counts, out=off[1:])

        def cat(name, dt):
            if off[-1] == 0:
                return np.zeros(0, dt)
            return np.concatenate([np.asarray(getattr(a, name)) for a in anchor_sets]).astype(dt)

        return AnchorCSR(off, cat("read_pos", np.int32), cat("ref_pos", np.int32),
                         cat("length", np.int32), cat("strand", np.int8))

    @staticmethod
    def of(batch) -> "AnchorCSR":
        if isinstance(batch, AnchorCSR):
            return batch
        return AnchorCSR(np.asarray(batch.read_off, np.int64), np.asarray(batch.read_pos, np.int32),
                         np.asarray(batch.ref_pos, np.int32), np.asarray(batch.length, np.int32),
                         np.asarray(batch.strand, np.int8))


@dataclass
class DeviceAnchors:
    n_reads: int
    n_anchors: int
    read_off: torch.Tensor
    read_pos: torch.Tensor
    ref_pos: torch.Tensor
    length: torch.Tensor
    strand: torch.Tensor
    device: torch.device

    @property
    def h2d_bytes(self) -> int:
        ts = (self.read_off, self.read_pos, self.ref_pos, self.length, self.strand)
        return int(sum(t.numel() * t.element_size() for t in ts))


def upload_anchors(batch, device=None) -> DeviceAnchors:
    a = AnchorCSR.of(batch)
    dev = require_cuda(device)
    counts = np.diff(a.read_off)
    if len(counts) and counts.max() > _native.MAX_READ_ANCHORS:
        raise ValueError(f"a read has more than {_native.MAX_READ_ANCHORS} anchors")
    pad = lambda x, dt: x if len(x) else np.zeros(1, dt)  # noqa: E731
    return DeviceAnchors(len(a), int(a.read_off[-1]), to_device(a.read_off, dev),
                         to_device(pad(a.read_pos, np.int32), dev), to_device(pad(a.ref_pos, np.int32), dev),
                         to_device(pad(a.length, np.int32), dev), to_device(pad(a.strand, np.int8), dev), dev)


@dataclass
class ChainOutputs:
    n_chains: torch.Tensor
    score: torch.Tensor
    strand: torch.Tensor
    span: torch.Tensor
    is_primary: torch.Tensor
    n_members: torch.Tensor
    members: torch.Tensor
    max_chains: int

    @staticmethod
    def allocate(da: DeviceAnchors, max_chains: int) -> "ChainOutputs":
        dev, R, A = da.device, max(da.n_reads, 1), max(da.n_anchors, 1)
        i32 = dict(dtype=torch.int32, device=dev)
        return ChainOutputs(torch.empty(R, **i32), torch.empty(R * max_chains, dtype=torch.float64, device=dev),
                            torch.empty(R * max_chains, **i32), torch.empty(R * max_chains * 4, **i32),
                            torch.empty(R * max_chains, **i32), torch.empty(R * max_chains, **i32),
                            torch.empty(A, **i32), max_chains)


def launch_chain_batch(da: DeviceAnchors, cfg: ChainingConfig, out: Optional[ChainOutputs] = None,
                       sorted_layout=None, sorted_weight: Optional[torch.Tensor] = None,
                       sorted_bonus: Optional[torch.Tensor] = None,
                       stream: Optional[torch.cuda.Stream] = None) -> ChainOutputs:
    cp = chain_params(cfg)
    out = out or ChainOutputs.allocate(da, cp.max_chains)
    lut = LUTS.get(da.device, cfg.max_gap, cfg.gap_open, cfg.gap_extend, cfg.log_coeff)
    need = int(_native.lib().gmf_chain_workspace_bytes(da.n_reads, da.n_anchors))
    ws = WORKSPACE.get(da.device, need)
    sp = stream_handle(stream, da.device)
    bind(da.device, sp)
    batch = _native.GmfAnchorBatch(da.n_reads, ptr(da.read_off), ptr(da.read_pos), ptr(da.ref_pos),
                                   ptr(da.length), ptr(da.strand))
    res = _native.GmfChainResults(ptr(out.n_chains), ptr(out.score), ptr(out.strand), ptr(out.span),
                                  ptr(out.is_primary), ptr(out.n_members), ptr(out.members))
    st = _native.lib().gmf_chain_batch(
        ctypes.byref(batch), ctypes.byref(cp), ctypes.c_void_p(lut.data_ptr()), lut.numel(),
        ctypes.byref(sorted_layout) if sorted_layout is not None else None,
        ptr(sorted_weight), ptr(sorted_bonus), ctypes.byref(res),
        ctypes.c_void_p(ws.data_ptr()), need, ctypes.c_void_p(sp))
    _native.check("gmf_chain_batch", st)
    return out


@dataclass
class ChainResult:
    """Host copy of a batch's chains."""

    read_off: np.ndarray
    n_chains: np.ndarray
    score: np.ndarray  # (R, max_chains)
    strand: np.ndarray
    span: np.ndarray  # (R, max_chains, 4)
    is_primary: np.ndarray
    n_members: np.ndarray
    members: np.ndarray  # (A,)
    d2h_bytes: int = 0

    def chains(self, r: int) -> list:
        out, pos = [], int(self.read_off[r])
        for k in range(int(self.n_chains[r])):
            m = int(self.n_members[r, k])
            sp = self.span[r, k]
            out.append(Chain(anchor_idx=self.members[pos: pos + m].astype(np.int64),
                             score=float(self.score[r, k]), strand=int(self.strand[r, k]),
                             read_start=int(sp[0]), read_end=int(sp[1]), ref_start=int(sp[2]),
                             ref_end=int(sp[3]), is_primary=bool(self.is_primary[r, k])))
            pos += m
        return out


def fetch_chains(out: ChainOutputs, read_off: np.ndarray) -> ChainResult:
    R = len(read_off) - 1
    mc = out.max_chains
    ts = [out.n_chains, out.score, out.strand, out.span, out.is_primary, out.n_members, out.members]
    host = [t.to("cpu", non_blocking=True) for t in ts]
    torch.cuda.current_stream(out.n_chains.device).synchronize()
    nbytes = sum(t.numel() * t.element_size() for t in host)
    h = [t.numpy() for t in host]
    return ChainResult(read_off, h[0][:R], h[1][: R * mc].reshape(R, mc), h[2][: R * mc].reshape(R, mc),
                       h[3][: R * mc * 4].reshape(R, mc, 4), h[4][: R * mc].reshape(R, mc),
                       h[5][: R * mc].reshape(R, mc), h[6], nbytes)


def chain_anchor_batch(batch, cfg: Optional[ChainingConfig] = None, device=None) -> ChainResult:
    """Host anchors in (CSR), host chains out: upload, chain, download."""
    cfg = cfg or ChainingConfig()
    a = AnchorCSR.of(batch)
    da = upload_anchors(a, device)
    return fetch_chains(launch_chain_batch(da, cfg), a.read_off)


# --------------------------------------------------------------------------- #
# DP primitives
# --------------------------------------------------------------------------- #
def _launch_chain_dp(row_off: torch.Tensor, read_end: torch.Tensor, ref_end: torch.Tensor,
                     weight: torch.Tensor, bonus: Optional[torch.Tensor], lookback: int, max_gap: int,
                     lut: torch.Tensor, f: torch.Tensor, parent: torch.Tensor, n_rows: int) -> None:
    dev = f.device
    sp = stream_handle(None, dev)
    bind(dev, sp)
    st = _native.lib().gmf_chain_dp(
        n_rows, ptr(row_off), ptr(read_end), ptr(ref_end), ptr(weight), ptr(bonus), int(lookback),
        int(max_gap), ptr(lut), lut.numel(), ptr(f), ptr(parent), ctypes.c_void_p(sp))
    _native.check("gmf_chain_dp", st)


def chain_dp_rows(read_end, ref_end, weight, cfg: ChainingConfig, bonus=None, device=None):
    """``chain_dp_numpy`` (chaining.py L129-180) on the GPU for one row of
    anchors sorted by reference end: ``(f float64, predecessor int64)``."""
    dev = require_cuda(device)
    re = np.ascontiguousarray(read_end, dtype=np.int64)
    n = len(re)
    f = np.zeros(n, np.float64)
    parent = np.full(n, NO_PREDECESSOR, np.int64)
    if n == 0:
        return f, parent
    lb = max(1, int(cfg.max_lookback))
    lut = LUTS.get(dev, cfg.max_gap, cfg.gap_open, cfg.gap_extend, cfg.log_coeff)
    fd = torch.empty(n, dtype=torch.float64, device=dev)
    pd = torch.empty(n, dtype=torch.int32, device=dev)
    bd = None
    if bonus is not None:
        bd = to_device(np.ascontiguousarray(bonus, dtype=np.float64).reshape(n, lb), dev)
    _launch_chain_dp(to_device(np.array([0, n], np.int64), dev), to_device(re.astype(np.int32), dev),
                     to_device(np.asarray(ref_end).astype(np.int32), dev),
                     to_device(np.asarray(weight, dtype=np.float64), dev), bd, lb, cfg.max_gap, lut, fd, pd, 1)
    return fd.cpu().numpy(), pd.cpu().numpy().astype(np.int64)


def chain_dp(anchors: torch.Tensor, n_anchors: torch.Tensor, lookback: int, max_gap: int,
             gap_open: float, gap_extend: float, log_coeff: float, bonus: Optional[torch.Tensor] = None,
             weights: Optional[torch.Tensor] = None):
    """Batched chaining DP with the cuda_kernels.py L440-501 signature:
    ``anchors (B, A, 3)`` int32 ``(read_end, ref_end, reserved)`` sorted by
    reference end, ``n_anchors (B,)``, optional ``bonus (B, A, lookback)`` and
    ``weights (B, A)``.  Returns ``(f (B, A) float64, p (B, A) int64)``;
    padded slots hold 0 / -1."""
    dev = require_cuda(anchors.device if anchors.is_cuda else None)
    B, A, _ = anchors.shape
    lb = max(1, int(lookback))
    an = anchors.to(dev)
    counts = n_anchors.to(dev).long().clamp(0, A)
    valid = torch.arange(A, device=dev)[None, :] < counts[:, None]
    row_off = torch.zeros(B + 1, dtype=torch.int64, device=dev)
    row_off[1:] = torch.cumsum(counts, 0)
    read_end = an[..., 0][valid].to(torch.int32).contiguous()
    ref_end = an[..., 1][valid].to(torch.int32).contiguous()
    w = (weights.to(dev) if weights is not None else an[..., 2])[valid].to(torch.float64).contiguous()
    bd = None
    if bonus is not None:
        bd = bonus.to(dev)[valid].to(torch.float64).reshape(-1, lb).contiguous()
    lut = LUTS.get(dev, max_gap, gap_open, gap_extend, log_coeff)
    n = int(read_end.numel())
    f_flat = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
    p_flat = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    if n:
        _launch_chain_dp(row_off, read_end, ref_end, w, bd, lb, max_gap, lut, f_flat, p_flat, B)
    f = torch.zeros((B, A), dtype=torch.float64, device=dev)
    p = torch.full((B, A), NO_PREDECESSOR, dtype=torch.int64, device=dev)
    f[valid] = f_flat[:n]
    p[valid] = p_flat[:n].long()
    return f, p


# --------------------------------------------------------------------------- #
# Stage entry point
# --------------------------------------------------------------------------- #
class AffineChainer:
    """Stage 2 entry point (chaining.py L292-745): anchors -> ranked chains.

    Fast mode (length weights, no graph context) runs entirely on the
    device.  Contexts that change weights or add a bonus (hybrid mode) are
    prepared on the host by :mod:`graphmambaformer_b200.hybrid` and fed to the
    same device DP / peel / select.
    """

    def __init__(self, cfg: Optional[ChainingConfig] = None, backend: str = "b200",
                 workers: Optional[int] = None, device=None):
        self.cfg = cfg or ChainingConfig()
        self.backend = backend
        self._workers = workers
        self._device = device

    def chain(self, anchors: AnchorSet, ctx=None, device=None) -> list:
        return self.chain_batch([anchors], [ctx], device=device)[0]

    def chain_batch(self, anchor_sets: Sequence, contexts=None, device=None) -> list:
        dev = require_cuda(device if device is not None else self._device)
        contexts = list(contexts or [None] * len(anchor_sets))
        if not anchor_sets:
            return []
        from . import hybrid

        if hybrid.needs_host_inputs(self.cfg, anchor_sets, contexts):
            return hybrid.chain_batch_hybrid(self, anchor_sets, contexts, dev)
        res = chain_anchor_batch(AnchorCSR.from_sets(anchor_sets), self.cfg, dev)
        return [res.chains(r) for r in range(len(anchor_sets))]
