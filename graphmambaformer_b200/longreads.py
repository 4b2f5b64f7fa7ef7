"""Long-read stress path: chaining with a wide predecessor window, then
banded SW over the gaps between chained anchors.

The reference extends one window per chain (alignment/extension.py
L469-641); for 50-100 kb reads that window would be a 100 kb x 4 kb band, so
this path aligns the chain piecewise instead.  The segmentation rule, used
by both the device path and the oracle parity tests:

* only the read's primary chain (the first chain ``select`` keeps) is used;
* its member anchors, in read order (the chain's own orientation: reverse-
  complement read coordinates for strand -1), are kept greedily from the
  first one: an anchor is kept when its read start is at least
  ``min_spacing`` (1,000) bases after the last kept one; the last member is
  always kept;
* consecutive kept anchors u, v give one segment: query = read[u.read_pos :
  v.read_pos] (in the chain's orientation), target = ref[u.ref_pos - pad :
  v.ref_pos + pad] clipped to the reference (pad = 32), band offset =
  u.ref_pos - target start, half band = clip(32 + |drift| + qlen * b //
  1000, 32, 2000) where drift = (v.ref_pos - u.ref_pos) - (v.read_pos -
  u.read_pos) and b is the band growth per kb;
* two modes: ``FINE`` (min_spacing 1,000, b = 20, i.e. qlen // 50: bands of
  about 50-80 on 1 kb gaps) and ``WIDE`` (min_spacing 8,000, b = 250: the
  chain cut into 8 kb stretches whose half bands reach the 2,000 limit, the
  shorter last stretch of each chain below it: the stress configuration's
  bands up to 2,000);
* each segment is a local banded SW + traceback with the extension stage's
  scoring (``banded_affine_sw_batch`` + ``traceback_banded`` semantics, B = 1
  per segment), which is what the parity tests compare.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from . import _native
from .chaining import AnchorCSR, ChainingConfig
from .config import ExtensionConfig
from .device import bind, require_cuda
from .extension import SWResult, fetch, longest_first, params_from_config
from .serving import BatchAligner

MIN_SPACING = 1000
PAD = 32
BASE_BAND = 32
MAX_BAND = 2000
BAND_PER_KB = 20

# segmentation modes: (min_spacing, band growth per kb)
FINE = (MIN_SPACING, BAND_PER_KB)
WIDE = (8000, 250)


@dataclass
class Segments:
    """Gap segments of a batch: read index, strand, query slice (in the
    chain's orientation), target slice of the reference, band."""

    read: np.ndarray      # int64
    strand: np.ndarray    # int8
    q_start: np.ndarray   # int64, in the chain's orientation
    q_len: np.ndarray     # int64
    t_start: np.ndarray   # int64
    t_len: np.ndarray     # int64
    half_band: np.ndarray  # int32
    band_offset: np.ndarray  # int32

    def __len__(self) -> int:
        return len(self.read)


def segment_chain(read_pos: np.ndarray, ref_pos: np.ndarray, ref_len: int,
                  min_spacing: int = MIN_SPACING, pad: int = PAD, band_per_kb: int = BAND_PER_KB):
    """Segments of one chain from its member anchors (read order): lists of
    (q_start, q_len, t_start, t_len, half_band, band_offset)."""
    rp = np.asarray(read_pos, np.int64)
    fp = np.asarray(ref_pos, np.int64)
    if len(rp) < 2:
        return []
    kept = [0]
    for i in range(1, len(rp) - 1):
        if rp[i] >= rp[kept[-1]] + min_spacing:
            kept.append(i)
    if kept[-1] != len(rp) - 1:
        kept.append(len(rp) - 1)
    out = []
    for u, v in zip(kept[:-1], kept[1:]):
        qs, qe = int(rp[u]), int(rp[v])
        if qe <= qs:
            continue
        ts = max(0, int(fp[u]) - pad)
        te = min(ref_len, int(fp[v]) + pad)
        drift = (int(fp[v]) - int(fp[u])) - (qe - qs)
        hb = int(np.clip(BASE_BAND + abs(drift) + (qe - qs) * band_per_kb // 1000, BASE_BAND, MAX_BAND))
        out.append((qs, qe - qs, ts, max(te - ts, 0), hb, int(fp[u]) - ts))
    return out


class LongReadAligner(BatchAligner):
    """Device path of the long-read stress workload: ``gmf_chain_batch``
    (lookback 200 by default), the segmentation above on the host,
    ``gmf_gather_segments`` for queries and targets, batched
    ``gmf_banded_sw``."""

    def __init__(self, ref_d: torch.Tensor, device, chain_cfg: Optional[ChainingConfig] = None,
                 ext_cfg: Optional[ExtensionConfig] = None, stream=None):
        super().__init__(ref_d, device, chain_cfg or ChainingConfig(max_lookback=200), ext_cfg or ExtensionConfig(),
                         stream)

    def primary_chains(self, reads, anchors):
        """(strand, member read_pos, member ref_pos) of each read's primary
        chain (None when a read has no chain), from the device chainer."""
        from .chaining import launch_chain_batch, upload_anchors, fetch_chains

        a = AnchorCSR.of(anchors)
        with torch.cuda.stream(self.stream):
            da = upload_anchors(a, self.device)
            res = fetch_chains(launch_chain_batch(da, self.ccfg, stream=self.stream), a.read_off)
        out = []
        for r in range(len(a)):
            ch = res.chains(r)
            if not ch:
                out.append(None)
                continue
            g = a.read_off[r] + ch[0].anchor_idx
            order = np.argsort(a.read_pos[g], kind="stable")
            out.append((int(ch[0].strand), a.read_pos[g][order], a.ref_pos[g][order]))
        return out, res

    def segments(self, reads, primaries, mode=FINE) -> Segments:
        """Gap segments of the primary chains under a segmentation mode
        (``FINE`` or ``WIDE``)."""
        cols = [[] for _ in range(8)]
        spacing, per_kb = mode
        for r, pc in enumerate(primaries):
            if pc is None:
                continue
            strand, rp, fp = pc
            for s in segment_chain(rp, fp, self.ref_len, min_spacing=spacing, band_per_kb=per_kb):
                for c, v in zip(cols, (r, strand) + s):
                    c.append(v)
        return Segments(np.array(cols[0], np.int64), np.array(cols[1], np.int8), np.array(cols[2], np.int64),
                        np.array(cols[3], np.int64), np.array(cols[4], np.int64), np.array(cols[5], np.int64),
                        np.array(cols[6], np.int32), np.array(cols[7], np.int32))

    def align_segments(self, reads, seg: Segments, traceback: bool = True) -> SWResult:
        """Banded SW + traceback of every segment (one launch)."""
        from .extension import SWOutputs, DevicePairs, launch_banded_sw

        s, up, db = self.stream, self.buf.upload, self.buf.device_buf
        sp = int(s.cuda_stream)
        bind(self.device, sp)
        S = len(seg)
        rl = np.array([len(x) for x in reads], np.int64)
        roff = np.zeros(len(reads) + 1, np.int64)
        np.cumsum(rl, out=roff[1:])
        reads_d = up("lr_reads", np.concatenate(reads).astype(np.int8) if roff[-1] else np.zeros(1, np.int8), s)
        # query slice in the chain's orientation: for strand -1, revcomp(read)[a:b] is
        # read[L-b : L-a] reversed and complemented
        L = rl[seg.read]
        src_start = np.where(seg.strand < 0, roff[seg.read] + L - (seg.q_start + seg.q_len),
                             roff[seg.read] + seg.q_start)
        qoff = np.zeros(S + 1, np.int64)
        np.cumsum(seg.q_len, out=qoff[1:])
        toff = np.zeros(S + 1, np.int64)
        np.cumsum(seg.t_len, out=toff[1:])
        qd = db("lr_q", max(int(qoff[-1]), 1), torch.int8)
        td = db("lr_t", max(int(toff[-1]), 1), torch.int8)
        vp = ctypes.c_void_p
        self._call("gmf_gather_segments", vp(reads_d.data_ptr()), int(roff[-1]), S,
                   vp(up("lr_qs", src_start, s).data_ptr()), vp(up("lr_ql", seg.q_len.astype(np.int32), s).data_ptr()),
                   vp(up("lr_rc", (seg.strand < 0).astype(np.int8), s).data_ptr()), vp(qd.data_ptr()),
                   vp(up("lr_qo", qoff, s).data_ptr()), vp(sp))
        self._call("gmf_gather_segments", vp(self.ref_d.data_ptr()), self.ref_len, S,
                   vp(up("lr_ts", seg.t_start, s).data_ptr()), vp(up("lr_tl", seg.t_len.astype(np.int32), s).data_ptr()),
                   None, vp(td.data_ptr()), vp(up("lr_to", toff, s).data_ptr()), vp(sp))
        dp = DevicePairs(n=S, query=qd, query_off=up("lr_qo2", qoff, s), target=td, target_off=up("lr_to2", toff, s),
                         half_band=up("lr_hb", seg.half_band, s), band_offset=up("lr_bo", seg.band_offset, s),
                         order=up("lr_ord", longest_first(seg.q_len.astype(np.int32), seg.half_band), s),
                         max_half_band=int(seg.half_band.max()) if S else 0,
                         h_qlen=seg.q_len.astype(np.int32), h_tlen=seg.t_len.astype(np.int32), h_hb=seg.half_band,
                         device=self.device)
        with torch.cuda.stream(s):
            out = launch_banded_sw(dp, self.sw, traceback, stream=s)
            return fetch(out, S)
