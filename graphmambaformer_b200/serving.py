"""Serving loop: chaining + extension for a stream of read requests.

A request carries 1..64 reads (base codes) and, when the server holds no
minimizer index, their raw minimizer anchors (client-side seeding).  The
server keeps the reference codes, the chaining penalty table and optionally
the minimizer index resident on the device and, per batch of reads, runs the
classical path (alignment/seeding.py L1056-1101 MinimizerIndex seeding, then
alignment/chaining.py L620-745 and alignment/extension.py L469-641):

  0. with an index: ``gmf_seed_count`` / ``gmf_seed_fill`` on the device;
  1. ``gmf_chain_batch``: strand split + sort, DP, chain peeling, select;
  2. the window and band of every kept chain (extension.py L489-509, on the
     host from the chain records), then ``gmf_gather_segments`` builds the
     queries (reads, reverse-complemented for strand -1) and the target
     windows from the resident buffers on the device;
  3. ``gmf_banded_sw`` (batched form) + CIGAR assembly with soft clips.

Continuous batching: a dispatcher admits pending requests first-come
first-served into a batch whenever one of the workers is free, as long as
the batch's estimated device memory fits the working-memory budget (8 GB by
default) next to the batches in flight.  Each worker runs its batches on its
own CUDA stream, so a batch formed from requests that arrived while others
were on the GPU overlaps with them on the device.  Per-read results do not
depend on the batch (every stage is per read / per pair), so a request gets
the same alignments alone or in any mix.
"""

from __future__ import annotations

import ctypes
import queue
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np
import torch

from . import _native
from .chaining import LUTS, AnchorCSR, ChainingConfig, chain_params
from .config import ExtensionConfig
from .device import bind, require_cuda
from .extension import longest_first, params_from_config
from .session import _Buffers


def estimate_bytes(read_lens: np.ndarray, n_anchors: int, cfg: ExtensionConfig, max_chains: int) -> int:
    """Upper bound on a batch's device working memory: anchors with the
    chaining workspace, and every possible chain's traceback bits."""
    W = 2 * cfg.max_half_band + 1
    cells = int(np.sum((np.asarray(read_lens, np.int64) + 2 * cfg.flank) * W)) * min(max_chains, 2)
    return int(120 * n_anchors + cells // 2 + 64 * len(read_lens) + (1 << 20))


class BatchAlignments:
    """The alignments of a batch of reads, kept as arrays: one entry per kept
    chain, chains in read order and, within a read, in select order.  Item
    ``i`` is read i's list of ExtensionResults (as AffineChainer.chain +
    ExtensionEngine.extend_chains give them), built when it is read; a slice
    is a view of a range of reads.  Holding the batch as arrays keeps the
    serving loop free of per-chain Python work; a client pays for the
    objects of the reads it looks at."""

    def __init__(self, n_reads: int, chain_off: np.ndarray, cols: Optional[dict] = None,
                 words: Optional[np.ndarray] = None, objects: Optional[list] = None, lo: int = 0,
                 hi: Optional[int] = None, chains: Optional[dict] = None):
        self.n_reads = int(n_reads)
        self.chain_off = chain_off  # n_reads + 1: the chains of read r are chain_off[r] .. chain_off[r+1]-1
        self.cols = cols            # per chain: score, qs, qe, ts, te, counts (C, 4), cstart, clen, clip_l, clip_r
        self.words = words          # CIGAR words (run << 4 | op), without the soft clips
        self.objects = objects      # or per chain, ready ExtensionResults (the WFA path)
        self.chains = chains        # per chain: the chain's score (f64), strand and primary flag
        self.lo = int(lo)
        self.hi = self.n_reads if hi is None else int(hi)

    @staticmethod
    def empty(n_reads: int) -> "BatchAlignments":
        z = np.zeros(0, np.int32)
        return BatchAlignments(n_reads, np.zeros(n_reads + 1, np.int64), objects=[],
                               chains=dict(score=np.zeros(0), strand=z, prim=z))

    def __len__(self) -> int:
        return self.hi - self.lo

    def _chain(self, c: int):
        from .types import ExtensionResult, add_soft_clips, words_to_cigar

        if self.objects is not None:
            return self.objects[c]
        k = self.cols
        s0, n = int(k["cstart"][c]), int(k["clen"][c])
        cnt = k["counts"][c]
        return ExtensionResult(
            score=float(k["score"][c]),
            cigar=add_soft_clips(words_to_cigar(self.words[s0: s0 + n]), int(k["clip_l"][c]), int(k["clip_r"][c])),
            read_start=int(k["qs"][c]), read_end=int(k["qe"][c]), ref_start=int(k["ts"][c]),
            ref_end=int(k["te"][c]), n_match=int(cnt[0]), n_mismatch=int(cnt[1]), n_insertion=int(cnt[2]),
            n_deletion=int(cnt[3]))

    def __getitem__(self, i):
        if isinstance(i, slice):
            a, b, step = i.indices(len(self))
            if step != 1:
                raise ValueError("BatchAlignments slices take consecutive reads")
            return BatchAlignments(self.n_reads, self.chain_off, self.cols, self.words, self.objects,
                                   self.lo + a, self.lo + max(a, b), self.chains)
        if i < 0:
            i += len(self)
        if not 0 <= i < len(self):
            raise IndexError(i)
        r = self.lo + i
        return [self._chain(c) for c in range(int(self.chain_off[r]), int(self.chain_off[r + 1]))]

    def __iter__(self):
        for i in range(len(self)):
            yield self[i]


class BatchAligner:
    """The device pipeline for one batch of reads on one stream (grow-only
    buffers, reused between batches)."""

    def __init__(self, ref_d: torch.Tensor, device, chain_cfg: ChainingConfig, ext_cfg: ExtensionConfig,
                 stream: Optional[torch.cuda.Stream] = None, index=None):
        self.device = require_cuda(device)
        self.index = index  # a resident DeviceMinimizerIndex: seed on the device when no anchors are given
        self.ref_d = ref_d
        self.ref_len = int(ref_d.numel())
        self.ccfg, self.ecfg = chain_cfg, ext_cfg
        self.cp = chain_params(chain_cfg)
        self.sw = params_from_config(ext_cfg)
        self.lut = LUTS.get(self.device, chain_cfg.max_gap, chain_cfg.gap_open, chain_cfg.gap_extend,
                            chain_cfg.log_coeff)
        self.stream = stream or torch.cuda.Stream(self.device)
        self.buf = _Buffers(self.device)

    def _call(self, name, *args):
        _native.check(name, getattr(_native.lib(), name)(*args))

    def align(self, reads: Sequence[np.ndarray], anchors=None) -> list:
        """Per read, the list of its chains' ExtensionResults (in select
        order), exactly as AffineChainer.chain + ExtensionEngine.extend_chains
        give them.  Without ``anchors`` the reads are seeded on the device
        against the resident minimizer index."""
        R = len(reads)
        if R == 0:
            return []
        if anchors is None and self.index is None:
            raise ValueError("anchors are required unless the aligner holds a minimizer index")
        s, up, db = self.stream, self.buf.upload, self.buf.device_buf
        sp = int(s.cuda_stream)
        bind(self.device, sp)
        rl = np.array([len(x) for x in reads], np.int64)
        roff = np.zeros(R + 1, np.int64)
        np.cumsum(rl, out=roff[1:])
        codes = np.concatenate(reads).astype(np.int8) if roff[-1] else np.zeros(1, np.int8)
        reads_d = up("reads", codes, s)
        pad = lambda x, dt: x if len(x) else np.zeros(1, dt)  # noqa: E731
        if anchors is None:  # device seeding: both orientations, forward anchors first
            sd = self.index.seed_device(reads_d, up("roff", roff, s), R, True, stream=s)
            ro, rp, fp, ln, st = sd["read_off"], sd["read_pos"], sd["ref_pos"], sd["length"], sd["strand"]
            A = int(sd["n_anchors"])
            per_read = int(sd["max_read_anchors"])
        else:
            a = AnchorCSR.of(anchors)
            if R != len(a):
                raise ValueError("one anchor set per read is required")
            A = int(a.read_off[-1])
            per_read = int(np.diff(a.read_off).max(initial=0))
            ro = up("ro", a.read_off, s)
            rp = up("rp", pad(a.read_pos, np.int32), s)
            fp = up("fp", pad(a.ref_pos, np.int32), s)
            ln = up("ln", pad(a.length, np.int32), s)
            st = up("st", pad(a.strand, np.int8), s)
        if per_read > _native.MAX_READ_ANCHORS:
            raise ValueError(f"a read has more than {_native.MAX_READ_ANCHORS} anchors")
        mc = self.cp.max_chains
        o = dict(n=db("n", R, torch.int32), score=db("score", R * mc, torch.float64),
                 strand=db("strand", R * mc, torch.int32), span=db("span", 4 * R * mc, torch.int32),
                 prim=db("prim", R * mc, torch.int32), nmem=db("nmem", R * mc, torch.int32),
                 mem=db("mem", max(A, 1), torch.int32))
        need = int(_native.lib().gmf_chain_workspace_bytes(R, A))
        ws = db("cws", need, torch.uint8)
        batch_c = _native.GmfAnchorBatch(R, ro.data_ptr(), rp.data_ptr(), fp.data_ptr(), ln.data_ptr(), st.data_ptr())
        res_c = _native.GmfChainResults(o["n"].data_ptr(), o["score"].data_ptr(), o["strand"].data_ptr(),
                                        o["span"].data_ptr(), o["prim"].data_ptr(), o["nmem"].data_ptr(),
                                        o["mem"].data_ptr())
        self._call("gmf_chain_batch", ctypes.byref(batch_c), ctypes.byref(self.cp),
                   ctypes.c_void_p(self.lut.data_ptr()), self.lut.numel(), None, None, None, ctypes.byref(res_c),
                   ctypes.c_void_p(ws.data_ptr()), need, ctypes.c_void_p(sp))
        # the diagonal spread of every chain, on the device beside the chain records
        spread_d = db("spread", R * mc, torch.int32)
        self._call("gmf_chain_spread", ctypes.byref(batch_c), ctypes.byref(res_c), mc,
                   ctypes.c_void_p(spread_d.data_ptr()), ctypes.c_void_p(sp))
        dl = self.buf.download
        h = {k: dl("h_" + k, t, n, s) for k, t, n in
             (("n", o["n"], R), ("strand", o["strand"], R * mc), ("span", o["span"], 4 * R * mc),
              ("spread", spread_d, R * mc), ("score", o["score"], R * mc), ("prim", o["prim"], R * mc))}
        s.synchronize()
        n_ch = np.minimum(h["n"][:R].numpy(), mc)
        strand = h["strand"][: R * mc].numpy().reshape(R, mc)
        span = h["span"][: 4 * R * mc].numpy().reshape(R, mc, 4)
        spread_all = h["spread"][: R * mc].numpy().reshape(R, mc)

        # ---- one pair per kept chain, in read order ----
        cr, ck = np.nonzero(np.arange(mc)[None, :] < n_ch[:, None])  # (read, slot) of every chain
        C = len(cr)
        chain_off = np.zeros(R + 1, np.int64)
        np.cumsum(n_ch, out=chain_off[1:])
        if C == 0:
            return BatchAlignments.empty(R)
        spread = spread_all[cr, ck].astype(np.int64)
        chains = dict(score=h["score"][: R * mc].numpy().reshape(R, mc)[cr, ck],
                      strand=strand[cr, ck].copy(), prim=h["prim"][: R * mc].numpy().reshape(R, mc)[cr, ck])
        rc = strand[cr, ck] < 0
        sp4 = span[cr, ck].astype(np.int64)  # read_start, read_end, ref_start, ref_end
        if self.ecfg.algorithm == "wfa":
            return BatchAlignments(R, chain_off, objects=self._extend_wfa(R, rl, roff, reads_d, cr, rc, sp4, spread),
                                   chains=chains)
        cols, words = self._extend_sw(R, rl, roff, reads_d, cr, rc, sp4, spread, shared=True)
        return BatchAlignments(R, chain_off, cols, words, chains=chains)

    def _gather(self, tag: str, reads_d, roff, rl, cr, rc, wstart, wlen) -> tuple:
        """Queries (reverse-complemented for strand -1) and reference
        windows of the pairs, gathered from the resident buffers."""
        s, up, db = self.stream, self.buf.upload, self.buf.device_buf
        sp = int(s.cuda_stream)
        C = len(cr)
        rlen = rl[cr]
        qoff = np.zeros(C + 1, np.int64)
        np.cumsum(rlen, out=qoff[1:])
        toff = np.zeros(C + 1, np.int64)
        np.cumsum(wlen, out=toff[1:])
        qd = db(tag + "q", max(int(qoff[-1]), 1), torch.int8)
        td = db(tag + "t", max(int(toff[-1]), 1), torch.int8)
        qs_d, ql_d = up(tag + "qs", roff[cr], s), up(tag + "ql", rlen.astype(np.int32), s)
        rc_d, qo_d = up(tag + "rc", rc.astype(np.int8), s), up(tag + "qo", qoff, s)
        ts_d, tl_d, to_d = up(tag + "ts", wstart, s), up(tag + "tl", wlen.astype(np.int32), s), up(tag + "to", toff, s)
        self._call("gmf_gather_segments", ctypes.c_void_p(reads_d.data_ptr()), int(roff[-1]), C,
                   ctypes.c_void_p(qs_d.data_ptr()), ctypes.c_void_p(ql_d.data_ptr()),
                   ctypes.c_void_p(rc_d.data_ptr()), ctypes.c_void_p(qd.data_ptr()),
                   ctypes.c_void_p(qo_d.data_ptr()), ctypes.c_void_p(sp))
        self._call("gmf_gather_segments", ctypes.c_void_p(self.ref_d.data_ptr()), self.ref_len, C,
                   ctypes.c_void_p(ts_d.data_ptr()), ctypes.c_void_p(tl_d.data_ptr()), None,
                   ctypes.c_void_p(td.data_ptr()), ctypes.c_void_p(to_d.data_ptr()), ctypes.c_void_p(sp))
        return qd, qo_d, td, to_d, qoff, toff

    def _extend_sw(self, R, rl, roff, reads_d, cr, rc, sp4, spread, shared: bool) -> list:
        """Banded SW + traceback of the pairs (extension.py L489-641).  With
        ``shared``, the chains of a read take its widest band and stop
        together under x-drop, as one extend_chains call; without, every
        chain is a call of its own (the WFA fallback)."""
        s, up, db, dl = self.stream, self.buf.upload, self.buf.device_buf, self.buf.download
        sp = int(s.cuda_stream)
        cfg = self.ecfg
        C = len(cr)
        diag = sp4[:, 2] - sp4[:, 0]
        rlen = rl[cr]
        wstart = np.maximum(0, diag - cfg.flank)
        wend = np.minimum(self.ref_len, diag + rlen + cfg.flank)
        wend = np.where(wend - wstart > cfg.max_window, wstart + cfg.max_window, wend)
        wlen = np.maximum(wend - wstart, 0)
        hb = np.minimum(cfg.half_band + spread, cfg.max_half_band)
        goff = None
        if shared:
            hb_read = np.zeros(R, np.int64)
            np.maximum.at(hb_read, cr, hb)  # every chain of a read takes its widest band
            hb = hb_read[cr]
            goff = np.zeros(R + 1, np.int32)  # the chains of a read stop together under x-drop
            np.cumsum(np.bincount(cr, minlength=R), out=goff[1:])
        hb = hb.astype(np.int32)
        boff = (diag - wstart).astype(np.int32)
        qd, qo_d, td, to_d, qoff, toff = self._gather("s", reads_d, roff, rl, cr, rc, wstart, wlen)
        hb_d, bo_d = up("hb", hb, s), up("bo", boff, s)
        ord_d = up("ord", longest_first(rlen.astype(np.int32), hb), s)
        out = dict(score=db("sc", C, torch.int32), qe=db("qe", C, torch.int32), te=db("te", C, torch.int32),
                   qs=db("qs2", C, torch.int32), ts=db("ts2", C, torch.int32), clen=db("cl", C, torch.int32),
                   counts=db("cn", 4 * C, torch.int32), cstart=db("cs", C, torch.int64),
                   used=db("used", 1, torch.int64), err=db("err", 1, torch.int32))
        cap = int(qoff[-1] + toff[-1] + C)
        cigar = db("cigar", cap, torch.int32)
        need = int(_native.lib().gmf_banded_sw_workspace_bytes(
            C, rlen.astype(np.int32).ctypes.data_as(ctypes.c_void_p),
            wlen.astype(np.int32).ctypes.data_as(ctypes.c_void_p), hb.ctypes.data_as(ctypes.c_void_p), 1))
        sws = db("sws", need, torch.uint8)
        go_d = up("go", goff, s) if goff is not None else None
        pairs_c = _native.GmfPairs(C, qd.data_ptr(), qo_d.data_ptr(), td.data_ptr(), to_d.data_ptr(), hb_d.data_ptr(),
                                   bo_d.data_ptr(), ord_d.data_ptr(), int(hb.max()),
                                   go_d.data_ptr() if go_d is not None else None, R if goff is not None else 0)
        sres = _native.GmfSwResults(out["score"].data_ptr(), out["qe"].data_ptr(), out["te"].data_ptr(),
                                    out["qs"].data_ptr(), out["ts"].data_ptr(), out["counts"].data_ptr(),
                                    cigar.data_ptr(), cap, out["cstart"].data_ptr(), out["clen"].data_ptr(),
                                    out["used"].data_ptr(), out["err"].data_ptr())
        self._call("gmf_banded_sw", ctypes.byref(pairs_c), ctypes.byref(self.sw), ctypes.byref(sres),
                   ctypes.c_void_p(sws.data_ptr()), need, ctypes.c_void_p(sp))
        hh = {k: dl("h2_" + k, out[k], n, s) for k, n in
              (("score", C), ("qe", C), ("te", C), ("qs", C), ("ts", C), ("clen", C), ("counts", 4 * C),
               ("cstart", C), ("used", 1), ("err", 1))}
        s.synchronize()
        used = int(hh["used"][0])
        words = dl("h2_cigar", cigar, used, s)
        s.synchronize()
        err = int(hh["err"][0])
        if err:
            raise RuntimeError(f"gmf_banded_sw reported error flags {err}")
        # ExtensionEngine._finish as arrays: reference coordinates from the window start, soft clips from
        # the unaligned ends of the read (copies: the staging buffers are reused by the next batch)
        qs, qe = hh["qs"][:C].numpy().copy(), hh["qe"][:C].numpy().copy()
        cols = dict(score=hh["score"][:C].numpy().copy(), qs=qs, qe=qe,
                    ts=hh["ts"][:C].numpy().astype(np.int64) + wstart,
                    te=hh["te"][:C].numpy().astype(np.int64) + wstart,
                    counts=hh["counts"][: 4 * C].numpy().reshape(C, 4).copy(),
                    cstart=hh["cstart"][:C].numpy().copy(), clen=hh["clen"][:C].numpy().copy(),
                    clip_l=qs, clip_r=rlen - qe)
        if not shared:  # the WFA fallback wants ExtensionResults of these chains
            b = BatchAlignments(C, np.arange(C + 1, dtype=np.int64), cols, words[:used].numpy().view(np.uint32).copy())
            return [b[c][0] for c in range(C)]
        return cols, words[:used].numpy().view(np.uint32).copy()

    def _extend_wfa(self, R, rl, roff, reads_d, cr, rc, sp4, spread) -> list:
        """The extension's wfa mode (extension.py L643-730) on the gathered
        pairs: global wavefront alignment against the stretch the chain's
        read-zero diagonal and net indel imply; chains beyond the distance
        bound go to banded SW one chain per call, as the reference re-enters
        extend_chains."""
        from .extension import wfa_extension_result
        from .wfa import DeviceWfaPairs, align_device_pairs

        cfg = self.ecfg
        rlen = rl[cr]
        wstart = np.clip(sp4[:, 2] - sp4[:, 0], 0, max(self.ref_len - 1, 0))
        net = (sp4[:, 3] - sp4[:, 2]) - (sp4[:, 1] - sp4[:, 0])
        wend = np.minimum(self.ref_len, wstart + np.maximum(1, rlen + net))
        wlen = np.maximum(wend - wstart, 0)
        qd, qo_d, td, to_d, _, _ = self._gather("w", reads_d, roff, rl, cr, rc, wstart, wlen)
        dp = DeviceWfaPairs(len(cr), qd, qo_d, td, to_d, rlen.astype(np.int32), wlen.astype(np.int32), self.device)
        res = align_device_pairs(dp, cfg.wfa_max_distance, stream=self.stream,
                                 workspace=lambda nb: self.buf.device_buf("wws", nb, torch.uint8))
        exts = [None] * len(cr)
        far = np.nonzero(res.distance < 0)[0]
        for c in np.nonzero(res.distance >= 0)[0]:
            exts[c] = wfa_extension_result(res.cigar(int(c)), int(wstart[c]), int(wlen[c]), int(rlen[c]), cfg)
        if len(far):
            for c, e in zip(far, self._extend_sw(R, rl, roff, reads_d, cr[far], rc[far], sp4[far], spread[far],
                                                 shared=False)):
                exts[c] = e
        return exts


@dataclass
class Request:
    rid: int
    reads: list
    anchors: object
    nbytes: int
    arrival: float
    future: Future = field(default_factory=Future)
    done: float = 0.0


class AlignServer:
    """Continuous-batching server of chaining + extension requests."""

    def __init__(self, ref_codes: np.ndarray, device=None, chain_cfg: Optional[ChainingConfig] = None,
                 ext_cfg: Optional[ExtensionConfig] = None, budget_bytes: int = 8 << 30,
                 max_batch_reads: int = 512, workers: int = 2, index=None):
        self.device = require_cuda(device)
        self.ccfg = chain_cfg or ChainingConfig()
        self.ecfg = ext_cfg or ExtensionConfig()
        self.budget = int(budget_bytes)
        self.max_batch_reads = int(max_batch_reads)
        torch.cuda.set_device(self.device)
        self.ref_d = torch.from_numpy(np.ascontiguousarray(ref_codes, np.int8)).to(self.device)  # resident
        self.index = index  # with a resident minimizer index, requests carry reads only
        self.workers = [BatchAligner(self.ref_d, self.device, self.ccfg, self.ecfg, index=index)
                        for _ in range(workers)]
        self.free: "queue.Queue[BatchAligner]" = queue.Queue()
        for w in self.workers:
            self.free.put(w)
        self.pending: "queue.Queue[Request]" = queue.Queue()
        self.in_flight_bytes = 0
        self.lock = threading.Lock()
        self.completed: list = []
        self.batches = 0
        self._next = 0
        self._stop = threading.Event()
        self._dispatcher = threading.Thread(target=self._dispatch, daemon=True)
        self._threads: list = []

    # -- client side -------------------------------------------------------------
    def submit(self, reads: Sequence[np.ndarray], anchors=None) -> Future:
        """Queue a request; ``anchors`` (per read, both orientations) are
        required unless the server holds a minimizer index, in which case the
        reads are seeded on the device and client anchors are not used."""
        rl = np.array([len(x) for x in reads], np.int64)
        if self.index is not None:
            a = None
            n_anchors = int(rl.sum() * 2 * 2 // (self.index.w + 1)) + 1  # minimizer density bound
        else:
            if anchors is None:
                raise ValueError("anchors are required: the server has no minimizer index")
            a = AnchorCSR.of(anchors)
            n_anchors = int(a.read_off[-1])
        nb = estimate_bytes(rl, n_anchors, self.ecfg, self.ccfg.max_chains)
        if nb > self.budget:
            raise ValueError("request larger than the working-memory budget")
        with self.lock:
            rid = self._next
            self._next += 1
        req = Request(rid, list(reads), a, nb, time.perf_counter())
        self.pending.put(req)
        return req.future

    def start(self) -> "AlignServer":
        self._dispatcher.start()
        return self

    def stop(self) -> None:
        self._stop.set()
        self._dispatcher.join(timeout=30)
        for t in self._threads:
            t.join(timeout=60)

    # -- server side -------------------------------------------------------------
    def _dispatch(self) -> None:
        carry: Optional[Request] = None
        while not self._stop.is_set():
            try:
                w = self.free.get(timeout=0.05)
            except queue.Empty:
                continue
            batch, nbytes, nreads = [], 0, 0
            deadline = time.perf_counter() + 0.5
            while True:
                if carry is None:
                    try:
                        carry = self.pending.get(timeout=0.001 if batch else 0.05)
                    except queue.Empty:
                        if batch or self._stop.is_set() or time.perf_counter() > deadline:
                            break
                        continue
                with self.lock:
                    fits = self.in_flight_bytes + nbytes + carry.nbytes <= self.budget
                if batch and (not fits or nreads + len(carry.reads) > self.max_batch_reads):
                    break
                if not batch and not fits:  # wait for memory to free up
                    time.sleep(0.001)
                    continue
                batch.append(carry)
                nbytes += carry.nbytes
                nreads += len(carry.reads)
                carry = None
            if not batch:
                self.free.put(w)
                continue
            with self.lock:
                self.in_flight_bytes += nbytes
            t = threading.Thread(target=self._run, args=(w, batch, nbytes), daemon=True)
            self._threads = [x for x in self._threads if x.is_alive()] + [t]
            t.start()

    def _run(self, w: BatchAligner, batch: list, nbytes: int) -> None:
        try:
            reads = [r for req in batch for r in req.reads]
            anchors = None
            if self.index is None:
                anchors = AnchorCSR.from_sets(
                    [_ReadAnchors(req.anchors, i) for req in batch for i in range(len(req.reads))])
            res = w.align(reads, anchors)
            pos = 0
            now = time.perf_counter()
            for req in batch:
                out = res[pos: pos + len(req.reads)]
                pos += len(req.reads)
                req.done = now
                req.future.set_result(out)
            with self.lock:
                self.completed.extend(batch)
                self.batches += 1
        except BaseException as e:  # surface the error to every request of the batch
            for req in batch:
                if not req.future.done():
                    req.future.set_exception(e)
        finally:
            with self.lock:
                self.in_flight_bytes -= nbytes
            self.free.put(w)

    def latency_stats(self) -> dict:
        with self.lock:
            lat = np.array([(r.done - r.arrival) * 1e3 for r in self.completed])
            nreads = sum(len(r.reads) for r in self.completed)
        if not len(lat):
            return {"requests": 0}
        return {"requests": int(len(lat)), "reads": int(nreads), "batches": self.batches,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}


class _ReadAnchors:
    """Read i of an AnchorCSR viewed as an AnchorSet-like object (for
    AnchorCSR.from_sets)."""

    def __init__(self, a: AnchorCSR, i: int):
        s, e = int(a.read_off[i]), int(a.read_off[i + 1])
        self.read_pos, self.ref_pos = a.read_pos[s:e], a.ref_pos[s:e]
        self.length, self.strand = a.length[s:e], a.strand[s:e]

    def __len__(self) -> int:
        return len(self.read_pos)


def serve_stream(server: AlignServer, pool, requests: list, time_scale: float = 1.0) -> dict:
    """Replay a request stream against a started server (see below)."""
    return _serve_stream(server, pool, requests, time_scale)


def _serve_stream(server: AlignServer, pool, requests: list, time_scale: float = 1.0) -> dict:
    """Replay a request stream (list of (arrival seconds, read indices)
    into ``pool``) against a started server, then wait for every result.
    Returns latency / throughput figures."""
    t0 = time.perf_counter()
    futs = []
    for arr, idx in requests:
        wait = t0 + arr * time_scale - time.perf_counter()
        if wait > 0:
            time.sleep(wait)
        if server.index is not None:  # the server seeds: the request carries bare reads
            futs.append(server.submit([pool.reads[int(i)] for i in idx]))
        else:
            reads, anchors = pool.take(idx)
            futs.append(server.submit(reads, anchors))
    for f in futs:
        f.result(timeout=600)
    wall = time.perf_counter() - t0
    st = server.latency_stats()
    st["wall_s"] = wall
    st["reads_per_s"] = st.get("reads", 0) / wall if wall > 0 else 0.0
    return st
