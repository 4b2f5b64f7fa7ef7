"""Throughput API: reusable sessions for repeated batches.

A session keeps pinned host staging buffers, device input/output buffers and
the workspace alive between calls (all grow-only), so a steady stream of
batches pays only the copies and the kernels.  ``align`` / ``chain`` take
host arrays and return host arrays: this is the end-to-end path a service
calls, and the one ``bench.py`` measures as ``e2e``.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from . import _native
from .chaining import AnchorCSR, ChainResult, ChainingConfig, LUTS, chain_params
from .device import bind, require_cuda
from .extension import SWResult, longest_first, sw_params
from .synth import PairSet


class _Buffers:
    """Grow-only pinned host + device buffer pairs, one per named slot."""

    def __init__(self, device: torch.device):
        self.device = device
        self.host: dict[str, torch.Tensor] = {}
        self.dev: dict[str, torch.Tensor] = {}

    def _grow(self, table, name, n, dtype, pinned):
        t = table.get(name)
        if t is None or t.numel() < n or t.dtype != dtype:
            size = max(n, int(t.numel() * 1.25) if t is not None and t.dtype == dtype else n, 1)
            if pinned:
                t = torch.empty(size, dtype=dtype, pin_memory=True)
            else:
                t = torch.empty(size, dtype=dtype, device=self.device)
            table[name] = t
        return t

    def upload(self, name: str, a: np.ndarray, stream) -> torch.Tensor:
        """Stage ``a`` in pinned memory and copy it to the device buffer."""
        a = np.ascontiguousarray(a)
        dt = torch.from_numpy(a[:0]).dtype if a.size == 0 else torch.from_numpy(a).dtype
        n = a.size
        h = self._grow(self.host, name, n, dt, True)
        d = self._grow(self.dev, name, n, dt, False)
        if n:
            h[:n].copy_(torch.from_numpy(a.reshape(-1)))  # torch's host copy runs on several threads
            with torch.cuda.stream(stream):
                d[:n].copy_(h[:n], non_blocking=True)
        return d

    def device_buf(self, name: str, n: int, dtype) -> torch.Tensor:
        return self._grow(self.dev, name, n, dtype, False)

    def host_buf(self, name: str, n: int, dtype) -> torch.Tensor:
        return self._grow(self.host, name, n, dtype, True)

    def download(self, name: str, d: torch.Tensor, n: int, stream) -> torch.Tensor:
        h = self._grow(self.host, name, n, d.dtype, True)
        if n:
            with torch.cuda.stream(stream):
                h[:n].copy_(d[:n], non_blocking=True)
        return h


class ExtensionSession:
    """Repeated banded SW + traceback on host batches."""

    def __init__(self, device=None, match_score=2.0, mismatch_penalty=4.0, gap_open=6.0,
                 gap_extend=2.0, x_drop=0.0, traceback: bool = True,
                 stream: Optional[torch.cuda.Stream] = None, form: str = "batched"):
        self.device = require_cuda(device)
        self.form = form
        self.params = sw_params(match_score, mismatch_penalty, gap_open, gap_extend, x_drop)
        self.traceback = traceback
        self.stream = stream or torch.cuda.Stream(self.device)
        self.buf = _Buffers(self.device)
        self.h2d_bytes = 0
        self.d2h_bytes = 0

    def align(self, pairs: PairSet, order: Optional[np.ndarray] = None) -> SWResult:
        B = len(pairs)
        s = self.stream
        qlen = np.diff(pairs.query_off).astype(np.int32)
        tlen = np.diff(pairs.target_off).astype(np.int32)
        hb = np.asarray(pairs.half_band, np.int32)
        if B and (hb.min() < 0 or hb.max() > _native.MAX_HALF_BAND):
            raise ValueError(f"half_band must be within [0, {_native.MAX_HALF_BAND}]")
        if order is None and B:
            order = longest_first(qlen, hb)
        up = self.buf.upload
        q = up("q", pairs.query.astype(np.int8, copy=False), s)
        qo = up("qo", pairs.query_off.astype(np.int64, copy=False), s)
        t = up("t", pairs.target.astype(np.int8, copy=False), s)
        to = up("to", pairs.target_off.astype(np.int64, copy=False), s)
        hbd = up("hb", hb, s)
        off = up("off", np.asarray(pairs.band_offset, np.int32), s)
        od = up("order", np.asarray(order if order is not None else np.zeros(0), np.int32), s)
        self.h2d_bytes = int(pairs.query.size + pairs.target.size + 16 * (B + 1) + 12 * B)
        n = max(B, 1)
        cap = int(qlen.astype(np.int64).sum() + tlen.astype(np.int64).sum() + B) if self.traceback else 0
        db = self.buf.device_buf
        out = {k: db(k, n, torch.int32) for k in ("score", "qe", "te", "qs", "ts", "clen")}
        counts = db("counts", 4 * n, torch.int32)
        cstart = db("cstart", n, torch.int64)
        cigar = db("cigar", max(cap, 1), torch.int32)
        used = db("used", 1, torch.int64)
        err = db("err", 1, torch.int32)
        need = int(_native.lib().gmf_banded_sw_workspace_bytes(
            B, qlen.ctypes.data_as(ctypes.c_void_p), tlen.ctypes.data_as(ctypes.c_void_p),
            hb.ctypes.data_as(ctypes.c_void_p), 1 if self.traceback else 0))
        ws = db("ws", need, torch.uint8)
        goff = pairs.xdrop_group_off
        gd = up("goff", np.asarray(goff, np.int32), s) if goff is not None else None
        pairs_c = _native.GmfPairs(B, q.data_ptr(), qo.data_ptr(), t.data_ptr(), to.data_ptr(),
                                   hbd.data_ptr(), off.data_ptr(), od.data_ptr() if B else None,
                                   int(hb.max()) if B else 0, gd.data_ptr() if gd is not None else None,
                                   len(goff) - 1 if goff is not None else 0)
        tb = self.traceback
        res_c = _native.GmfSwResults(
            out["score"].data_ptr(), out["qe"].data_ptr(), out["te"].data_ptr(),
            out["qs"].data_ptr() if tb else None, out["ts"].data_ptr() if tb else None,
            counts.data_ptr() if tb else None, cigar.data_ptr() if tb else None,
            cigar.numel() if tb else 0, cstart.data_ptr() if tb else None,
            out["clen"].data_ptr() if tb else None, used.data_ptr(), err.data_ptr())
        sp = int(s.cuda_stream)
        bind(self.device, sp)
        fn = _native.lib().gmf_banded_sw if self.form == "batched" else _native.lib().gmf_banded_sw_plain
        st = fn(ctypes.byref(pairs_c), ctypes.byref(self.params), ctypes.byref(res_c),
                ctypes.c_void_p(ws.data_ptr()), ws.numel(), ctypes.c_void_p(sp))
        _native.check("gmf_banded_sw", st)
        dl = self.buf.download
        names = ["score", "qe", "te"] + (["qs", "ts", "clen"] if tb else [])
        host = {k: dl("h_" + k, out[k], B, s) for k in names}
        h_used = dl("h_used", used, 1, s)
        h_err = dl("h_err", err, 1, s)
        if tb:
            h_counts = dl("h_counts", counts, 4 * B, s)
            h_cstart = dl("h_cstart", cstart, B, s)
        s.synchronize()
        res = SWResult(host["score"][:B].numpy().copy(), host["qe"][:B].numpy().copy(),
                       host["te"][:B].numpy().copy(), error_flags=int(h_err[0]))
        nbytes = 12 * B + 12
        if tb:
            nu = int(h_used[0])
            h_cig = dl("h_cigar", cigar, nu, s)
            s.synchronize()
            res.query_start = host["qs"][:B].numpy().copy()
            res.target_start = host["ts"][:B].numpy().copy()
            res.cigar_len = host["clen"][:B].numpy().copy()
            res.op_counts = h_counts[: 4 * B].numpy().reshape(B, 4).copy()
            res.cigar_start = h_cstart[:B].numpy().copy()
            res.cigar_words = h_cig[:nu].numpy().view(np.uint32).copy()
            nbytes += 36 * B + 4 * nu
        self.d2h_bytes = nbytes
        res.d2h_bytes = nbytes
        if res.error_flags:
            raise RuntimeError(f"gmf_banded_sw reported error flags {res.error_flags}")
        return res


def run_cuts(read_off: np.ndarray, chunks: Optional[int] = None) -> np.ndarray:
    """Read boundaries of the runs a chain batch goes through: run k covers
    reads [cut[k], cut[k+1]), about A / C anchors each, no run empty (a batch
    without reads is one empty run).  ``chunks`` = C; by default two runs
    from 4 M anchors on, else one.  A run's launch lasts at least as long as
    its longest reads, so more runs add launch tails faster than they hide
    copies (on a B200 the 5,000-read HiFi batch takes 9.5, 8.3, 9.6 and
    14.5 ms end to end in 1, 2, 4 and 8 runs)."""
    read_off = np.asarray(read_off, np.int64)
    R, A = len(read_off) - 1, int(read_off[-1])
    if R <= 0:
        return np.array([0, 0], np.int64)
    C = chunks if chunks is not None else min(2, max(1, A // 2_000_000))
    C = max(1, min(int(C), R))
    inner = np.searchsorted(read_off, np.linspace(0, A, C + 1)[1:-1], side="left")
    return np.unique(np.concatenate([[0], np.clip(inner, 0, R), [R]])).astype(np.int64)


def _is_pinned(a: np.ndarray) -> bool:
    """True when the array's memory is page-locked (asynchronous copies can
    read it directly)."""
    return a.size > 0 and a.flags.c_contiguous and torch.from_numpy(a).is_pinned()


def pin_anchors(batch) -> AnchorCSR:
    """A copy of an anchor batch whose columns live in page-locked host
    memory: ChainSession.chain copies such columns straight to the device,
    with no staging copy on the host."""
    a = AnchorCSR.of(batch)

    def pin(x, dt):
        t = torch.empty(max(len(x), 1), dtype=dt, pin_memory=True)
        t[: len(x)].copy_(torch.from_numpy(np.ascontiguousarray(x)))
        return t.numpy()[: len(x)]

    return AnchorCSR(a.read_off.copy(), pin(a.read_pos, torch.int32), pin(a.ref_pos, torch.int32),
                     pin(a.length, torch.int32), pin(a.strand, torch.int8))


class ChainSession:
    """Repeated fast-mode chaining (sort, DP, peel, select) on host batches.
    Columns already in page-locked memory (see :func:`pin_anchors`) are
    copied to the device directly; the results come back into page-locked
    arrays that the returned ChainResult owns."""

    def __init__(self, cfg: Optional[ChainingConfig] = None, device=None,
                 stream: Optional[torch.cuda.Stream] = None):
        self.cfg = cfg or ChainingConfig()
        self.device = require_cuda(device)
        self.stream = stream or torch.cuda.Stream(self.device)
        self.buf = _Buffers(self.device)
        self.cp = chain_params(self.cfg)
        self.lut = LUTS.get(self.device, self.cfg.max_gap, self.cfg.gap_open, self.cfg.gap_extend,
                            self.cfg.log_coeff)
        self.h2d_bytes = 0
        self.d2h_bytes = 0
        # copies in and out run on streams of their own, beside the kernels
        self.copy_in = torch.cuda.Stream(self.device)
        self.copy_out = torch.cuda.Stream(self.device)
        self._events: list = []

    def chain(self, batch, chunks: Optional[int] = None) -> ChainResult:
        """Chain a host batch.  Large batches go through in ``chunks`` runs of
        whole reads (default: two from 4 M anchors on, see run_cuts): run k+1's
        inputs go to the device while run k chains on the session stream,
        and run k's chains come back while run k+1 chains.  Reads are chained
        independently, so the result does not depend on the split."""
        a = AnchorCSR.of(batch)
        R, A = len(a), int(a.read_off[-1])
        if R and np.diff(a.read_off).max() > _native.MAX_READ_ANCHORS:
            raise ValueError(f"a read has more than {_native.MAX_READ_ANCHORS} anchors")
        cut = run_cuts(a.read_off, chunks)
        C = len(cut) - 1
        s = self.stream
        mc = self.cp.max_chains
        hb, db = self.buf.host_buf, self.buf.device_buf
        nR, nA = max(R, 1), max(A, 1)
        inputs = dict(rp=(a.read_pos, torch.int32), fp=(a.ref_pos, torch.int32), ln=(a.length, torch.int32),
                      st=(a.strand, torch.int8))
        direct = {k: _is_pinned(np.asarray(arr)) for k, (arr, _) in inputs.items()}
        h_in = {k: hb(k, nA, dt) for k, (_, dt) in inputs.items() if not direct[k]}
        d_in = {k: db(k, nA, dt) for k, (_, dt) in inputs.items()}
        h_ro, d_ro = hb("ro", nR + C, torch.int64), db("ro", nR + C, torch.int64)
        sizes = dict(n=(1, torch.int32), score=(mc, torch.float64), strand=(mc, torch.int32),
                     span=(4 * mc, torch.int32), prim=(mc, torch.int32), nmem=(mc, torch.int32))
        d_out = {k: db(k, nR * w, dt) for k, (w, dt) in sizes.items()}
        # results land in page-locked arrays of their own, which the ChainResult keeps
        h_out = {k: torch.empty(nR * w, dtype=dt, pin_memory=True) for k, (w, dt) in sizes.items()}
        d_mem, h_mem = db("mem", nA, torch.int32), torch.empty(nA, dtype=torch.int32, pin_memory=True)
        widest_r = int(np.diff(cut).max()) if R else 0
        widest_a = int(max(a.read_off[cut[k + 1]] - a.read_off[cut[k]] for k in range(C))) if R else 0
        need = int(_native.lib().gmf_chain_workspace_bytes(widest_r, widest_a))
        ws = db("ws", max(need, 1), torch.uint8)
        sp = int(s.cuda_stream)
        bind(self.device, sp)
        while len(self._events) < C:
            self._events.append((torch.cuda.Event(), torch.cuda.Event(), torch.cuda.Event()))
        cin, cout = self.copy_in, self.copy_out
        cin.wait_stream(s)  # the previous call's kernels are done with the input buffers
        out = {k: h_out[k].numpy()[: R * w] for k, (w, _) in sizes.items()}
        members = h_mem.numpy()[:A]
        h2d = 0

        def stage(k):
            nonlocal h2d
            ev_in, ev_done, ev_out = self._events[k]
            r0, r1 = int(cut[k]), int(cut[k + 1])
            a0, a1 = int(a.read_off[r0]), int(a.read_off[r1])
            ro = h_ro[r0 + k: r1 + k + 1]
            ro.copy_(torch.from_numpy(a.read_off[r0: r1 + 1] - a0))
            with torch.cuda.stream(cin):
                d_ro[r0 + k: r1 + k + 1].copy_(ro, non_blocking=True)
            h2d += ro.numel() * 8
            for name, (arr, _) in inputs.items():
                if a1 > a0:
                    if direct[name]:
                        src = torch.from_numpy(arr[a0:a1])
                    else:
                        src = h_in[name][a0:a1]
                        src.copy_(torch.from_numpy(arr[a0:a1]))
                    with torch.cuda.stream(cin):
                        d_in[name][a0:a1].copy_(src, non_blocking=True)
                    h2d += (a1 - a0) * arr.itemsize
            ev_in.record(cin)
            s.wait_event(ev_in)
            batch_c = _native.GmfAnchorBatch(
                r1 - r0, d_ro.data_ptr() + 8 * (r0 + k), d_in["rp"].data_ptr() + 4 * a0,
                d_in["fp"].data_ptr() + 4 * a0, d_in["ln"].data_ptr() + 4 * a0, d_in["st"].data_ptr() + a0)
            o = {name: d_out[name].data_ptr() + d_out[name].element_size() * w * r0
                 for name, (w, _) in sizes.items()}
            res_c = _native.GmfChainResults(o["n"], o["score"], o["strand"], o["span"], o["prim"], o["nmem"],
                                            d_mem.data_ptr() + 4 * a0)
            rc = _native.lib().gmf_chain_batch(ctypes.byref(batch_c), ctypes.byref(self.cp),
                                               ctypes.c_void_p(self.lut.data_ptr()), self.lut.numel(), None,
                                               None, None, ctypes.byref(res_c), ctypes.c_void_p(ws.data_ptr()),
                                               need, ctypes.c_void_p(sp))
            _native.check("gmf_chain_batch", rc)
            ev_done.record(s)
            cout.wait_event(ev_done)
            with torch.cuda.stream(cout):
                for name, (w, _) in sizes.items():
                    h_out[name][w * r0: w * r1].copy_(d_out[name][w * r0: w * r1], non_blocking=True)
                h_mem[a0:a1].copy_(d_mem[a0:a1], non_blocking=True)
            ev_out.record(cout)

        # every run is enqueued at once; the results of a run are in place once
        # its copies out have finished
        for k in range(C):
            stage(k)
        for k in range(C):
            self._events[k][2].synchronize()
        s.wait_stream(cout)  # the next call's kernels follow these copies out
        self.h2d_bytes = h2d
        self.d2h_bytes = int(R * sum(w * torch.tensor([], dtype=dt).element_size() for w, dt in sizes.values())
                             + A * 4)
        return ChainResult(a.read_off, out["n"], out["score"].reshape(R, mc), out["strand"].reshape(R, mc),
                           out["span"].reshape(R, mc, 4), out["prim"].reshape(R, mc),
                           out["nmem"].reshape(R, mc), members, self.d2h_bytes)
