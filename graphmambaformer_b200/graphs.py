"""Banded SW replayed from a captured CUDA graph.

One ``gmf_banded_sw`` call enqueues three memsets, the device classifier, up
to seven class kernels forked onto side streams and joined back, and the
traceback walk.  For a stream of small batches (a serving loop) the launch
overhead of that sequence is comparable to the work, so
:class:`GraphedAligner` keeps fixed-capacity device and pinned host buffers,
pads every batch to the capacity with empty pairs (which the kernels finish
at once), and replays one captured graph per batch: the host-to-device
copies of the inputs, the whole call, and the device-to-host copies of the
fixed-size results.  Only the CIGAR words, whose count varies, are copied
after the replay.  The graph is captured again only when a batch needs a
larger workspace than the one it was captured with.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _native
from .device import bind, require_cuda
from .extension import SWResult, longest_first
from .synth import PairSet


class GraphedAligner:
    def __init__(self, device, params: _native.GmfSwParams, cap_pairs: int, cap_query: int, cap_target: int,
                 max_half_band: int, traceback: bool = True):
        if not 0 <= max_half_band <= _native.MAX_HALF_BAND:
            raise ValueError(f"max_half_band must be within [0, {_native.MAX_HALF_BAND}]")
        self.device = require_cuda(device)
        self.params = params
        self.cap_pairs, self.cap_query, self.cap_target = int(cap_pairs), int(cap_query), int(cap_target)
        self.max_hb = int(max_half_band)
        self.traceback = traceback
        self.stream = torch.cuda.Stream(self.device)
        dev, P = self.device, self.cap_pairs
        pin = dict(pin_memory=True)

        def pair(n, dt):
            return torch.zeros(n, dtype=dt, **pin), torch.zeros(n, dtype=dt, device=dev)

        self.h_q, self.d_q = pair(max(self.cap_query, 1), torch.int8)
        self.h_t, self.d_t = pair(max(self.cap_target, 1), torch.int8)
        self.h_qo, self.d_qo = pair(P + 1, torch.int64)
        self.h_to, self.d_to = pair(P + 1, torch.int64)
        self.h_hb, self.d_hb = pair(P, torch.int32)
        self.h_off, self.d_off = pair(P, torch.int32)
        self.h_ord, self.d_ord = pair(P, torch.int32)
        # x-drop groups padded to P (trailing groups empty), so the captured count never changes
        self.h_go, self.d_go = pair(P + 1, torch.int32)
        i32 = dict(dtype=torch.int32, device=dev)
        self.o = {k: torch.zeros(P, **i32) for k in ("score", "qe", "te", "qs", "ts", "clen")}
        self.o["counts"] = torch.zeros(4 * P, **i32)
        self.o["cstart"] = torch.zeros(P, dtype=torch.int64, device=dev)
        self.o["used"] = torch.zeros(1, dtype=torch.int64, device=dev)
        self.o["err"] = torch.zeros(1, **i32)
        self.cig_cap = self.cap_query + self.cap_target + P
        self.cigar = torch.zeros(max(self.cig_cap, 1), dtype=torch.int32, device=dev)
        self.h_o = {k: torch.zeros(v.numel(), dtype=v.dtype, **pin) for k, v in self.o.items()}
        self.ws = torch.empty(256, dtype=torch.uint8, device=dev)
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        self.replays = 0
        self.captures = 0

    # -- staging ---------------------------------------------------------------
    def _stage(self, pairs: PairSet) -> tuple:
        n = len(pairs)
        qlen = np.diff(pairs.query_off).astype(np.int32)
        tlen = np.diff(pairs.target_off).astype(np.int32)
        hb = np.asarray(pairs.half_band, np.int32)
        if n > self.cap_pairs or int(pairs.query_off[-1]) > self.cap_query or \
                int(pairs.target_off[-1]) > self.cap_target:
            raise ValueError("batch exceeds the aligner's capacity")
        if n and (hb.min() < 0 or hb.max() > self.max_hb):
            raise ValueError(f"half_band must be within [0, {self.max_hb}]")
        P = self.cap_pairs
        qo = np.full(P + 1, pairs.query_off[-1], np.int64)
        qo[: n + 1] = pairs.query_off
        to = np.full(P + 1, pairs.target_off[-1], np.int64)
        to[: n + 1] = pairs.target_off
        hbp = np.zeros(P, np.int32)
        hbp[:n] = hb
        offp = np.zeros(P, np.int32)
        offp[:n] = np.asarray(pairs.band_offset, np.int32)
        order = np.arange(P, dtype=np.int32)
        if n:
            order[:n] = longest_first(qlen, hb)
        go = np.full(P + 1, n, np.int32)
        g = pairs.xdrop_group_off
        if g is None:
            go[: n + 1] = np.arange(n + 1, dtype=np.int32)
        else:
            g = np.asarray(g, np.int32)
            if len(g) - 1 > P or g[0] != 0 or g[-1] != n or np.any(np.diff(g) < 0):
                raise ValueError("xdrop_group_off must rise from 0 to the number of pairs")
            go[: len(g)] = g
        nq, nt = int(pairs.query_off[-1]), int(pairs.target_off[-1])
        if nq:
            self.h_q[:nq].numpy()[...] = pairs.query.astype(np.int8, copy=False)
        if nt:
            self.h_t[:nt].numpy()[...] = pairs.target.astype(np.int8, copy=False)
        self.h_qo.numpy()[...] = qo
        self.h_to.numpy()[...] = to
        self.h_hb.numpy()[...] = hbp
        self.h_off.numpy()[...] = offp
        self.h_ord.numpy()[...] = order
        self.h_go.numpy()[...] = go
        # workspace this batch needs (the padding pairs need none)
        need = int(_native.lib().gmf_banded_sw_workspace_bytes(
            P, np.ascontiguousarray(qo[1:] - qo[:-1], np.int32).ctypes.data_as(ctypes.c_void_p),
            np.ascontiguousarray(to[1:] - to[:-1], np.int32).ctypes.data_as(ctypes.c_void_p),
            hbp.ctypes.data_as(ctypes.c_void_p), 1 if self.traceback else 0))
        return n, need

    # -- the captured sequence -------------------------------------------------
    def _sequence(self) -> None:
        for h, d in ((self.h_q, self.d_q), (self.h_t, self.d_t), (self.h_qo, self.d_qo), (self.h_to, self.d_to),
                     (self.h_hb, self.d_hb), (self.h_off, self.d_off), (self.h_ord, self.d_ord),
                     (self.h_go, self.d_go)):
            d.copy_(h, non_blocking=True)
        o, tb = self.o, self.traceback
        pairs_c = _native.GmfPairs(self.cap_pairs, self.d_q.data_ptr(), self.d_qo.data_ptr(), self.d_t.data_ptr(),
                                   self.d_to.data_ptr(), self.d_hb.data_ptr(), self.d_off.data_ptr(),
                                   self.d_ord.data_ptr(), self.max_hb, self.d_go.data_ptr(), self.cap_pairs)
        res_c = _native.GmfSwResults(
            o["score"].data_ptr(), o["qe"].data_ptr(), o["te"].data_ptr(),
            o["qs"].data_ptr() if tb else None, o["ts"].data_ptr() if tb else None,
            o["counts"].data_ptr() if tb else None, self.cigar.data_ptr() if tb else None,
            self.cigar.numel() if tb else 0, o["cstart"].data_ptr() if tb else None,
            o["clen"].data_ptr() if tb else None, o["used"].data_ptr(), o["err"].data_ptr())
        sp = int(self.stream.cuda_stream)
        bind(self.device, sp)
        st = _native.lib().gmf_banded_sw(ctypes.byref(pairs_c), ctypes.byref(self.params), ctypes.byref(res_c),
                                         ctypes.c_void_p(self.ws.data_ptr()), self.ws.numel(), ctypes.c_void_p(sp))
        _native.check("gmf_banded_sw", st)
        for k, d in o.items():
            self.h_o[k].copy_(d, non_blocking=True)

    def _capture(self) -> None:
        # the library cannot ask a capturing stream for its device: select it
        _native.check("gmf_set_device", _native.lib().gmf_set_device(self.device.index))
        with torch.cuda.stream(self.stream):
            self._sequence()  # eager run: kernel images, side streams, function attributes
        self.stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream, capture_error_mode="thread_local"):
            self._sequence()
        self.graph = g
        self.captures += 1

    # -- public ----------------------------------------------------------------
    def align(self, pairs: PairSet) -> SWResult:
        n, need = self._stage(pairs)
        if need > self.ws.numel():
            self.ws = torch.empty(int(need * 1.25) + 256, dtype=torch.uint8, device=self.device)
            self.graph = None
        if self.graph is None:
            self._capture()
        with torch.cuda.stream(self.stream):  # replay() launches on the current stream
            self.graph.replay()
        self.replays += 1
        self.stream.synchronize()
        h = {k: v.numpy() for k, v in self.h_o.items()}
        res = SWResult(h["score"][:n].copy(), h["qe"][:n].copy(), h["te"][:n].copy(), error_flags=int(h["err"][0]))
        if self.traceback:
            used = int(h["used"][0])
            words = self.cigar[:used].to("cpu").numpy().view(np.uint32).copy() if used else np.zeros(0, np.uint32)
            res.query_start = h["qs"][:n].copy()
            res.target_start = h["ts"][:n].copy()
            res.op_counts = h["counts"][: 4 * n].reshape(n, 4).copy()
            res.cigar_start = h["cstart"][:n].copy()
            res.cigar_len = h["clen"][:n].copy()
            res.cigar_words = words
        if res.error_flags:
            raise RuntimeError(f"gmf_banded_sw reported error flags {res.error_flags}")
        return res
