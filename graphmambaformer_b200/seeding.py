"""Minimizer seeding on the device.

The index is the reference's (w, k) minimizer table (alignment/seeding.py
L524-538: pack_kmers, hash64, minimizer_mask, KmerTable.build with
max_occ), built once on the host by the same functions
(``synth.MinimizerSketch`` restates them) and kept on the device.  Reads are
seeded by ``gmf_seed_count`` / ``gmf_seed_fill``: both orientations, forward
anchors first, reverse-complement anchors in the reverse-complemented read's
coordinates -- what SeedingEngine.seed_read (L1056-1101) collects from
MinimizerIndex.query before merging diagonals.
"""

from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np
import torch

from . import _native
from .chaining import AnchorCSR
from .device import bind, require_cuda, to_device


class DeviceMinimizerIndex:
    def __init__(self, ref_codes: np.ndarray, k: int = 15, w: int = 10, max_occ: int = 0, device=None):
        from .synth import MinimizerSketch

        if not 1 <= k <= 31 or not 1 <= w <= 256:
            raise ValueError("k must be within [1, 31] and w within [1, 256]")
        self.device = require_cuda(device)
        self.k, self.w = int(k), int(w)
        sk = MinimizerSketch(np.asarray(ref_codes, np.int8), k=k, w=w, max_occ=max_occ)
        pad = lambda x, dt: x.astype(dt) if len(x) else np.zeros(1, dt)  # noqa: E731
        self.n_keys = len(sk.keys)
        self.keys = to_device(pad(sk.keys, np.int64), self.device)
        self.offsets = to_device(sk.offsets.astype(np.int64), self.device)
        self.positions = to_device(pad(sk.positions, np.int32), self.device)
        self.bytes = int(self.keys.numel() * 8 + self.offsets.numel() * 8 + self.positions.numel() * 4)

    def c(self) -> _native.GmfMinimizerIndex:
        return _native.GmfMinimizerIndex(self.k, self.w, self.n_keys, self.keys.data_ptr(), self.offsets.data_ptr(),
                                         self.positions.data_ptr())

    def seed_device(self, codes_d: torch.Tensor, read_off_d: torch.Tensor, n_reads: int, both_strands: bool = True,
                    stream: Optional[torch.cuda.Stream] = None) -> dict:
        """Seed reads already on the device (codes CSR).  Returns device
        tensors read_off (n_reads + 1, per read: forward then reverse
        anchors), read_pos, ref_pos, length, strand, the anchor count and the
        largest read's anchor count."""
        s = stream or torch.cuda.current_stream(self.device)
        sp = int(s.cuda_stream)
        bind(self.device, sp)
        idx = self.c()
        vp = ctypes.c_void_p
        # every allocation and torch op on the caller's stream: the library's
        # kernels run there, and a worker's stream is not ordered with the
        # thread's default stream
        with torch.cuda.stream(s):
            counts = torch.empty(max(2 * n_reads, 1), dtype=torch.int64, device=self.device)
            _native.check("gmf_seed_count", _native.lib().gmf_seed_count(
                ctypes.byref(idx), n_reads, vp(codes_d.data_ptr()), vp(read_off_d.data_ptr()),
                1 if both_strands else 0, vp(counts.data_ptr()), vp(sp)))
            aoff = torch.zeros(2 * n_reads + 1, dtype=torch.int64, device=self.device)
            if n_reads:
                torch.cumsum(counts[: 2 * n_reads], 0, out=aoff[1:])
            # the total sizes the outputs; the largest read is checked against the chaining limit (one
            # host round trip for both)
            per_read = (counts[0: 2 * n_reads: 2] + counts[1: 2 * n_reads: 2]).max() if n_reads else counts[0] * 0
            total, most = (int(x) for x in torch.stack([aoff[-1], per_read]).cpu().tolist())
            i32 = dict(dtype=torch.int32, device=self.device)
            out = dict(read_pos=torch.empty(max(total, 1), **i32), ref_pos=torch.empty(max(total, 1), **i32),
                       length=torch.empty(max(total, 1), **i32),
                       strand=torch.empty(max(total, 1), dtype=torch.int8, device=self.device))
            _native.check("gmf_seed_fill", _native.lib().gmf_seed_fill(
                ctypes.byref(idx), n_reads, vp(codes_d.data_ptr()), vp(read_off_d.data_ptr()),
                1 if both_strands else 0, vp(aoff.data_ptr()), vp(out["read_pos"].data_ptr()),
                vp(out["ref_pos"].data_ptr()), vp(out["length"].data_ptr()), vp(out["strand"].data_ptr()), vp(sp)))
            out["read_off"] = aoff[::2].contiguous()
        out["n_anchors"] = total
        out["max_read_anchors"] = most
        return out

    def seed(self, reads: Sequence[np.ndarray], both_strands: bool = True) -> AnchorCSR:
        """Host reads in, host anchors (CSR, per read forward then reverse) out."""
        n = len(reads)
        off = np.zeros(n + 1, np.int64)
        np.cumsum([len(r) for r in reads], out=off[1:])
        codes = np.concatenate([np.asarray(r, np.int8) for r in reads]) if off[-1] else np.zeros(1, np.int8)
        d = self.seed_device(to_device(codes, self.device), to_device(off, self.device), n, both_strands)
        torch.cuda.synchronize(self.device)
        t = d["n_anchors"]
        return AnchorCSR(d["read_off"].cpu().numpy(), d["read_pos"][:t].cpu().numpy(), d["ref_pos"][:t].cpu().numpy(),
                         d["length"][:t].cpu().numpy(), d["strand"][:t].cpu().numpy())
