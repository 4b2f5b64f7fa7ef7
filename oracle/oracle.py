"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle restates the reference's CPU algorithms for the alignment hot path
(see ``gmf_oracle.c`` for the line-by-line citations).  Only the test suite,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use it, as
the checker; the shipped library never calls it.

Parity pin: ``tests/test_oracle_golden.py`` checks every function here against
golden vectors produced by the reference itself (``tests/golden``).
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import build_oracle

_lib: Optional[ctypes.CDLL] = None

OPS = "=XIDS"


class SWParams(ctypes.Structure):
    _fields_ = [
        ("match", ctypes.c_float),
        ("mismatch", ctypes.c_float),
        ("gap_open", ctypes.c_float),
        ("gap_extend", ctypes.c_float),
        ("x_drop", ctypes.c_float),
    ]


class ChainParams(ctypes.Structure):
    _fields_ = [
        ("max_lookback", ctypes.c_int32),
        ("max_gap", ctypes.c_int64),
        ("min_chain_anchors", ctypes.c_int64),
        ("min_chain_score", ctypes.c_double),
        ("max_chains", ctypes.c_int64),
        ("secondary_overlap", ctypes.c_double),
        ("secondary_score_ratio", ctypes.c_double),
    ]


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = build_oracle.LIB
        if not os.path.exists(path):
            build_oracle.build()
        _lib = ctypes.CDLL(path)
        _lib.oracle_wfa_align.restype = ctypes.c_int64
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def penalty_lut(max_gap: int, gap_open: float, gap_extend: float, log_coeff: float) -> np.ndarray:
    """``_penalty`` of chaining.py L120-126 tabulated for gaps ``0..max_gap``.

    numpy evaluates it element-wise with the same expression, so entry ``g``
    is bit-identical to what the reference computes for a gap of ``g``.
    """
    gap = np.arange(int(max_gap) + 1, dtype=np.int64)
    return np.where(gap > 0, gap_open + gap_extend * gap + log_coeff * np.log2(gap + 1.0), 0.0)


# --------------------------------------------------------------------------- #
# Banded SW + traceback
# --------------------------------------------------------------------------- #
@dataclass
class SWOut:
    score: np.ndarray  # float32 (B,)
    query_end: np.ndarray  # int64 (B,)
    target_end: np.ndarray
    query_start: np.ndarray
    target_start: np.ndarray
    cigars: list  # list of [(op, n), ...]
    counts: np.ndarray  # (B, 4) = X I D


def _ragged(seqs: Sequence[np.ndarray]) -> tuple[np.ndarray, np.ndarray]:
    lens = np.array([len(s) for s in seqs], dtype=np.int64)
    off = np.zeros(len(seqs) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    flat = (np.concatenate([np.asarray(s, dtype=np.int16) for s in seqs])
            if len(seqs) and off[-1] > 0 else np.zeros(1, dtype=np.int16))
    return np.ascontiguousarray(flat, dtype=np.int16), off


def sw_batch(
    queries: Sequence[np.ndarray],
    targets: Sequence[np.ndarray],
    half_band: Sequence[int] | int,
    band_offset: Sequence[int] | int,
    match: float = 2.0,
    mismatch: float = 4.0,
    gap_open: float = 6.0,
    gap_extend: float = 2.0,
    x_drop: float = 600.0,
    traceback: bool = True,
    threads: int = 1,
    group_off: Optional[Sequence[int]] = None,
) -> SWOut:
    """``banded_affine_sw_batch`` + ``traceback_banded``: per pair (B=1), or,
    with ``group_off``, one reference batch per group of consecutive pairs
    (pairs group_off[g] .. group_off[g+1]-1), whose x-drop stop is shared."""
    B = len(queries)
    hb = np.broadcast_to(np.asarray(half_band, dtype=np.int32), (B,)).copy()
    off = np.broadcast_to(np.asarray(band_offset, dtype=np.int32), (B,)).copy()
    q, q_off = _ragged(queries)
    t, t_off = _ragged(targets)
    cap = (q_off[1:] - q_off[:-1]) + (t_off[1:] - t_off[:-1]) + 1
    c_off = np.zeros(B + 1, dtype=np.int64)
    np.cumsum(cap, out=c_off[1:])
    cigar = np.zeros(max(int(c_off[-1]), 1), dtype=np.uint32)
    score = np.zeros(B, dtype=np.float32)
    qe = np.zeros(B, dtype=np.int64)
    te = np.zeros(B, dtype=np.int64)
    qs = np.zeros(B, dtype=np.int64)
    ts = np.zeros(B, dtype=np.int64)
    cn = np.zeros(B, dtype=np.int32)
    counts = np.zeros((B, 4), dtype=np.int32)
    params = SWParams(match, mismatch, gap_open, gap_extend, x_drop)
    g_off = None
    if group_off is not None:
        g_off = np.ascontiguousarray(group_off, dtype=np.int64)
        if len(g_off) < 1 or g_off[0] != 0 or g_off[-1] != B or np.any(np.diff(g_off) < 0):
            raise ValueError("group_off must rise from 0 to the number of pairs")
    status = lib().oracle_sw_batch(
        ctypes.c_int32(B), _p(q), _p(q_off), _p(t), _p(t_off), _p(hb), _p(off),
        ctypes.byref(params), ctypes.c_int32(1 if traceback else 0), ctypes.c_int32(threads),
        _p(score), _p(qe), _p(te), _p(qs), _p(ts), _p(cigar), _p(c_off), _p(cn), _p(counts),
        None if g_off is None else _p(g_off), ctypes.c_int32(0 if g_off is None else len(g_off) - 1),
    )
    if status != 0:
        raise MemoryError("oracle_sw_batch could not allocate its DP matrices")
    cigars = []
    for b in range(B):
        words = cigar[c_off[b]: c_off[b] + cn[b]]
        cigars.append([(OPS[int(w) & 15], int(w) >> 4) for w in words])
    return SWOut(score, qe, te, qs, ts, cigars, counts)


def sw_matrices(query: np.ndarray, target: np.ndarray, half_band: int, band_offset: int,
                match=2.0, mismatch=4.0, gap_open=6.0, gap_extend=2.0, x_drop=600.0):
    """Full H/E/F matrices of one pair, as the reference stores them."""
    q = np.ascontiguousarray(query, dtype=np.int16)
    t = np.ascontiguousarray(target, dtype=np.int16)
    W = 2 * half_band + 1
    rows = len(q) + 1
    H = np.zeros((rows, W), dtype=np.float32)
    E = np.zeros((rows, W), dtype=np.float32)
    F = np.zeros((rows, W), dtype=np.float32)
    sc = ctypes.c_float()
    qe = ctypes.c_int64()
    te = ctypes.c_int64()
    params = SWParams(match, mismatch, gap_open, gap_extend, x_drop)
    lib().oracle_sw_pair(
        _p(q if len(q) else np.zeros(1, np.int16)), ctypes.c_int32(len(q)),
        _p(t if len(t) else np.zeros(1, np.int16)), ctypes.c_int32(len(t)),
        ctypes.c_int32(half_band), ctypes.c_int32(band_offset), ctypes.byref(params),
        _p(H), _p(E), _p(F), ctypes.byref(sc), ctypes.byref(qe), ctypes.byref(te))
    return H, E, F, float(sc.value), int(qe.value), int(te.value)


# --------------------------------------------------------------------------- #
# Chaining
# --------------------------------------------------------------------------- #
def chain_dp(read_end, ref_end, weight, lut: np.ndarray, max_lookback: int = 64,
             max_gap: int = 5000, bonus: Optional[np.ndarray] = None):
    """``chain_dp_numpy`` (chaining.py L129-180) -> ``(f float64, parent int64)``."""
    re = np.ascontiguousarray(read_end, dtype=np.int64)
    fe = np.ascontiguousarray(ref_end, dtype=np.int64)
    w = np.ascontiguousarray(weight, dtype=np.float64)
    n = len(re)
    f = np.zeros(max(n, 1), dtype=np.float64)
    parent = np.full(max(n, 1), -1, dtype=np.int64)
    lut = np.ascontiguousarray(lut, dtype=np.float64)
    bptr = None
    if bonus is not None:
        bonus = np.ascontiguousarray(bonus, dtype=np.float64)
        bptr = _p(bonus)
    if n:
        lib().oracle_chain_dp(
            ctypes.c_int64(n), _p(re), _p(fe), _p(w), bptr, ctypes.c_int32(max_lookback),
            ctypes.c_int64(max_gap), _p(lut), ctypes.c_int64(len(lut)), _p(f), _p(parent))
    return f[:n], parent[:n]


def chain_backtrack(f, parent, read_pos, read_end, ref_pos, ref_end, global_idx, strand: int,
                    min_chain_anchors: int = 1, min_chain_score: float = 20.0):
    """``_backtrack`` (chaining.py L530-576) -> list of chain dicts (pre-select)."""
    n = len(f)
    arr = [np.ascontiguousarray(a, dtype=np.int64)
           for a in (parent, read_pos, read_end, ref_pos, ref_end, global_idx)]
    f = np.ascontiguousarray(f, dtype=np.float64)
    m = max(n, 1)
    score = np.zeros(m, np.float64)
    span = np.zeros((m, 4), np.int64)
    moff = np.zeros(m, np.int64)
    nmem = np.zeros(m, np.int64)
    nch = ctypes.c_int64()
    members = np.zeros(m, np.int64)
    lib().oracle_chain_backtrack(
        ctypes.c_int64(n), _p(f), *[_p(a) for a in arr], ctypes.c_int32(strand),
        ctypes.c_int64(min_chain_anchors), ctypes.c_double(min_chain_score), _p(score),
        _p(span), _p(moff), _p(nmem), ctypes.byref(nch), _p(members))
    out = []
    for k in range(nch.value):
        out.append(dict(score=float(score[k]), strand=strand,
                        read_start=int(span[k, 0]), read_end=int(span[k, 1]),
                        ref_start=int(span[k, 2]), ref_end=int(span[k, 3]),
                        anchor_idx=members[moff[k]: moff[k] + nmem[k]].copy()))
    return out


@dataclass
class ChainBatchOut:
    n_chains: np.ndarray  # (R,)
    score: np.ndarray  # (R, max_chains)
    strand: np.ndarray
    span: np.ndarray  # (R, max_chains, 4) read_start, read_end, ref_start, ref_end
    primary: np.ndarray
    n_members: np.ndarray
    members: np.ndarray  # per read: kept chains' anchor indices back to back

    def chains(self, read_off: np.ndarray, r: int) -> list[dict]:
        out, pos = [], int(read_off[r])
        for k in range(int(self.n_chains[r])):
            m = int(self.n_members[r, k])
            out.append(dict(
                score=float(self.score[r, k]), strand=int(self.strand[r, k]),
                read_start=int(self.span[r, k, 0]), read_end=int(self.span[r, k, 1]),
                ref_start=int(self.span[r, k, 2]), ref_end=int(self.span[r, k, 3]),
                is_primary=bool(self.primary[r, k]),
                anchor_idx=self.members[pos: pos + m].copy()))
            pos += m
        return out


def chain_batch(read_off, read_pos, ref_pos, length, strand, lut, max_lookback=64,
                max_gap=5000, min_chain_anchors=1, min_chain_score=20.0, max_chains=8,
                secondary_overlap=0.5, secondary_score_ratio=0.6, threads=1) -> ChainBatchOut:
    """``AffineChainer.chain`` (fast mode) for a batch of reads in CSR layout."""
    read_off = np.ascontiguousarray(read_off, dtype=np.int64)
    R = len(read_off) - 1
    cols = [np.ascontiguousarray(a, dtype=np.int64) for a in (read_pos, ref_pos, length)]
    st = np.ascontiguousarray(strand, dtype=np.int8)
    total = max(int(read_off[-1]), 1)
    if len(cols[0]) == 0:
        cols = [np.zeros(1, np.int64)] * 3
        st = np.zeros(1, np.int8)
    mc = int(max_chains)
    out = ChainBatchOut(
        n_chains=np.zeros(R, np.int32), score=np.zeros((R, mc), np.float64),
        strand=np.zeros((R, mc), np.int32), span=np.zeros((R, mc, 4), np.int64),
        primary=np.zeros((R, mc), np.int32), n_members=np.zeros((R, mc), np.int64),
        members=np.zeros(total, np.int64))
    cp = ChainParams(max_lookback, max_gap, min_chain_anchors, min_chain_score, mc,
                     secondary_overlap, secondary_score_ratio)
    lut = np.ascontiguousarray(lut, dtype=np.float64)
    lib().oracle_chain_batch(
        ctypes.c_int64(R), _p(read_off), *[_p(a) for a in cols], _p(st), ctypes.byref(cp),
        _p(lut), ctypes.c_int64(len(lut)), ctypes.c_int32(threads), _p(out.score),
        _p(out.strand), _p(out.span), _p(out.primary), _p(out.n_members), _p(out.members),
        _p(out.n_chains))
    return out


def wfa_align(query: np.ndarray, target: np.ndarray, max_distance: int) -> tuple[int, list]:
    """WavefrontAligner.align (extension.py L353-463): (edit distance, CIGAR
    runs); distance -1 when it exceeds ``max_distance`` (where the reference
    raises RuntimeError)."""
    q = np.ascontiguousarray(query, np.int16)
    t = np.ascontiguousarray(target, np.int16)
    words = np.zeros(len(q) + len(t) + 2, np.uint32)
    nw = ctypes.c_int64(0)
    d = lib().oracle_wfa_align(_p(q), ctypes.c_int64(len(q)), _p(t), ctypes.c_int64(len(t)),
                               ctypes.c_int64(int(max_distance)), _p(words), ctypes.byref(nw))
    if d == -2:
        raise MemoryError("oracle_wfa_align: out of memory")
    if d < 0:
        return -1, []
    return int(d), [(OPS[w & 15], int(w >> 4)) for w in words[: nw.value]]
