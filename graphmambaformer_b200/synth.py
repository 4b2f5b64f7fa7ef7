"""Seeded synthetic workloads for the alignment hot path.

No public dataset is involved: every workload is generated from
``np.random.default_rng(seed)`` with the shapes, sizes and error processes of
the reference's synthetic simulator.  The per-base edit process follows
``graphmambaformer/data/synthetic.py`` L470-580 (insertions drawn before each
template base, then deletion / substitution / match), written here in
vectorised numpy.

Workloads:

* ``extension_pairs_150bp`` -- 10,000 read/target pairs from a uniform-ACGT
  1 Mb reference; reads are 150 bp windows with 1% substitutions and 0.1%
  indels, targets are the true window +-32 bp, half band 32, band offset 32.
* ``chaining_reads_hifi`` -- 5,000 HiFi-like reads (15 kb +-20%, 0.1% error,
  random strand) on a uniform 10 Mb reference; anchors are raw (k=15, w=10)
  minimizer hits of both read orientations.
* ``extension_pairs_mixed`` -- pairs with log-normal lengths clipped to
  [150, 20000] bp, one third each Illumina-like (1% sub), HiFi-like (0.1%
  mixed) and ONT-like (5% error, 60% of it indels); half band
  ``clip(32 + band_slope * len, 32, 500)``.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

A, C, G, T, N = 1, 2, 3, 4, 5
_COMPLEMENT = np.array([0, 4, 3, 2, 1, 5], dtype=np.int8)
_ENCODE = np.full(256, N, dtype=np.int8)
for _b, _c in zip("ACGT", (A, C, G, T)):
    _ENCODE[ord(_b)] = _c
    _ENCODE[ord(_b.lower())] = _c


def encode_bases(seq: str) -> np.ndarray:
    """ASCII -> int8 codes A=1 C=2 G=3 T=4, anything else N=5
    (the alphabet of graphmambaformer/alignment/seeding.py L44-69)."""
    if not seq:
        return np.zeros(0, dtype=np.int8)
    return _ENCODE[np.frombuffer(seq.encode("ascii", errors="replace"), dtype=np.uint8)]


def decode_bases(codes: np.ndarray) -> str:
    lut = np.frombuffer(b"$ACGTN", dtype=np.uint8)
    return lut[np.clip(np.asarray(codes), 0, 5)].tobytes().decode("ascii")


def reverse_complement(codes: np.ndarray) -> np.ndarray:
    """Reverse complement of int8 codes (seeding.py L78-80 convention)."""
    return _COMPLEMENT[np.asarray(codes)[::-1]]


def random_reference(length: int, rng: np.random.Generator) -> np.ndarray:
    return rng.integers(1, 5, size=int(length), dtype=np.int8)


@dataclass
class ErrorProfile:
    p_sub: float
    p_ins: float
    p_del: float


ILLUMINA = ErrorProfile(0.01, 0.0, 0.0)
HIFI = ErrorProfile(0.0004, 0.0003, 0.0003)
# 5% total error, 60% of it indels (split evenly between insertions and deletions)
ONT = ErrorProfile(0.02, 0.015, 0.015)
# the 150 bp extension workload: 1% substitutions, 0.1% indels of length 1
SHORT_READ = ErrorProfile(0.01, 0.0005, 0.0005)


def apply_errors(template: np.ndarray, prof: ErrorProfile, rng: np.random.Generator) -> np.ndarray:
    """Per-base edit process: optional insertions before each template base,
    then deletion / substitution / match, plus trailing insertions."""
    n = len(template)
    if n == 0:
        return template.copy()
    r = rng.random(n)
    deleted = r < prof.p_del
    subst = (~deleted) & (r < prof.p_del + prof.p_sub)
    out_base = template.copy()
    if subst.any():
        shift = rng.integers(1, 4, size=int(subst.sum()), dtype=np.int8)
        # a different base: rotate the code by 1..3 within 1..4
        out_base[subst] = ((template[subst] - 1 + shift) % 4) + 1
    # insertions before each base (geometric count with parameter p_ins)
    if prof.p_ins > 0:
        n_ins = rng.geometric(1.0 - prof.p_ins, size=n + 1) - 1
    else:
        n_ins = np.zeros(n + 1, dtype=np.int64)
    keep = ~deleted
    counts = n_ins[:n] + keep.astype(np.int64)
    total = int(counts.sum() + n_ins[n])
    out = np.empty(total, dtype=np.int8)
    # positions of the kept template bases in the output
    ends = np.cumsum(counts)
    kept_pos = ends[keep] - 1
    out[kept_pos] = out_base[keep]
    mask = np.ones(total, dtype=bool)
    mask[kept_pos] = False
    n_new = int(mask.sum())
    if n_new:
        out[mask] = rng.integers(1, 5, size=n_new, dtype=np.int8)
    return out


# --------------------------------------------------------------------------- #
# Extension pairs
# --------------------------------------------------------------------------- #
@dataclass
class PairSet:
    """Ragged read/target pairs with per-pair band geometry (CSR layout)."""

    query: np.ndarray  # int8 codes, concatenated
    query_off: np.ndarray  # int64 (B+1,)
    target: np.ndarray
    target_off: np.ndarray
    half_band: np.ndarray  # int32 (B,)
    band_offset: np.ndarray  # int32 (B,)
    profile: Optional[np.ndarray] = None  # int8 per pair (0 illumina, 1 hifi, 2 ont)
    meta: dict = field(default_factory=dict)
    # x-drop groups: pairs [off[g], off[g+1]) stop together (the reference's
    # batch rule, e.g. the chains of one read); None = each pair alone
    xdrop_group_off: Optional[np.ndarray] = None

    def __len__(self) -> int:
        return len(self.half_band)

    @property
    def query_len(self) -> np.ndarray:
        return np.diff(self.query_off).astype(np.int32)

    @property
    def target_len(self) -> np.ndarray:
        return np.diff(self.target_off).astype(np.int32)

    def q(self, b: int) -> np.ndarray:
        return self.query[self.query_off[b]: self.query_off[b + 1]]

    def t(self, b: int) -> np.ndarray:
        return self.target[self.target_off[b]: self.target_off[b + 1]]

    def subset(self, idx) -> "PairSet":
        idx = np.asarray(idx, dtype=np.int64)
        qs = [self.q(int(b)) for b in idx]
        ts = [self.t(int(b)) for b in idx]
        return PairSet.from_lists(qs, ts, self.half_band[idx], self.band_offset[idx],
                                  None if self.profile is None else self.profile[idx], self.meta)

    def cells(self) -> int:
        """In-band valid DP cells: sum over pairs of #{(i, d): 1<=i<=qlen,
        0<=d<W, 1 <= i + off - hb + d <= tlen}."""
        return int(band_cells(self.query_len, self.target_len, self.half_band,
                              self.band_offset).sum())

    @staticmethod
    def from_lists(queries, targets, half_band, band_offset, profile=None, meta=None) -> "PairSet":
        ql = np.array([len(x) for x in queries], dtype=np.int64)
        tl = np.array([len(x) for x in targets], dtype=np.int64)
        qo = np.zeros(len(ql) + 1, dtype=np.int64)
        to = np.zeros(len(tl) + 1, dtype=np.int64)
        np.cumsum(ql, out=qo[1:])
        np.cumsum(tl, out=to[1:])
        qq = np.concatenate(queries).astype(np.int8) if len(queries) and qo[-1] else np.zeros(0, np.int8)
        tt = np.concatenate(targets).astype(np.int8) if len(targets) and to[-1] else np.zeros(0, np.int8)
        B = len(queries)
        return PairSet(qq, qo, tt, to,
                       np.broadcast_to(np.asarray(half_band, dtype=np.int32), (B,)).copy(),
                       np.broadcast_to(np.asarray(band_offset, dtype=np.int32), (B,)).copy(),
                       None if profile is None else np.asarray(profile, dtype=np.int8),
                       dict(meta or {}))


def band_cells(qlen, tlen, hb, off) -> np.ndarray:
    """Closed-form in-band cell count per pair (vectorised)."""
    qlen = np.asarray(qlen, dtype=np.int64)
    tlen = np.asarray(tlen, dtype=np.int64)
    hb = np.asarray(hb, dtype=np.int64)
    off = np.asarray(off, dtype=np.int64)
    W = 2 * hb + 1
    c = off - hb
    # cells = #{(i, d): 1<=i<=qlen, 0<=d<W, 1-c <= i+d <= tlen-c}.  For fixed
    # s = i + d the count n(s) is a trapezoid in s, so the total is a
    # difference of its prefix sums.
    P = np.minimum(qlen, W)
    Q = np.maximum(qlen, W)
    L = qlen + W - 1

    def prefix(x):
        x = np.clip(x, 0, L)
        a = x * (x + 1) // 2
        b = P * (P + 1) // 2 + (x - P) * P
        cc = P * (P + 1) // 2 + (Q - P) * P + ((L - Q) * (L - Q + 1) - (L - x) * (L - x + 1)) // 2
        return np.where(x <= P, a, np.where(x <= Q, b, cc))

    lo = np.maximum(1, 1 - c)
    hi = np.minimum(L, tlen - c)
    out = np.where((hi >= lo) & (qlen > 0), prefix(hi) - prefix(lo - 1), 0)
    return out.astype(np.int64)


def extension_pairs_150bp(n_pairs: int = 10_000, seed: int = 1, ref_len: int = 1_000_000,
                          read_len: int = 150, flank: int = 32, half_band: int = 32) -> PairSet:
    rng = np.random.default_rng(seed)
    ref = random_reference(ref_len, rng)
    starts = rng.integers(flank, ref_len - read_len - flank, size=n_pairs)
    queries, targets = [], []
    for s in starts:
        tmpl = ref[s: s + read_len]
        queries.append(apply_errors(tmpl, SHORT_READ, rng))
        targets.append(ref[s - flank: s + read_len + flank])
    return PairSet.from_lists(queries, targets, half_band, flank,
                              meta=dict(workload="extension_pairs_150bp", seed=seed,
                                        ref_len=ref_len))


def extension_pairs_mixed(n_pairs: int = 100_000, seed: int = 3, ref_len: int = 10_000_000,
                          min_len: int = 150, max_len: int = 20_000, log_mean: float = 7.0,
                          log_sigma: float = 1.2, band_slope: float = 0.02,
                          min_band: int = 32, max_band: int = 500, flank: int = 32) -> PairSet:
    """Mixed-length extension pairs; the band grows with the read length."""
    rng = np.random.default_rng(seed)
    ref = random_reference(ref_len, rng)
    lens = np.clip(rng.lognormal(log_mean, log_sigma, size=n_pairs), min_len, max_len).astype(np.int64)
    prof_id = rng.integers(0, 3, size=n_pairs).astype(np.int8)
    profs = (ILLUMINA, HIFI, ONT)
    queries, targets, hbs = [], [], []
    starts = rng.integers(flank, ref_len - max_len - flank - 1, size=n_pairs)
    for b in range(n_pairs):
        L = int(lens[b])
        s = int(starts[b])
        tmpl = ref[s: s + L]
        queries.append(apply_errors(tmpl, profs[prof_id[b]], rng))
        targets.append(ref[s - flank: s + L + flank])
        hbs.append(int(np.clip(min_band + band_slope * L, min_band, max_band)))
    return PairSet.from_lists(queries, targets, np.array(hbs, np.int32), flank, prof_id,
                              meta=dict(workload="extension_pairs_mixed", seed=seed,
                                        band_slope=band_slope, ref_len=ref_len))


def wfa_pairs_mixed(n_pairs: int = 20_000, seed: int = 8, flank: int = 32, **kw) -> tuple:
    """End-to-end pairs for the wavefront aligner: the mixed-length reads of
    :func:`extension_pairs_mixed` against the reference stretch they came from
    (the window the WFA extension takes from an exact chain: no flanks).
    Returns (queries, targets) lists of int8 codes."""
    ps = extension_pairs_mixed(n_pairs=n_pairs, seed=seed, flank=flank, **kw)
    qs = [ps.q(b) for b in range(len(ps))]
    ts = [ps.t(b)[flank: len(ps.t(b)) - flank] for b in range(len(ps))]
    return qs, ts


# --------------------------------------------------------------------------- #
# Minimizer sketch (host side, used to produce chaining anchors)
# --------------------------------------------------------------------------- #
def hash64(x: np.ndarray) -> np.ndarray:
    """Thomas Wang's invertible 64-bit integer hash as used by minimap2
    (the same function as seeding.py L83-98)."""
    x = x.astype(np.uint64, copy=True)
    u = np.uint64
    with np.errstate(over="ignore"):
        x = (~x) + (x << u(21))
        x ^= x >> u(24)
        x = x + (x << u(3)) + (x << u(8))
        x ^= x >> u(14)
        x = x + (x << u(2)) + (x << u(4))
        x ^= x >> u(28)
        x = x + (x << u(31))
    return x


def pack_kmers(codes: np.ndarray, k: int) -> tuple[np.ndarray, np.ndarray]:
    m = len(codes) - k + 1
    if m <= 0:
        return np.zeros(0, np.int64), np.zeros(0, bool)
    digits = codes.astype(np.int64) - 1
    bad = digits > 3
    packed = np.zeros(m, dtype=np.int64)
    invalid = np.zeros(m, dtype=bool)
    for o in range(k):
        packed = packed * 4 + digits[o: o + m]
        invalid |= bad[o: o + m]
    packed[invalid] = 0
    return packed, ~invalid


def minimizer_mask(h: np.ndarray, w: int) -> np.ndarray:
    """k-mers attaining the minimum hash of at least one window of ``w``
    consecutive k-mers (ties all kept)."""
    m = len(h)
    if m == 0:
        return np.zeros(0, bool)
    w = max(1, min(w, m))
    wmin = np.lib.stride_tricks.sliding_window_view(h, w).min(axis=1)
    nw = len(wmin)
    sel = np.zeros(m, dtype=bool)
    for o in range(w):
        sel[o: o + nw] |= h[o: o + nw] == wmin
    return sel


class MinimizerSketch:
    """Sorted (w, k) minimizer table of a reference (CSR of positions)."""

    def __init__(self, ref: np.ndarray, k: int = 15, w: int = 10, max_occ: int = 200):
        self.k, self.w = k, w
        packed, valid = pack_kmers(ref, k)
        sel = valid & minimizer_mask(hash64(packed), w)
        pos = np.flatnonzero(sel).astype(np.int64)
        keys = packed[pos]
        order = np.argsort(keys, kind="stable")
        keys, pos = keys[order], pos[order]
        uniq, counts = np.unique(keys, return_counts=True)
        if max_occ > 0 and len(uniq) and counts.max() > max_occ:
            keep_key = counts <= max_occ
            keep = np.repeat(keep_key, counts)
            keys, pos = keys[keep], pos[keep]
            uniq, counts = uniq[keep_key], counts[keep_key]
        self.keys = uniq
        self.offsets = np.zeros(len(uniq) + 1, dtype=np.int64)
        np.cumsum(counts, out=self.offsets[1:])
        self.positions = pos

    def query(self, codes: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        packed, valid = pack_kmers(codes, self.k)
        sel = valid & minimizer_mask(hash64(packed), self.w)
        qpos = np.flatnonzero(sel)
        keys = packed[qpos]
        if len(self.keys) == 0 or len(keys) == 0:
            z = np.zeros(0, np.int64)
            return z, z.copy()
        idx = np.searchsorted(self.keys, keys)
        idx_c = np.minimum(idx, len(self.keys) - 1)
        hit = self.keys[idx_c] == keys
        start = np.where(hit, self.offsets[idx_c], 0)
        count = np.where(hit, self.offsets[idx_c + 1] - self.offsets[idx_c], 0)
        total = int(count.sum())
        if total == 0:
            z = np.zeros(0, np.int64)
            return z, z.copy()
        read_pos = np.repeat(qpos, count)
        base = np.repeat(np.cumsum(count) - count, count)
        within = np.arange(total, dtype=np.int64) - base
        ref_pos = self.positions[np.repeat(start, count) + within]
        return read_pos.astype(np.int64), ref_pos


@dataclass
class AnchorBatch:
    """Anchors of many reads in CSR layout (original per-read order:
    forward-orientation hits first, then reverse-complement hits)."""

    read_off: np.ndarray  # int64 (R+1,)
    read_pos: np.ndarray  # int32
    ref_pos: np.ndarray  # int32
    length: np.ndarray  # int32
    strand: np.ndarray  # int8 (+1 / -1)
    read_len: np.ndarray  # int64 (R,)
    meta: dict = field(default_factory=dict)

    def __len__(self) -> int:
        return len(self.read_off) - 1

    @property
    def n_anchors(self) -> int:
        return int(self.read_off[-1])

    def read(self, r: int):
        s, e = int(self.read_off[r]), int(self.read_off[r + 1])
        return (self.read_pos[s:e], self.ref_pos[s:e], self.length[s:e], self.strand[s:e])

    def subset(self, idx) -> "AnchorBatch":
        idx = np.asarray(idx, dtype=np.int64)
        parts = [self.read(int(r)) for r in idx]
        counts = np.array([len(p[0]) for p in parts], dtype=np.int64)
        off = np.zeros(len(idx) + 1, dtype=np.int64)
        np.cumsum(counts, out=off[1:])
        cat = lambda k, dt: (np.concatenate([p[k] for p in parts]).astype(dt)
                             if len(parts) and off[-1] else np.zeros(0, dt))
        return AnchorBatch(off, cat(0, np.int32), cat(1, np.int32), cat(2, np.int32),
                           cat(3, np.int8), self.read_len[idx].copy(), dict(self.meta))


def chaining_reads_hifi(n_reads: int = 5_000, seed: int = 2, ref_len: int = 10_000_000,
                        mean_len: int = 15_000, spread: float = 0.2, k: int = 15, w: int = 10,
                        profile: ErrorProfile = HIFI, keep_reads: bool = False) -> AnchorBatch:
    rng = np.random.default_rng(seed)
    ref = random_reference(ref_len, rng)
    sketch = MinimizerSketch(ref, k=k, w=w)
    lens = rng.integers(int(mean_len * (1 - spread)), int(mean_len * (1 + spread)) + 1, size=n_reads)
    starts = rng.integers(0, ref_len - lens.max() - 1, size=n_reads)
    strands = np.where(rng.random(n_reads) < 0.5, 1, -1)
    rp, fp, ln, st, counts, rlen = [], [], [], [], [], []
    reads = []
    for r in range(n_reads):
        tmpl = ref[starts[r]: starts[r] + lens[r]]
        if strands[r] < 0:
            tmpl = reverse_complement(tmpl)
        read = apply_errors(tmpl, profile, rng)
        if keep_reads:
            reads.append(read)
        rlen.append(len(read))
        n = 0
        for s, codes in ((1, read), (-1, reverse_complement(read))):
            a, b = sketch.query(codes)
            rp.append(a)
            fp.append(b)
            ln.append(np.full(len(a), k, np.int64))
            st.append(np.full(len(a), s, np.int8))
            n += len(a)
        counts.append(n)
    off = np.zeros(n_reads + 1, dtype=np.int64)
    np.cumsum(counts, out=off[1:])
    batch = AnchorBatch(off, np.concatenate(rp).astype(np.int32), np.concatenate(fp).astype(np.int32),
                        np.concatenate(ln).astype(np.int32), np.concatenate(st).astype(np.int8),
                        np.array(rlen, np.int64),
                        dict(workload="chaining_reads_hifi", seed=seed, ref_len=ref_len))
    if keep_reads:
        batch.meta["reads"] = reads
        batch.meta["ref"] = ref
    return batch


# --------------------------------------------------------------------------- #
# Serving workload: reads of the mixed profile with their anchors, requests
# arriving as a Poisson stream
# --------------------------------------------------------------------------- #
@dataclass
class ReadPool:
    """Simulated reads (codes, as sequenced) of one reference, with their raw
    minimizer anchors in both orientations (client-side seeding)."""

    ref: np.ndarray
    reads: list
    anchors: AnchorBatch
    profile: np.ndarray  # int8 per read (0 illumina, 1 hifi, 2 ont)

    def __len__(self) -> int:
        return len(self.reads)

    def take(self, idx) -> tuple:
        idx = np.asarray(idx, dtype=np.int64)
        return [self.reads[int(i)] for i in idx], self.anchors.subset(idx)


def mixed_read_pool(n_reads: int = 4000, seed: int = 4, ref_len: int = 10_000_000, min_len: int = 150,
                    max_len: int = 20_000, log_mean: float = 7.0, log_sigma: float = 1.2, k: int = 15,
                    w: int = 10) -> ReadPool:
    """Reads with the length and error mix of the mixed extension workload
    (log-normal lengths, one third each Illumina-like, HiFi-like and
    ONT-like), random strand and position, seeded by (k, w) minimizers."""
    rng = np.random.default_rng(seed)
    ref = random_reference(ref_len, rng)
    sketch = MinimizerSketch(ref, k=k, w=w)
    lens = np.clip(rng.lognormal(log_mean, log_sigma, size=n_reads), min_len, max_len).astype(np.int64)
    prof_id = rng.integers(0, 3, size=n_reads).astype(np.int8)
    strands = np.where(rng.random(n_reads) < 0.5, 1, -1)
    starts = rng.integers(0, ref_len - max_len - 1, size=n_reads)
    profs = (ILLUMINA, HIFI, ONT)
    reads, rp, fp, ln, st, counts = [], [], [], [], [], []
    for r in range(n_reads):
        tmpl = ref[starts[r]: starts[r] + lens[r]]
        if strands[r] < 0:
            tmpl = reverse_complement(tmpl)
        read = apply_errors(tmpl, profs[prof_id[r]], rng)
        reads.append(read)
        n = 0
        for s, codes in ((1, read), (-1, reverse_complement(read))):
            a, b = sketch.query(codes)
            rp.append(a)
            fp.append(b)
            ln.append(np.full(len(a), k, np.int64))
            st.append(np.full(len(a), s, np.int8))
            n += len(a)
        counts.append(n)
    off = np.zeros(n_reads + 1, dtype=np.int64)
    np.cumsum(counts, out=off[1:])
    batch = AnchorBatch(off, np.concatenate(rp).astype(np.int32), np.concatenate(fp).astype(np.int32),
                        np.concatenate(ln).astype(np.int32), np.concatenate(st).astype(np.int8),
                        np.array([len(x) for x in reads], np.int64),
                        dict(workload="mixed_read_pool", seed=seed, ref_len=ref_len))
    return ReadPool(ref, reads, batch, prof_id)


def poisson_requests(n_requests: int, reads_per_s: float, pool_size: int, seed: int = 5, min_reads: int = 1,
                     max_reads: int = 64) -> list:
    """Requests of ``min_reads``..``max_reads`` reads (uniform) drawn from a
    pool, arriving as a Poisson process whose rate gives ``reads_per_s``
    reads per second on average: a list of (arrival seconds, read indices)."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(min_reads, max_reads + 1, size=n_requests)
    rate = reads_per_s / ((min_reads + max_reads) / 2.0)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_requests))
    return [(float(arrivals[i]), rng.integers(0, pool_size, size=int(sizes[i]))) for i in range(n_requests)]


def long_reads_ont(n_reads: int = 2000, seed: int = 6, ref_len: int = 50_000_000, min_len: int = 50_000,
                   max_len: int = 100_000, k: int = 15, w: int = 10, profile: ErrorProfile = ONT,
                   seeder=None) -> ReadPool:
    """Long-read stress workload: ONT-like reads (5% error, 60% indels) of
    uniform length in [min_len, max_len], random strand and position on a
    seeded reference, with raw (k, w) minimizer anchors in both
    orientations (about 10k per read).  ``seeder(ref)``, when given, returns
    an object whose ``seed(reads)`` gives the anchors (the device minimizer
    index); otherwise the host sketch finds them."""
    rng = np.random.default_rng(seed)
    ref = random_reference(ref_len, rng)
    lens = rng.integers(min_len, max_len + 1, size=n_reads)
    strands = np.where(rng.random(n_reads) < 0.5, 1, -1)
    starts = rng.integers(0, ref_len - max_len - 1, size=n_reads)
    reads = []
    for r in range(n_reads):
        tmpl = ref[starts[r]: starts[r] + lens[r]]
        if strands[r] < 0:
            tmpl = reverse_complement(tmpl)
        reads.append(apply_errors(tmpl, profile, rng))
    meta = dict(workload="long_reads_ont", seed=seed, ref_len=ref_len)
    if seeder is not None:
        a = seeder(ref).seed(reads)
        batch = AnchorBatch(a.read_off.astype(np.int64), a.read_pos.astype(np.int32), a.ref_pos.astype(np.int32),
                            a.length.astype(np.int32), a.strand.astype(np.int8),
                            np.array([len(x) for x in reads], np.int64), dict(meta, seeding="device index"))
        return ReadPool(ref, reads, batch, np.full(n_reads, 2, np.int8))
    sketch = MinimizerSketch(ref, k=k, w=w)
    rp, fp, ln, st, counts = [], [], [], [], []
    for read in reads:
        n = 0
        for s, codes in ((1, read), (-1, reverse_complement(read))):
            a, b = sketch.query(codes)
            rp.append(a)
            fp.append(b)
            ln.append(np.full(len(a), k, np.int64))
            st.append(np.full(len(a), s, np.int8))
            n += len(a)
        counts.append(n)
    off = np.zeros(n_reads + 1, dtype=np.int64)
    np.cumsum(counts, out=off[1:])
    batch = AnchorBatch(off, np.concatenate(rp).astype(np.int32), np.concatenate(fp).astype(np.int32),
                        np.concatenate(ln).astype(np.int32), np.concatenate(st).astype(np.int8),
                        np.array([len(x) for x in reads], np.int64), meta)
    return ReadPool(ref, reads, batch, np.full(n_reads, 2, np.int8))
