"""The columnar record path on the CPU: records built as arrays from a
batch's chain and extension columns (``record_table``) and laid out for the
SAM kernels (``sam_batch``) equal, field by field, what the per-record object
path gives: ``read_alignments`` (pipeline.py L486-511 with L365-426) per read,
then ``sam_records`` (alignment_io.py L55-187)."""

from __future__ import annotations

from dataclasses import fields

import numpy as np
import pytest

from graphmambaformer_b200.records import (AlignmentRecord, ReadAlignments, RecordTable, _clip_words,
                                           margin_mapq, margin_mapq_rows, read_alignments, record_table,
                                           sam_batch, sam_records)
from graphmambaformer_b200.serving import BatchAlignments
from graphmambaformer_b200.synth import decode_bases
from graphmambaformer_b200.types import AnchorSet, Chain, add_soft_clips, words_to_cigar


def _same_layout(a, b):
    for f in fields(a):
        x, y = getattr(a, f.name), getattr(b, f.name)
        if f.name == "modalities":
            assert list(x) == list(y)
        else:
            assert np.array_equal(np.asarray(x), np.asarray(y)), f.name
            assert np.asarray(x).dtype == np.asarray(y).dtype, f.name


def test_margin_mapq_rows_equals_per_read_rule():
    rng = np.random.default_rng(1)
    R, mc = 400, 6
    scores = np.round(rng.normal(40, 30, size=(R, mc)), rng.integers(0, 3))
    scores[::7, 1] = scores[::7, 0]          # ties for the best
    scores[::11] = -np.abs(scores[::11])     # nothing positive
    scores[5, 0] = 0.0
    n = rng.integers(0, mc + 1, size=R)
    got = margin_mapq_rows(scores, n, 60)
    for r in range(R):
        ch = [Chain(np.zeros(0, np.int64), float(x), 1, 0, 0, 0, 0) for x in scores[r, : n[r]]]
        assert got[r] == margin_mapq(ch, 60), r
    # margins that land exactly on .5 round half to even, as Python's round does
    half = np.array([[4.0, 3.0], [8.0, 7.0]])
    for mq in (2, 6, 10):
        got = margin_mapq_rows(half, np.array([2, 2]), mq)
        want = [margin_mapq([Chain(np.zeros(0, np.int64), float(x), 1, 0, 0, 0, 0) for x in row], mq) for row in half]
        assert list(got) == want


def test_clip_words_equal_add_soft_clips():
    rng = np.random.default_rng(2)
    K = 300
    clen = rng.integers(0, 6, size=K)
    clen[::9] = 0
    cstart = np.zeros(K, np.int64)
    np.cumsum(clen[:-1], out=cstart[1:])
    words = (rng.integers(1, 50, size=int(clen.sum())) << 4 | rng.integers(0, 4, size=int(clen.sum()))).astype(np.uint32)
    left = rng.integers(0, 3, size=K) * rng.integers(0, 20, size=K)
    right = rng.integers(0, 3, size=K) * rng.integers(0, 20, size=K)
    out, off = _clip_words(words, cstart, clen, left, right)
    for k in range(K):
        want = add_soft_clips(words_to_cigar(words[cstart[k]: cstart[k] + clen[k]]), int(left[k]), int(right[k]))
        assert words_to_cigar(out[off[k]: off[k + 1]]) == want, k


def _synthetic_batch(rng, R=60, mc=4):
    """A BatchAlignments as BatchAligner builds it (SW columns), with reads
    that have no chains, chains without a primary and empty CIGARs."""
    n = rng.integers(0, mc + 1, size=R)
    n[::5] = 0
    C = int(n.sum())
    chain_off = np.zeros(R + 1, np.int64)
    np.cumsum(n, out=chain_off[1:])
    clen = rng.integers(0, 5, size=C)
    cstart = np.zeros(C, np.int64)
    np.cumsum(clen[:-1], out=cstart[1:])
    W = int(clen.sum())
    words = (rng.integers(1, 40, size=W) << 4 | rng.integers(0, 4, size=W)).astype(np.uint32)
    qs = rng.integers(0, 30, size=C).astype(np.int32)
    qe = qs + rng.integers(0, 200, size=C).astype(np.int32)
    ts = rng.integers(0, 10 ** 6, size=C).astype(np.int64)
    cols = dict(score=rng.integers(0, 300, size=C).astype(np.int32), qs=qs, qe=qe, ts=ts,
                te=ts + rng.integers(0, 200, size=C), counts=rng.integers(0, 50, size=(C, 4)).astype(np.int32),
                cstart=cstart, clen=clen.astype(np.int32), clip_l=qs, clip_r=rng.integers(0, 25, size=C))
    prim = np.zeros(C, np.int32)
    for r in range(R):
        if n[r] and r % 7:
            prim[chain_off[r] + rng.integers(0, n[r])] = 1
    chains = dict(score=np.round(rng.normal(50, 30, size=C), 1), strand=rng.choice([-1, 1], size=C).astype(np.int32),
                  prim=prim)
    return BatchAlignments(R, chain_off, cols, words, chains=chains)


def _object_results(ba, names, lens):
    """The same batch through the per-read object path."""
    out = []
    for r in range(len(ba)):
        c0 = int(ba.chain_off[ba.lo + r])
        chains = [Chain(np.zeros(0, np.int64), float(ba.chains["score"][c0 + i]), int(ba.chains["strand"][c0 + i]),
                        0, 0, 0, 0, is_primary=bool(ba.chains["prim"][c0 + i])) for i in range(len(ba[r]))]
        out.append(read_alignments(names[r], int(lens[r]), AnchorSet.empty(), chains, ba[r]))
    return out


@pytest.mark.parametrize("secondary", [False, True])
def test_record_table_and_layout_equal_object_path(secondary):
    rng = np.random.default_rng(3)
    ba = _synthetic_batch(rng)
    R = ba.n_reads
    lens = rng.integers(0, 300, size=R)
    codes = [rng.integers(1, 6, size=int(L)).astype(np.int8) for L in lens]
    names = [f"read/{r}" + ("é" if r % 13 == 0 else "") for r in range(R)]
    quals = [rng.integers(0, 120, size=int(L)) if r % 3 == 0 else None for r, L in enumerate(lens)]
    mods = ["ont" if r % 4 else "hifi" for r in range(R)]
    seq_off = np.zeros(R + 1, np.int64)
    np.cumsum(lens, out=seq_off[1:])
    flat = np.concatenate(codes)
    qual = np.concatenate([q if q is not None else np.zeros(int(L), np.int64) for q, L in zip(quals, lens)])
    refs = {0: 10 ** 7, 3: 500}
    table = record_table(ba, ref_id=0)
    objs = _object_results(ba, names, lens)
    # the records themselves
    recs = [rec for ra in objs for rec in ra.records]
    assert len(recs) == len(table)
    for i, rec in enumerate(recs):
        w = table.cigar[table.cigar_off[i]: table.cigar_off[i + 1]]
        assert words_to_cigar(w) == [tuple(x) for x in rec.cigar], i
        assert (table.ref_id[i] >= 0) == rec.is_mapped
        if rec.is_mapped:
            assert (table.ref_start[i], table.ref_end[i], table.strand[i], table.mapq[i], bool(table.is_primary[i])) == \
                (rec.ref_start, rec.ref_end, rec.strand, rec.mapq, rec.is_primary), i
    reads = [type("Read", (), dict(read_id=names[r], seq=decode_bases(codes[r]), quals=quals[r], modality=mods[r]))()
             for r in range(R)]
    want = sam_records(objs, reads, "pacbio_hifi", secondary, refs, {0: "chr1"})
    got = sam_batch(table, names, flat, seq_off, qual, mods, secondary, refs, {0: "chr1"})
    _same_layout(got, want)
    # ASCII bases and a (bytes, offsets) name column give the same layout
    ascii_ = np.frombuffer("".join(decode_bases(c) for c in codes).encode(), np.uint8)
    raw = "".join(names).encode()
    noff = np.zeros(R + 1, np.int64)
    np.cumsum([len(x.encode()) for x in names], out=noff[1:])
    got2 = sam_batch(table, (np.frombuffer(raw, np.uint8), noff), ascii_, seq_off, qual, mods, secondary, refs,
                     {0: "chr1"})
    _same_layout(got2, want)


def test_record_table_of_a_slice_and_of_no_chains():
    rng = np.random.default_rng(4)
    ba = _synthetic_batch(rng, R=30)
    whole = record_table(ba)
    part = record_table(ba[10:20])
    rows = np.flatnonzero((whole.read >= 10) & (whole.read < 20))
    assert np.array_equal(part.read, whole.read[rows] - 10)
    for name in ("ref_id", "ref_start", "ref_end", "strand", "mapq", "is_primary"):
        assert np.array_equal(getattr(part, name), getattr(whole, name)[rows]), name
    for i, j in enumerate(rows):
        assert np.array_equal(part.cigar[part.cigar_off[i]: part.cigar_off[i + 1]],
                              whole.cigar[whole.cigar_off[j]: whole.cigar_off[j + 1]])
    empty = record_table(BatchAlignments.empty(3))
    assert list(empty.read) == [0, 1, 2] and (empty.ref_id == -1).all() and len(empty.cigar) == 0


def test_sam_batch_of_hand_made_records_equals_object_path():
    """Records a caller builds directly (several per read, unmapped ones,
    a read with no primary) lay out as sam_records lays out their objects."""
    recs = [[AlignmentRecord("a", 5, 0, 10, 15, -1, 33, cigar=[("S", 1), ("=", 4)], is_mapped=True, is_primary=False),
             AlignmentRecord("a", 5, 2, 30, 35, 1, 7, cigar=[("=", 5)], is_mapped=True, is_primary=True)],
            [AlignmentRecord.unmapped("b", 3)],
            [AlignmentRecord("c", 4, 0, 0, 4, 1, 300, cigar=[("X", 4)], is_mapped=True, is_primary=False)]]
    results = [ReadAlignments(r[0].read_id, r[0].read_len, records=r) for r in recs]
    seqs = ["ACGTA", "GGA", "TTTT"]
    flat = [rec for r in recs for rec in r]
    cig = [[(int(n) << 4) | "=XIDS".index(op) for op, n in rec.cigar] if rec.is_mapped else [] for rec in flat]
    off = np.zeros(len(flat) + 1, np.int64)
    np.cumsum([len(c) for c in cig], out=off[1:])
    table = RecordTable(read=np.array([0, 0, 1, 2]), ref_id=np.array([0, 2, -1, 0]),
                        ref_start=np.array([10, 30, -1, 0]), ref_end=np.array([15, 35, -1, 4]),
                        strand=np.array([-1, 1, 1, 1], np.int8), mapq=np.array([33, 7, 0, 300], np.int32),
                        is_primary=np.array([False, True, True, False]),
                        cigar=np.array([w for c in cig for w in c], np.uint32), cigar_off=off)
    s_off = np.array([0, 5, 8, 12])
    ascii_ = np.frombuffer("".join(seqs).encode(), np.uint8)
    for secondary in (False, True):
        for refs in (None, {0: 100, 2: 50}):
            want = sam_records(results, seqs, "illumina", secondary, refs)
            got = sam_batch(table, ["a", "b", "c"], ascii_, s_off, None, "illumina", secondary, refs)
            _same_layout(got, want)


def test_record_table_from_extension_objects_equals_object_path():
    """The WFA path's batches hold ready ExtensionResults instead of columns;
    record_table reads those the same way."""
    from graphmambaformer_b200.types import ExtensionResult

    rng = np.random.default_rng(6)
    cols_batch = _synthetic_batch(rng, R=25)
    objs = [cols_batch._chain(c) for c in range(int(cols_batch.chain_off[-1]))]
    assert all(isinstance(e, ExtensionResult) for e in objs)
    obj_batch = BatchAlignments(cols_batch.n_reads, cols_batch.chain_off, objects=objs, chains=cols_batch.chains)
    a, b = record_table(cols_batch), record_table(obj_batch)
    for f in fields(a):
        assert np.array_equal(getattr(a, f.name), getattr(b, f.name)), f.name
