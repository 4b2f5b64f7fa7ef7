"""Long-read stress path on the GPU: 50-60 kb ONT-like reads on a seeded
reference, chaining with a 200-anchor predecessor window, then banded SW over
the gaps of each read's primary chain (the segmentation rule of
graphmambaformer_b200.longreads).  Chains match the oracle bit for bit, and
every gap segment -- queries reverse-complemented on the device for strand
-1, windows gathered from the resident reference -- matches the oracle's
score, coordinates and CIGAR."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_long_read_chains_and_gap_segments_match_oracle():
    import torch

    from graphmambaformer_b200 import longreads, synth
    from oracle import oracle

    pool = synth.long_reads_ont(n_reads=4, seed=16, ref_len=3_000_000, min_len=50_000, max_len=60_000)
    al = longreads.LongReadAligner(torch.from_numpy(pool.ref).to("cuda:0"), "cuda:0")
    prim, res = al.primary_chains(pool.reads, pool.anchors)
    a = pool.anchors
    lut = oracle.penalty_lut(5000, 6.0, 0.05, 0.5)
    want = oracle.chain_batch(a.read_off, a.read_pos, a.ref_pos, a.length, a.strand, lut, max_lookback=200)
    assert np.array_equal(res.n_chains, want.n_chains)
    for r in range(len(pool)):
        for got, ref in zip(res.chains(r), want.chains(a.read_off, r)):
            assert got.score == ref["score"] and np.array_equal(got.anchor_idx, ref["anchor_idx"])
    assert all(p is not None for p in prim)

    seg = al.segments(pool.reads, prim)
    assert len(seg) > 100 and seg.half_band.min() >= longreads.BASE_BAND
    got = al.align_segments(pool.reads, seg)
    qs, ts = [], []
    for i in range(len(seg)):
        read = pool.reads[int(seg.read[i])]
        frame = read if seg.strand[i] > 0 else synth.reverse_complement(read)
        qs.append(frame[seg.q_start[i]: seg.q_start[i] + seg.q_len[i]])
        ts.append(pool.ref[seg.t_start[i]: seg.t_start[i] + seg.t_len[i]])
    exp = oracle.sw_batch(qs, ts, seg.half_band, seg.band_offset, 2, 4, 6, 2, 600, threads=8)
    assert np.array_equal(got.score.astype(np.float32), exp.score)
    assert np.array_equal(got.query_end, exp.query_end) and np.array_equal(got.target_end, exp.target_end)
    assert np.array_equal(got.query_start, exp.query_start) and np.array_equal(got.target_start, exp.target_start)
    assert all(got.cigar(i) == exp.cigars[i] for i in range(len(seg)))
