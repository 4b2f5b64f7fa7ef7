"""GPU parity on the full-size workloads the benchmark figures are quoted on.

* The mixed-length extension workload (100,000 pairs, 150 bp - 20 kb, bands
  32-432) runs as one batched call, so every pair lands in the class kernel
  (8/16-lane, one-warp, cooperative 2/4/8-warp, int32) it takes in the
  benchmark.  Every pair of 10 kb or more and a seeded sample of every length
  decile below are then compared with the oracle, field by field.
* The HiFi chaining workload: all 5,000 reads of 15 kb +- 20 %, h = 50.
* The long-read stress workload: 64 ONT-like reads spread over 50-100 kb on
  the 50 Mb reference, chained with h = 200, and every gap segment of each
  primary chain; four of them also with the wide segmentation (8 kb
  segments, half bands up to 2,000).

The oracle restates ``banded_affine_sw_batch`` + ``traceback_banded``
(graphmambaformer/alignment/extension.py L78-302) and ``AffineChainer.chain``
(graphmambaformer/alignment/chaining.py L129-180, L530-617).  Integer scores
and f64 chain scores are compared for equality.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from helpers import assert_sw_equal

pytestmark = pytest.mark.gpu


def _threads() -> int:
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return os.cpu_count() or 1


def _chains_equal(got, want, read_off):
    assert np.array_equal(got.n_chains, want.n_chains)
    for r in range(len(read_off) - 1):
        for a, b in zip(got.chains(r), want.chains(read_off, r)):
            assert a.score == b["score"] and a.strand == b["strand"] and a.is_primary == b["is_primary"], r
            assert [a.read_start, a.read_end, a.ref_start, a.ref_end] == [
                b["read_start"], b["read_end"], b["ref_start"], b["ref_end"]], r
            assert np.array_equal(a.anchor_idx, b["anchor_idx"]), r


def test_mixed_headline_workload_matches_oracle():
    from graphmambaformer_b200 import extension, synth
    from oracle import oracle

    ps = synth.extension_pairs_mixed(n_pairs=100_000, seed=1)
    params = (2, 4, 4, 2, 0)
    got = extension.align_pairs(ps, extension.sw_params(*params))  # the whole batch in one call
    qlen = ps.query_len
    long_idx = np.flatnonzero(qlen >= 10_000)
    rng = np.random.default_rng(17)
    short = np.flatnonzero(qlen < 10_000)
    order = short[np.argsort(qlen[short], kind="stable")]
    picks = [rng.choice(dec, size=min(250, len(dec)), replace=False) for dec in np.array_split(order, 10)]
    idx = np.unique(np.concatenate([long_idx] + picks))
    assert len(long_idx) > 3000 and len(idx) >= 5000 and qlen[idx].max() >= 19_000
    assert ps.half_band[idx].max() == ps.half_band.max()
    want = oracle.sw_batch([ps.q(int(b)) for b in idx], [ps.t(int(b)) for b in idx], ps.half_band[idx],
                           ps.band_offset[idx], *params, threads=_threads())
    assert_sw_equal(got, want, idx=idx, label="mixed 100k")


def test_hifi_chaining_workload_all_reads_match_oracle():
    from graphmambaformer_b200 import chaining, synth
    from graphmambaformer_b200.config import ChainingConfig
    from oracle import oracle

    batch = synth.chaining_reads_hifi(n_reads=5_000, seed=2)
    cfg = ChainingConfig(max_lookback=50, max_gap=5000)
    got = chaining.chain_anchor_batch(batch, cfg)
    want = oracle.chain_batch(batch.read_off, batch.read_pos, batch.ref_pos, batch.length, batch.strand,
                              oracle.penalty_lut(5000, 6.0, 0.05, 0.5), max_lookback=50, threads=_threads())
    assert batch.n_anchors > 10_000_000
    _chains_equal(got, want, batch.read_off)


def test_long_read_workload_chains_and_segments_match_oracle():
    import torch

    from graphmambaformer_b200 import longreads, synth
    from graphmambaformer_b200.seeding import DeviceMinimizerIndex
    from oracle import oracle

    pool = synth.long_reads_ont(n_reads=64, seed=6, seeder=lambda ref: DeviceMinimizerIndex(
        ref, k=15, w=10, max_occ=200, device="cuda:0"))
    lens = np.array([len(r) for r in pool.reads])
    assert lens.min() < 60_000 and lens.max() > 90_000
    al = longreads.LongReadAligner(torch.from_numpy(pool.ref).to("cuda:0"), "cuda:0")
    prim, res = al.primary_chains(pool.reads, pool.anchors)
    a = pool.anchors
    want = oracle.chain_batch(a.read_off, a.read_pos, a.ref_pos, a.length, a.strand,
                              oracle.penalty_lut(5000, 6.0, 0.05, 0.5), max_lookback=200, threads=_threads())
    _chains_equal(res, want, a.read_off)
    seg = al.segments(pool.reads, prim)
    got = al.align_segments(pool.reads, seg)
    qs, ts = [], []
    for i in range(len(seg)):
        read = pool.reads[int(seg.read[i])]
        frame = read if seg.strand[i] > 0 else synth.reverse_complement(read)
        qs.append(frame[seg.q_start[i]: seg.q_start[i] + seg.q_len[i]])
        ts.append(pool.ref[seg.t_start[i]: seg.t_start[i] + seg.t_len[i]])
    exp = oracle.sw_batch(qs, ts, seg.half_band, seg.band_offset, 2, 4, 6, 2, 600, threads=_threads())
    assert len(seg) > 3000
    assert_sw_equal(got, exp, label="long-read gap segments")

    # the wide segmentation (8 kb segments, half bands up to 2,000) on four reads
    wide = al.segments(pool.reads, prim[:4] + [None] * (len(prim) - 4), mode=longreads.WIDE)
    assert wide.half_band.max() == longreads.MAX_BAND and wide.half_band.min() < 1500
    got = al.align_segments(pool.reads, wide)
    qs, ts = [], []
    for i in range(len(wide)):
        read = pool.reads[int(wide.read[i])]
        frame = read if wide.strand[i] > 0 else synth.reverse_complement(read)
        qs.append(frame[wide.q_start[i]: wide.q_start[i] + wide.q_len[i]])
        ts.append(pool.ref[wide.t_start[i]: wide.t_start[i] + wide.t_len[i]])
    exp = oracle.sw_batch(qs, ts, wide.half_band, wide.band_offset, 2, 4, 6, 2, 600, threads=min(4, _threads()))
    assert_sw_equal(got, exp, label="long-read wide segments")
