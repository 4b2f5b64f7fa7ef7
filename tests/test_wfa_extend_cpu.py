"""The host half of `ExtensionEngine`'s WFA mode on the CPU: the windows
`_wfa_windows` derives from each chain, the oracle's wavefront alignment,
the score recomputed from the CIGAR (`wfa_extension_result`), and, past
the distance bound, banded SW over `_pairs`' window with soft clips.  Together
they reproduce the reference's WFA-mode `extend_chains` outputs in
wfa_golden.npz."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from helpers import load, words_to_cigar
from oracle import oracle


def test_wfa_mode_windows_through_the_oracle_match_reference_golden():
    from graphmambaformer_b200.config import ExtensionConfig
    from graphmambaformer_b200.extension import ExtensionEngine, wfa_extension_result
    from graphmambaformer_b200.synth import decode_bases, encode_bases
    from graphmambaformer_b200.types import AnchorSet, Chain, add_soft_clips

    g = load("wfa_golden.npz")
    ref_codes = encode_bases(decode_bases(g["ref"]))
    k = n_wfa = n_fallback = 0
    for c in range(len(g["calls"])):
        algo, md = int(g["calls"][c][0]), int(g["calls"][c][1])
        read = encode_bases(decode_bases(g["reads"][g["read_off"][c]: g["read_off"][c + 1]]))
        a = g["anchors"][g["anchor_off"][c]: g["anchor_off"][c + 1]]
        rp, fp, ln = a[:, 0], a[:, 1], a[:, 2]
        anchors = AnchorSet.from_lists(rp, fp, ln, a[:, 3].astype(np.int8))
        chains = [Chain(anchor_idx=np.arange(lo, hi), score=30.0, strand=int(cs), read_start=int(rp[lo:hi].min()),
                        read_end=int((rp[lo:hi] + ln[lo:hi]).max()), ref_start=int(fp[lo:hi].min()),
                        ref_end=int((fp[lo:hi] + ln[lo:hi]).max()))
                   for call, lo, hi, cs in g["chains"] if call == c]
        cfg = ExtensionConfig(algorithm="wfa" if algo else "banded_sw", wfa_max_distance=md)
        if not algo:
            k += len(chains)
            continue
        eng = ExtensionEngine.__new__(ExtensionEngine)  # the host logic only: no device
        eng.cfg = cfg
        item = (read, chains, anchors, ref_codes)
        qs, ts, meta = eng._wfa_windows([item])
        for (q, t, (_, ci, start, read_len)) in zip(qs, ts, meta):
            d, cigar = oracle.wfa_align(q, t, md)
            if d >= 0:
                got = wfa_extension_result(cigar, start, len(t), read_len, cfg)
                n_wfa += 1
            else:  # banded SW of this chain alone, as the reference re-enters extend_chains
                ps, pm = eng._pairs([(read, [chains[ci]], anchors, ref_codes)])
                out = oracle.sw_batch([ps.q(0)], [ps.t(0)], ps.half_band, ps.band_offset, cfg.match_score,
                                      cfg.mismatch_penalty, cfg.gap_open, cfg.gap_extend, cfg.x_drop)
                s0 = pm[0][1]
                qs0, qe0 = int(out.query_start[0]), int(out.query_end[0])
                cnt = [int(x) for x in out.counts[0]]
                got = SimpleNamespace(
                    score=float(out.score[0]), cigar=add_soft_clips(out.cigars[0], qs0, read_len - qe0),
                    read_start=qs0, read_end=qe0, ref_start=int(out.target_start[0]) + s0,
                    ref_end=int(out.target_end[0]) + s0, n_match=cnt[0], n_mismatch=cnt[1],
                    n_insertion=cnt[2], n_deletion=cnt[3])
                n_fallback += 1
            kk = k + ci
            assert got.cigar == words_to_cigar(g["x_cigar"][g["x_cigar_off"][kk]: g["x_cigar_off"][kk + 1]]), kk
            assert got.score == g["x_score"][kk], kk
            assert [got.read_start, got.read_end, got.ref_start, got.ref_end] == list(g["x_span"][kk]), kk
            assert [got.n_match, got.n_mismatch, got.n_insertion, got.n_deletion] == list(g["x_counts"][kk]), kk
        k += len(chains)
    assert k == len(g["x_score"]) and n_wfa > 0 and n_fallback > 0


def test_history_chunks_follow_the_greedy_split():
    """history_chunks equals the pair-by-pair greedy split: a range closes
    before the pair that would take it over the budget, and a pair above
    the budget stands alone."""
    from graphmambaformer_b200.wfa import history_chunks

    def greedy(hist, budget):
        out, cur, acc = [], [], 0
        for p, h in enumerate(hist):
            if cur and acc + h > budget:
                out.append((cur[0], cur[-1] + 1))
                cur, acc = [], 0
            cur.append(p)
            acc += int(h)
        if cur:
            out.append((cur[0], cur[-1] + 1))
        return out

    rng = np.random.default_rng(3)
    for n in (0, 1, 2, 17, 500):
        for budget in (1, 50, 1000, 10 ** 9):
            hist = rng.integers(0, 120, size=n) ** 2 * (rng.random(n) < 0.8)
            assert history_chunks(hist, budget) == greedy(hist, budget), (n, budget)


def test_wfa_batch_csr_layout():
    from graphmambaformer_b200.wfa import WfaBatch

    rng = np.random.default_rng(4)
    qs = [rng.integers(0, 4, size=L).astype(np.int8) for L in (0, 3, 9, 0, 5)]
    ts = [rng.integers(0, 4, size=L).astype(np.int8) for L in (2, 0, 9, 0, 6)]
    b = WfaBatch.of(qs, ts)
    assert len(b) == 5 and b.query.dtype == np.int8 and b.query_off.dtype == np.int64
    for i in range(5):
        assert np.array_equal(b.query[b.query_off[i]: b.query_off[i + 1]], qs[i])
        assert np.array_equal(b.target[b.target_off[i]: b.target_off[i + 1]], ts[i])
    with pytest.raises(ValueError):
        WfaBatch.of(qs, ts[:2])
