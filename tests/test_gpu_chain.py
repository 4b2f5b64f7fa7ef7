"""GPU parity of the chaining kernels: float64 DP values (bit patterns),
predecessors, chain membership, spans and primary flags against the
reference's golden vectors and the CPU oracle."""

from __future__ import annotations

import os
import pickle

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import load

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def chaining():
    from graphmambaformer_b200 import chaining

    return chaining


def _same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float64).view(np.int64), np.asarray(b, np.float64).view(np.int64))


def test_chain_dp_matches_reference_golden(chaining):
    from graphmambaformer_b200.config import ChainingConfig

    g = load("chain_golden.npz")
    off, boff = g["dp_off"], g["dp_bonus_off"]
    for c in range(len(off) - 1):
        s, e = off[c], off[c + 1]
        lb, mg = int(g["dp_lookback"][c]), int(g["dp_max_gap"][c])
        bonus = g["dp_bonus"][boff[c]: boff[c + 1]].reshape(e - s, lb) if g["dp_has_bonus"][c] else None
        f, p = chaining.chain_dp_rows(g["dp_read_end"][s:e], g["dp_ref_end"][s:e], g["dp_weight"][s:e],
                                      ChainingConfig(max_lookback=lb, max_gap=mg), bonus=bonus)
        assert _same_bits(f, g["dp_f"][s:e]), c
        assert np.array_equal(p, g["dp_parent"][s:e]), c


@pytest.mark.parametrize("lb", [1, 2, 31, 32, 33, 64, 65, 96, 97, 128, 160, 192, 224, 225, 300, 1024])
def test_chain_dp_every_window_width_matches_oracle(chaining, lb):
    """Window widths on both sides of every 32-anchor block boundary (the
    broadcast form keeps ceil(lb/32)+1 blocks in registers up to 224, the
    shared-memory ring form takes wider windows).  Dense anchors so that most
    of the window is a valid predecessor; integer and fractional weights,
    with and without a bonus; collinear runs for ties.  Bit patterns against
    the oracle."""
    from oracle import oracle

    from graphmambaformer_b200.config import ChainingConfig

    rng = np.random.default_rng(1000 + lb)
    cfg = ChainingConfig(max_lookback=lb, max_gap=400)
    lut = oracle.penalty_lut(400, cfg.gap_open, cfg.gap_extend, cfg.log_coeff)
    for n, frac, with_bonus in ((1, False, False), (33, False, True), (700, False, False),
                                (257, True, True), (96, False, False)):
        if n == 96:  # collinear: equal candidates from many predecessors
            re = np.repeat(np.arange(1, 49) * 7, 2)[:n].astype(np.int64)
            fe = re.copy()
        else:
            re = np.sort(rng.integers(1, 4 * n + 2, size=n)).astype(np.int64)
            fe = np.sort(rng.integers(1, 4 * n + 2, size=n)).astype(np.int64)
        w = rng.integers(5, 30, size=n).astype(np.float64)
        if frac:
            w += rng.random(n)
        bonus = rng.normal(0, 3, size=(n, lb)) if with_bonus else None
        f, p = chaining.chain_dp_rows(re, fe, w, cfg, bonus=bonus)
        ef, ep = oracle.chain_dp(re, fe, w, lut, lb, 400, bonus=bonus)
        assert _same_bits(f, ef), (lb, n)
        assert np.array_equal(p, ep), (lb, n)
        assert n < 200 or lb < 2 or (p >= 0).mean() > 0.5, "the case must chain most anchors"
    # a collinear run whose members sit the whole window apart, the anchors
    # between them ahead on the read (never a valid predecessor of the run)
    m = min(lb, 390)
    i = np.arange(600)
    run = i % m == 0
    re = np.where(run, i + 1, 1_000_000 + i).astype(np.int64)
    fe = (i + 1).astype(np.int64)
    w = np.full(600, 15.0)
    f, p = chaining.chain_dp_rows(re, fe, w, cfg)
    ef, ep = oracle.chain_dp(re, fe, w, lut, lb, 400)
    assert _same_bits(f, ef) and np.array_equal(p, ep), lb
    assert np.array_equal(p[run][1:], i[run][1:] - m)


def test_chain_dp_padded_known_answer(chaining):
    """tests/test_accel.py L347-370 of the reference, through the (B, A, 3)
    RawKernel signature; fractional weights, exact float64."""
    import torch

    anchors = torch.tensor([[[10, 10, 0], [20, 20, 0], [30, 31, 0]]], dtype=torch.int32, device="cuda")
    w = torch.tensor([[10.5, 9.25, 8.75]], dtype=torch.float64, device="cuda")
    f, p = chaining.chain_dp(anchors, torch.tensor([3], dtype=torch.int32, device="cuda"), 64, 5000,
                             6.0, 0.05, 0.5, weights=w)
    assert p[0].tolist() == [-1, 0, 1]
    from oracle import oracle

    ef, ep = oracle.chain_dp([10, 20, 30], [10, 20, 31], [10.5, 9.25, 8.75],
                             oracle.penalty_lut(5000, 6.0, 0.05, 0.5))
    assert _same_bits(f[0].cpu().numpy(), ef)


def test_chain_dp_padded_ragged_rows(chaining):
    """tests/test_alignment_stages.py L502-520: ragged rows of a padded batch."""
    import torch

    from oracle import oracle

    an = torch.tensor([[[10, 10, 0], [20, 21, 0], [30, 32, 0]], [[8, 8, 0], [18, 20, 0], [0, 0, 0]]],
                      dtype=torch.int32, device="cuda")
    w = torch.tensor([[10.5, 9.25, 8.75], [7.5, 8.25, 0.0]], dtype=torch.float64, device="cuda")
    f, p = chaining.chain_dp(an, torch.tensor([3, 2], device="cuda"), 4, 5000, 6.0, 0.05, 0.5, weights=w)
    lut = oracle.penalty_lut(5000, 6.0, 0.05, 0.5)
    for row, n in enumerate((3, 2)):
        ef, ep = oracle.chain_dp(an[row, :n, 0].cpu(), an[row, :n, 1].cpu(), w[row, :n].cpu(), lut, 4)
        assert _same_bits(f[row, :n].cpu().numpy(), ef)
        assert p[row, :n].cpu().tolist() == ep.tolist()
    assert float(f[1, 2]) == 0.0 and int(p[1, 2]) == -1


def _golden_reads():
    g = load("chain_golden.npz")
    from graphmambaformer_b200.types import AnchorSet

    reads = []
    off = g["read_off"]
    for r in range(len(off) - 1):
        s, e = off[r], off[r + 1]
        reads.append((AnchorSet.from_lists(g["read_pos"][s:e], g["ref_pos"][s:e], g["length"][s:e],
                                           g["strand"][s:e]), int(g["read_lookback"][r])))
    return g, reads


def test_chainer_matches_reference_golden(chaining):
    from graphmambaformer_b200.config import ChainingConfig

    g, reads = _golden_reads()
    moff = g["chain_members_off"]
    first = np.concatenate([[0], np.cumsum(g["n_chains"])])
    for lb in sorted({lb for _, lb in reads}):
        rows = [r for r, (_, l) in enumerate(reads) if l == lb]
        chainer = chaining.AffineChainer(ChainingConfig(max_lookback=lb, max_gap=5000))
        got = chainer.chain_batch([reads[r][0] for r in rows])
        for r, chains in zip(rows, got):
            assert len(chains) == g["n_chains"][r], r
            for k, c in enumerate(chains):
                gc = first[r] + k
                assert c.score == g["chain_score"][gc], (r, k)
                assert c.strand == g["chain_strand"][gc]
                assert [c.read_start, c.read_end, c.ref_start, c.ref_end] == list(g["chain_span"][gc])
                assert c.is_primary == bool(g["chain_primary"][gc])
                assert np.array_equal(c.anchor_idx, g["chain_members"][moff[gc]: moff[gc + 1]]), (r, k)


def test_chain_batch_matches_oracle_hifi_workload(chaining):
    """300 simulated 15 kb HiFi reads (minimizer anchors, h=50): every kept
    chain's score, strand, spans, primary flag and members."""
    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.config import ChainingConfig
    from oracle import oracle

    batch = synth.chaining_reads_hifi(n_reads=300, seed=8, ref_len=10_000_000)
    cfg = ChainingConfig(max_lookback=50, max_gap=5000)
    got = chaining.chain_anchor_batch(batch, cfg)
    want = oracle.chain_batch(batch.read_off, batch.read_pos, batch.ref_pos, batch.length,
                              batch.strand, oracle.penalty_lut(5000, 6.0, 0.05, 0.5), max_lookback=50,
                              threads=8)
    assert np.array_equal(got.n_chains, want.n_chains)
    for r in range(len(batch)):
        gc = got.chains(r)
        wc = want.chains(batch.read_off, r)
        for a, b in zip(gc, wc):
            assert a.score == b["score"] and a.strand == b["strand"] and a.is_primary == b["is_primary"]
            assert [a.read_start, a.read_end, a.ref_start, a.ref_end] == [
                b["read_start"], b["read_end"], b["ref_start"], b["ref_end"]]
            assert np.array_equal(a.anchor_idx, b["anchor_idx"])


@pytest.mark.parametrize("lb", [1, 16, 32, 96, 128, 160, 192, 224, 256])
def test_chain_batch_every_window_width_matches_oracle(chaining, lb):
    """The read-batch path (anchor lengths as weights) at window widths that
    select each register-block count of the broadcast DP, and the ring form
    beyond 224."""
    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.config import ChainingConfig
    from oracle import oracle

    batch = synth.chaining_reads_hifi(n_reads=24, seed=40 + lb, ref_len=2_000_000, mean_len=6000)
    cfg = ChainingConfig(max_lookback=lb, max_gap=5000)
    got = chaining.chain_anchor_batch(batch, cfg)
    want = oracle.chain_batch(batch.read_off, batch.read_pos, batch.ref_pos, batch.length,
                              batch.strand, oracle.penalty_lut(5000, 6.0, 0.05, 0.5), max_lookback=lb,
                              threads=8)
    assert np.array_equal(got.n_chains, want.n_chains)
    for r in range(len(batch)):
        for a, b in zip(got.chains(r), want.chains(batch.read_off, r)):
            assert a.score == b["score"] and a.is_primary == b["is_primary"]
            assert [a.read_start, a.read_end, a.ref_start, a.ref_end] == [
                b["read_start"], b["read_end"], b["ref_start"], b["ref_end"]]
            assert np.array_equal(a.anchor_idx, b["anchor_idx"])


def test_chain_batch_long_reads_wide_window(chaining):
    """ONT-like long reads (~10k anchors per read), lookback 200."""
    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.config import ChainingConfig
    from oracle import oracle

    batch = synth.chaining_reads_hifi(n_reads=6, seed=12, ref_len=5_000_000, mean_len=60_000,
                                      spread=0.1, profile=synth.ONT)
    cfg = ChainingConfig(max_lookback=200, max_gap=5000)
    got = chaining.chain_anchor_batch(batch, cfg)
    want = oracle.chain_batch(batch.read_off, batch.read_pos, batch.ref_pos, batch.length,
                              batch.strand, oracle.penalty_lut(5000, 6.0, 0.05, 0.5), max_lookback=200,
                              threads=6)
    assert np.array_equal(got.n_chains, want.n_chains)
    for r in range(len(batch)):
        for a, b in zip(got.chains(r), want.chains(batch.read_off, r)):
            assert a.score == b["score"] and np.array_equal(a.anchor_idx, b["anchor_idx"])


def test_chain_same_result_alone_and_in_the_mix(chaining):
    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.config import ChainingConfig

    batch = synth.chaining_reads_hifi(n_reads=40, seed=13, ref_len=2_000_000, mean_len=5000)
    cfg = ChainingConfig(max_lookback=50)
    mix = chaining.chain_anchor_batch(batch, cfg)
    for r in (0, 7, 39):
        alone = chaining.chain_anchor_batch(batch.subset([r]), cfg)
        for a, b in zip(alone.chains(0), mix.chains(r)):
            assert a.score == b.score and np.array_equal(a.anchor_idx, b.anchor_idx)


def test_hybrid_contexts_match_reference_golden(chaining):
    from graphmambaformer_b200.config import ChainingConfig
    from graphmambaformer_b200.hybrid import ChainingContext, GraphDistanceOracle
    from graphmambaformer_b200.types import AnchorSet

    with open(os.path.join(GOLDEN, "hybrid_golden.pkl"), "rb") as fh:
        g = pickle.load(fh)
    oracle_g = GraphDistanceOracle(g["edges"], g["n_nodes"], max_hops=3)
    sets, ctxs = [], []
    for rd in g["reads"]:
        a = AnchorSet.from_lists(rd["read_pos"], rd["ref_pos"], rd["length"], rd["strand"],
                                 node_id=rd["node_id"])
        a.score = rd["score"]
        sets.append(a)
        ctxs.append(ChainingContext(oracle=oracle_g if rd["use_oracle"] else None,
                                    backbone=g["backbone"] if rd["use_backbone"] else None,
                                    trust_neural=rd["trust"], learned_transitions=rd["transitions"]))
    chainer = chaining.AffineChainer(ChainingConfig(max_lookback=g["lookback"], max_gap=5000))
    got = chainer.chain_batch(sets, ctxs)
    for r, (chains, want) in enumerate(zip(got, g["chains"])):
        assert len(chains) == len(want), r
        for c, w in zip(chains, want):
            assert c.score == w["score"], (r, c.score, w["score"])
            assert c.strand == w["strand"] and c.is_primary == w["primary"]
            assert (c.read_start, c.read_end, c.ref_start, c.ref_end) == tuple(w["span"])
            assert np.array_equal(c.anchor_idx, w["members"])


def test_empty_reads_and_single_strand(chaining):
    from graphmambaformer_b200.config import ChainingConfig
    from graphmambaformer_b200.types import AnchorSet

    sets = [AnchorSet.empty(), AnchorSet.from_lists([0, 30, 60], [100, 130, 160], [20, 20, 20], [-1, -1, -1])]
    out = chaining.AffineChainer(ChainingConfig()).chain_batch(sets)
    assert out[0] == []
    assert len(out[1]) == 1 and out[1][0].strand == -1 and list(out[1][0].anchor_idx) == [0, 1, 2]


@pytest.mark.parametrize("pinned", [False, True])
@pytest.mark.parametrize("chunks", [None, 1, 3, 7])
def test_chain_session_host_batches_in_runs(chaining, chunks, pinned):
    """The host-buffer session (the e2e path): a batch split into runs of
    whole reads, staged (or, with page-locked columns, copied directly) while
    the previous run chains, gives the oracle's chains; so does a second call
    reusing the buffers, which leaves the first call's result untouched."""
    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.config import ChainingConfig
    from graphmambaformer_b200.session import ChainSession, pin_anchors
    from oracle import oracle

    batch = synth.chaining_reads_hifi(n_reads=60, seed=77, ref_len=2_000_000, mean_len=5000)
    cfg = ChainingConfig(max_lookback=50, max_gap=5000)
    want = oracle.chain_batch(batch.read_off, batch.read_pos, batch.ref_pos, batch.length, batch.strand,
                              oracle.penalty_lut(5000, 6.0, 0.05, 0.5), max_lookback=50, threads=8)
    sess = ChainSession(cfg, "cuda:0")
    src = pin_anchors(batch) if pinned else batch
    if pinned:
        import torch

        assert torch.from_numpy(src.read_pos).is_pinned()
    results = [sess.chain(src, chunks=chunks) for _ in range(2)]
    for got in results:
        assert np.array_equal(got.n_chains, want.n_chains)
        for r in range(len(batch)):
            for a, b in zip(got.chains(r), want.chains(batch.read_off, r)):
                assert a.score == b["score"] and a.is_primary == b["is_primary"]
                assert [a.read_start, a.read_end, a.ref_start, a.ref_end] == [
                    b["read_start"], b["read_end"], b["ref_start"], b["ref_end"]]
                assert np.array_equal(a.anchor_idx, b["anchor_idx"])
    assert sess.h2d_bytes > 0 and sess.d2h_bytes > 0
