"""Hybrid-mode chaining inputs on the CPU: the weights and bonus terms that
`hybrid.py` computes for each read (backbone bias, AGNES gate, graph
distance decay, learned transitions), fed to the oracle's DP and peel and
the reference's select, give the chains the reference itself produced
(hybrid_golden.pkl, made by `AffineChainer.chain` with a `ChainingContext`).
This pins the host half of hybrid mode without a GPU; the GPU suite checks
the same fixture through the device kernels."""

from __future__ import annotations

import os
import pickle

import numpy as np

from conftest import GOLDEN
from oracle import oracle


def _select(cands, cfg):
    """chaining.py `select` (L579-617): stable sort by -score, cutoff at
    best * ratio once a chain is kept, read-overlap rule against the primary."""
    order = sorted(range(len(cands)), key=lambda k: -cands[k]["score"])
    if not order:
        return []
    cutoff = cands[order[0]]["score"] * cfg.secondary_score_ratio
    kept = []
    for k in order:
        c = cands[k]
        if c["score"] < cutoff and kept:
            break
        overlap = 0.0
        if kept:
            p = kept[0]
            lo, hi = max(c["read_start"], p["read_start"]), min(c["read_end"], p["read_end"])
            if hi > lo:
                den = max(min(c["read_end"] - c["read_start"], p["read_end"] - p["read_start"]), 1)
                overlap = (hi - lo) / den
        if overlap > cfg.secondary_overlap:
            continue
        kept.append(c)
        if len(kept) >= cfg.max_chains:
            break
    return kept


def test_hybrid_inputs_through_the_oracle_match_reference_golden():
    from graphmambaformer_b200.config import ChainingConfig
    from graphmambaformer_b200.hybrid import (ChainingContext, GraphDistanceOracle, Segment, anchor_weights,
                                              bonus_rows, sorted_layout)
    from graphmambaformer_b200.types import AnchorSet

    with open(os.path.join(GOLDEN, "hybrid_golden.pkl"), "rb") as fh:
        g = pickle.load(fh)
    cfg = ChainingConfig(max_lookback=g["lookback"], max_gap=5000)
    lut = oracle.penalty_lut(cfg.max_gap, cfg.gap_open, cfg.gap_extend, cfg.log_coeff)
    graph = GraphDistanceOracle(g["edges"], g["n_nodes"], max_hops=3)
    n_bonus = 0
    for r, (rd, want) in enumerate(zip(g["reads"], g["chains"])):
        a = AnchorSet.from_lists(rd["read_pos"], rd["ref_pos"], rd["length"], rd["strand"],
                                 node_id=rd["node_id"])
        a.score = rd["score"]
        ctx = ChainingContext(oracle=graph if rd["use_oracle"] else None,
                              backbone=g["backbone"] if rd["use_backbone"] else None,
                              trust_neural=rd["trust"], learned_transitions=rd["transitions"])
        order, npl, nmi = sorted_layout(a)
        rp = np.asarray(a.read_pos, np.int64)
        fp = np.asarray(a.ref_pos, np.int64)
        ln = np.asarray(a.length, np.int64)
        cands = []
        for strand, s0, n in ((1, 0, npl), (-1, npl, nmi)):
            if n == 0:
                continue
            idx = order[s0: s0 + n]
            seg = Segment.of(a, idx)
            w = anchor_weights(cfg, seg, ctx)
            b = bonus_rows(cfg, seg, ctx)
            n_bonus += b is not None
            f, parent = oracle.chain_dp(rp[idx] + ln[idx], fp[idx] + ln[idx], w, lut, cfg.max_lookback,
                                        cfg.max_gap, bonus=b)
            cands += oracle.chain_backtrack(f, parent, rp[idx], rp[idx] + ln[idx], fp[idx], fp[idx] + ln[idx],
                                            idx, strand, cfg.min_chain_anchors, cfg.min_chain_score)
        got = _select(cands, cfg)
        assert len(got) == len(want), r
        for k, (c, w_) in enumerate(zip(got, want)):
            assert c["score"] == w_["score"], (r, k)
            assert c["strand"] == w_["strand"] and (k == 0) == bool(w_["primary"])
            assert (c["read_start"], c["read_end"], c["ref_start"], c["ref_end"]) == tuple(w_["span"])
            assert np.array_equal(c["anchor_idx"], w_["members"]), (r, k)
    assert n_bonus > 0, "the fixture must exercise the bonus terms"
