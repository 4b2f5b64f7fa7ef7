"""Pin the CPU oracle to the reference: every golden vector must reproduce
bit for bit (scores, end/start coordinates, CIGARs, chain DP values,
predecessors and chain records).  CPU only."""

from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import oracle

OPS = "=XIDS"


def _load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name))


def _words_to_cigar(words):
    return [(OPS[int(w) & 15], int(w) >> 4) for w in words]


def test_sw_oracle_matches_reference_golden(golden_dir):
    g = _load(golden_dir, "sw_golden.npz")
    B = len(g["half_band"])
    qs = [g["query"][g["query_off"][b]: g["query_off"][b + 1]] for b in range(B)]
    ts = [g["target"][g["target_off"][b]: g["target_off"][b + 1]] for b in range(B)]
    params = g["params"]
    mismatches = []
    for b in range(B):
        p = params[b]
        out = oracle.sw_batch([qs[b]], [ts[b]], int(g["half_band"][b]), int(g["band_offset"][b]),
                              match=p[0], mismatch=p[1], gap_open=p[2], gap_extend=p[3],
                              x_drop=p[4], traceback=True, threads=1)
        exp_cigar = _words_to_cigar(g["cigar"][g["cigar_off"][b]: g["cigar_off"][b + 1]])
        ok = (out.score[0] == g["score"][b] and out.query_end[0] == g["query_end"][b]
              and out.target_end[0] == g["target_end"][b]
              and out.query_start[0] == g["query_start"][b]
              and out.target_start[0] == g["target_start"][b]
              and out.cigars[0] == exp_cigar
              and list(out.counts[0]) == list(g["counts"][b]))
        if not ok:
            mismatches.append((b, str(g["tag"][b])))
    assert not mismatches, mismatches[:10]


def test_sw_oracle_batch_threads_agree(golden_dir):
    g = _load(golden_dir, "sw_golden.npz")
    sel = np.flatnonzero(g["tag"] == "cfg1")
    qs = [g["query"][g["query_off"][b]: g["query_off"][b + 1]] for b in sel]
    ts = [g["target"][g["target_off"][b]: g["target_off"][b + 1]] for b in sel]
    out = oracle.sw_batch(qs, ts, 32, 32, 2, 4, 4, 2, 0, threads=4)
    assert np.array_equal(out.score, g["score"][sel])
    assert np.array_equal(out.query_end, g["query_end"][sel])
    assert np.array_equal(out.target_start, g["target_start"][sel])


def test_chain_dp_oracle_matches_reference_golden(golden_dir):
    g = _load(golden_dir, "chain_golden.npz")
    off = g["dp_off"]
    boff = g["dp_bonus_off"]
    for c in range(len(off) - 1):
        s, e = off[c], off[c + 1]
        lb = int(g["dp_lookback"][c])
        mg = int(g["dp_max_gap"][c])
        lut = oracle.penalty_lut(mg, 6.0, 0.05, 0.5)
        bonus = None
        if g["dp_has_bonus"][c]:
            bonus = g["dp_bonus"][boff[c]: boff[c + 1]].reshape(e - s, lb)
        f, p = oracle.chain_dp(g["dp_read_end"][s:e], g["dp_ref_end"][s:e], g["dp_weight"][s:e],
                               lut, max_lookback=lb, max_gap=mg, bonus=bonus)
        # bit-exact: compare the float64 bit patterns
        assert np.array_equal(f.view(np.int64), g["dp_f"][s:e].view(np.int64)), c
        assert np.array_equal(p, g["dp_parent"][s:e]), c


def test_penalty_lut_matches_reference_lut(golden_dir):
    g = _load(golden_dir, "chain_golden.npz")
    lut = oracle.penalty_lut(5000, 6.0, 0.05, 0.5)
    assert np.array_equal(lut.view(np.int64), g["lut_default"].view(np.int64))


def test_chain_read_oracle_matches_reference_golden(golden_dir):
    g = _load(golden_dir, "chain_golden.npz")
    read_off = g["read_off"]
    lut = g["lut_default"]
    k = 0
    moff = g["chain_members_off"]
    for lb in np.unique(g["read_lookback"]):
        rows = np.flatnonzero(g["read_lookback"] == lb)
        for r in rows:
            s, e = read_off[r], read_off[r + 1]
            out = oracle.chain_batch(np.array([0, e - s]), g["read_pos"][s:e], g["ref_pos"][s:e],
                                     g["length"][s:e], g["strand"][s:e], lut, max_lookback=int(lb))
            got = out.chains(np.array([0, e - s]), 0)
            # the golden chains are stored read by read in read order
            first = int(g["n_chains"][:r].sum())
            n = int(g["n_chains"][r])
            assert len(got) == n, (r, len(got), n)
            for c in range(n):
                gc = first + c
                want = g["chain_members"][moff[gc]: moff[gc + 1]]
                assert got[c]["score"] == g["chain_score"][gc], (r, c)
                assert got[c]["strand"] == g["chain_strand"][gc]
                assert [got[c]["read_start"], got[c]["read_end"], got[c]["ref_start"],
                        got[c]["ref_end"]] == list(g["chain_span"][gc])
                assert got[c]["is_primary"] == bool(g["chain_primary"][gc])
                assert np.array_equal(got[c]["anchor_idx"], want), (r, c)
                k += 1
    assert k == int(g["n_chains"].sum())


def test_chain_known_answer():
    """tests/test_accel.py L347-370 of the reference: three anchors with
    fractional weights."""
    lut = oracle.penalty_lut(5000, 6.0, 0.05, 0.5)
    f, p = oracle.chain_dp([10, 20, 30], [10, 20, 31], [10.5, 9.25, 8.75], lut)
    assert p.tolist() == [-1, 0, 1]
    assert f[0] == 10.5 and f[1] == 10.5 + 9.25


def _levenshtein(a, b):
    prev = list(range(len(b) + 1))
    for i, ca in enumerate(a, 1):
        cur = [i]
        for j, cb in enumerate(b, 1):
            same = ca == cb and 0 <= ca != 5
            cur.append(min(prev[j] + 1, cur[j - 1] + 1, prev[j - 1] + (0 if same else 1)))
        prev = cur
    return prev[-1]


def test_wfa_oracle_matches_reference_golden(golden_dir):
    """oracle_wfa_align against WavefrontAligner.align (distance, CIGAR and
    the over-budget signal) on every golden case."""
    g = _load(golden_dir, "wfa_golden.npz")
    for i in range(len(g["distance"])):
        q = g["q"][g["q_off"][i]: g["q_off"][i + 1]]
        t = g["t"][g["t_off"][i]: g["t_off"][i + 1]]
        d, cigar = oracle.wfa_align(q, t, int(g["max_distance"][i]))
        assert d == g["distance"][i], i
        assert cigar == _words_to_cigar(g["cigar"][g["cigar_off"][i]: g["cigar_off"][i + 1]]), i


def test_wfa_oracle_is_levenshtein():
    """The reference's own property (tests/test_alignment_stages.py L1063-1091):
    distance == Levenshtein, and the CIGAR consumes both sequences with
    exactly `distance` edits."""
    rng = np.random.default_rng(7)
    for _ in range(60):
        a = rng.integers(1, 6, size=int(rng.integers(0, 40))).astype(np.int16)
        b = a.copy().tolist()
        for _ in range(int(rng.integers(0, 6))):
            pos = int(rng.integers(0, len(b) + 1))
            act = int(rng.integers(0, 3))
            if act == 0 and pos < len(b):
                b[pos] = int(rng.integers(1, 6))
            elif act == 1 and pos < len(b):
                b.pop(pos)
            else:
                b.insert(pos, int(rng.integers(1, 6)))
        b = np.array(b, np.int16)
        d, cigar = oracle.wfa_align(a, b, 4096)
        assert d == _levenshtein(a.tolist(), b.tolist())
        assert sum(n for op, n in cigar if op in "=XI") == len(a)
        assert sum(n for op, n in cigar if op in "=XD") == len(b)
        if len(a) and len(b):
            assert sum(n for op, n in cigar if op in "XID") == d


def test_grouped_sw_oracle_matches_reference_xdrop_golden(golden_dir):
    """The batch x-drop rule (extension.py L190-193): each golden batch is one
    group whose row loop stops together; ends, starts and CIGARs match the
    reference's `banded_affine_sw_batch` + `traceback_banded`.  Without the
    group, some pairs stop earlier and some results differ."""
    g = _load(golden_dir, "xdrop_golden.npz")
    differ = 0
    for b in range(len(g["batch_off"]) - 1):
        lo, hi = int(g["batch_off"][b]), int(g["batch_off"][b + 1])
        qs = [g["query"][g["query_off"][p]: g["query_off"][p + 1]] for p in range(lo, hi)]
        ts = [g["target"][g["target_off"][p]: g["target_off"][p + 1]] for p in range(lo, hi)]
        args = (qs, ts, g["half_band"][lo:hi], g["band_offset"][lo:hi], 2.0, 4.0, 6.0, 2.0, float(g["x_drop"][b]))
        out = oracle.sw_batch(*args, group_off=[0, hi - lo])
        alone = oracle.sw_batch(*args)
        for k, p in enumerate(range(lo, hi)):
            assert (float(out.score[k]), int(out.query_end[k]), int(out.target_end[k])) == (
                g["score"][p], g["qe"][p], g["te"][p]), p
            assert (int(out.query_start[k]), int(out.target_start[k])) == (g["qs"][p], g["ts"][p]), p
            assert out.cigars[k] == _words_to_cigar(g["cigar"][g["cigar_off"][p]: g["cigar_off"][p + 1]]), p
            differ += (float(alone.score[k]), int(alone.query_end[k])) != (float(out.score[k]), int(out.query_end[k]))
    assert differ > 0, "the fixture must contain pairs that the group keeps running"


def test_grouped_sw_oracle_edges():
    """Groups of one, x-drop off, and members with empty queries: the group
    rule reduces to the per-pair one where it should, and a group stops no
    later than its last member's query."""
    rng = np.random.default_rng(11)
    qs = [rng.integers(0, 4, int(n)).astype(np.int16) for n in rng.integers(0, 120, 12)]
    qs[3] = np.zeros(0, np.int16)
    ts = [np.concatenate([q, rng.integers(0, 4, 40).astype(np.int16)]) for q in qs]
    hb, off = np.full(12, 16), np.zeros(12, np.int64)
    for xd in (0.0, 5.0, 30.0):
        alone = oracle.sw_batch(qs, ts, hb, off, 2, 4, 6, 2, xd)
        ones = oracle.sw_batch(qs, ts, hb, off, 2, 4, 6, 2, xd, group_off=np.arange(13))
        grouped = oracle.sw_batch(qs, ts, hb, off, 2, 4, 6, 2, xd, group_off=[0, 4, 12])
        for k in range(12):
            assert (ones.score[k], ones.query_end[k], ones.cigars[k]) == (
                alone.score[k], alone.query_end[k], alone.cigars[k])
            if xd == 0.0:
                assert (grouped.score[k], grouped.query_end[k], grouped.cigars[k]) == (
                    alone.score[k], alone.query_end[k], alone.cigars[k])
            assert grouped.score[k] >= alone.score[k]  # a group only runs longer
        assert grouped.score[3] == 0 and grouped.cigars[3] == []
