"""Test helpers shared by the GPU parity suites."""

from __future__ import annotations

import os

import numpy as np

from conftest import GOLDEN

OPS = "=XIDS"


def load(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def words_to_cigar(words):
    return [(OPS[int(w) & 15], int(w) >> 4) for w in words]


def golden_sw_pairs():
    """The reference's SW golden cases grouped by scoring parameters:
    yields (params tuple, case indices, PairSet)."""
    from graphmambaformer_b200.synth import PairSet

    g = load("sw_golden.npz")
    B = len(g["half_band"])
    params = [tuple(p) for p in g["params"]]
    groups: dict = {}
    for b in range(B):
        groups.setdefault(params[b], []).append(b)
    for p, idx in groups.items():
        qs = [g["query"][g["query_off"][b]: g["query_off"][b + 1]] for b in idx]
        ts = [g["target"][g["target_off"][b]: g["target_off"][b + 1]] for b in idx]
        ps = PairSet.from_lists(qs, ts, g["half_band"][idx], g["band_offset"][idx])
        yield p, np.array(idx), ps, g


def cigar_score(cigar, match, mismatch, gap_open, gap_extend):
    """Score implied by a CIGAR under the reference's affine model (a gap of
    length L costs open + (L-1)*extend)."""
    s = 0
    for op, n in cigar:
        if op == "=":
            s += match * n
        elif op == "X":
            s -= mismatch * n
        elif op in ("I", "D"):
            s -= gap_open + (n - 1) * gap_extend
    return s


def assert_sw_equal(got, want, idx=None, label=""):
    """got: SWResult (GPU); want: oracle SWOut.  Bit-exact on every field."""
    n = len(want.score)
    sel = np.arange(n) if idx is None else idx
    assert np.array_equal(got.score[sel].astype(np.float32), want.score), label
    assert np.array_equal(got.query_end[sel], want.query_end), label
    assert np.array_equal(got.target_end[sel], want.target_end), label
    assert np.array_equal(got.query_start[sel], want.query_start), label
    assert np.array_equal(got.target_start[sel], want.target_start), label
    assert np.array_equal(got.op_counts[sel], want.counts), label
    for k, b in enumerate(sel):
        assert got.cigar(int(b)) == want.cigars[k], (label, int(b))
