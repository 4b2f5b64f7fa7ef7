"""The two shortcuts of the device peel, checked on the CPU against the
reference's loops (chaining.py L530-576 `_backtrack`, L579-617 `select`):

* walk starts: a node with a child of strictly higher f is claimed before its
  turn, so the walk may skip it -- the walks (members, stop nodes, order) are
  those of the full rank order;
* select: only the first maximum and the candidates at or above
  cutoff = best * ratio can be visited before the scan stops, so sorting and
  scanning only those keeps the same chains.

DP values and predecessors come from the oracle (ties included)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle


def _walks(f, parent, order):
    """The reference's claimed-mask walk over starts in the given order."""
    claimed = np.zeros(len(f), bool)
    out = []
    for i in order:
        if claimed[i]:
            continue
        members, node = [], i
        while node >= 0 and not claimed[node]:
            claimed[node] = True
            members.append(node)
            node = parent[node]
        out.append((i, tuple(members), node))
    return out


def _segments():
    lut = oracle.penalty_lut(5000, 6.0, 0.05, 0.5)
    rng = np.random.default_rng(5)
    for t in range(200):
        n = int(rng.integers(1, 250))
        re = np.sort(rng.integers(1, 3 * n + 2, n))
        fe = np.sort(rng.integers(1, 3 * n + 2, n))
        w = np.full(n, 15.0) if t % 3 == 0 else rng.integers(5, 30, n).astype(float)  # ties
        yield oracle.chain_dp(re, fe, w, lut, int(rng.choice([1, 4, 16, 50])), 5000)
    from graphmambaformer_b200 import synth

    cb = synth.chaining_reads_hifi(n_reads=6, seed=3, ref_len=2_000_000, mean_len=6000)
    for r in range(len(cb)):
        s, e = cb.read_off[r], cb.read_off[r + 1]
        for sd in (1, -1):
            m = cb.strand[s:e] == sd
            ln = cb.length[s:e][m]
            re, fe = (cb.read_pos[s:e] + cb.length[s:e])[m], (cb.ref_pos[s:e] + cb.length[s:e])[m]
            o = np.lexsort((re, fe))
            yield oracle.chain_dp(re[o], fe[o], ln[o].astype(float), lut, 50, 5000)


def test_skipping_dominated_starts_keeps_every_walk():
    n_seg = skipped = 0
    for f, parent in _segments():
        n = len(f)
        full = sorted(range(n), key=lambda x: (-f[x], x))  # argsort(-f), stable
        dom = np.zeros(n, bool)
        c = np.nonzero(parent >= 0)[0]
        dom[parent[c][f[c] > f[parent[c]]]] = True
        assert _walks(f, parent, full) == _walks(f, parent, [x for x in full if not dom[x]])
        n_seg += 1
        skipped += int(dom.sum())
    assert n_seg > 200 and skipped > 1000


def _select_full(score, span, ratio, sec, mc):
    """chaining.py `select`: stable sort by -score, cutoff, primary overlap."""
    order = sorted(range(len(score)), key=lambda c: (-score[c], c))
    cutoff = score[order[0]] * ratio
    kept = []
    for c in order:
        if score[c] < cutoff and kept:
            break
        overlap = 0.0
        if kept:
            x, y = span[c], span[kept[0]]
            lo, hi = max(x[0], y[0]), min(x[1], y[1])
            if hi > lo:
                overlap = (hi - lo) / max(min(x[1] - x[0], y[1] - y[0]), 1)
        if overlap > sec:
            continue
        kept.append(c)
        if len(kept) >= mc:
            break
    return kept


def _select_visitable(score, span, ratio, sec, mc):
    best = min(range(len(score)), key=lambda c: (-score[c], c))
    cutoff = score[best] * ratio
    cand = [c for c in range(len(score)) if c == best or score[c] >= cutoff]
    sub_score = [score[c] for c in cand]
    sub_span = [span[c] for c in cand]
    return [cand[k] for k in _select_full(sub_score, sub_span, ratio, sec, mc)]


@pytest.mark.parametrize("ratio", [0.0, 0.6, 1.0, 1.5, -0.5])
@pytest.mark.parametrize("sec", [0.5, 0.0, -0.1, 1.0])
def test_select_over_visitable_candidates_keeps_the_same_chains(ratio, sec):
    rng = np.random.default_rng(int(100 * ratio + 1000 * sec) % 2**31)
    for t in range(150):
        n = int(rng.integers(1, 40))
        if t % 4 == 0:
            score = rng.integers(-5, 5, n).astype(float)  # ties and negative scores
        else:
            score = rng.normal(30, 20, n)
        starts = rng.integers(0, 1000, n)
        span = [(int(s), int(s + rng.integers(1, 400))) for s in starts]
        for mc in (1, 3, 8):
            assert _select_full(score, span, ratio, sec, mc) == _select_visitable(score, span, ratio, sec, mc)
