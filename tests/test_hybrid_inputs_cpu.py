"""Hybrid-mode DP inputs on the CPU, pinned to the reference's own outputs.

``hybrid_inputs_golden.pkl`` holds ``AffineChainer._weights`` and
``AffineChainer._graph_bonus`` (graphmambaformer/alignment/chaining.py
L307-481) evaluated by the reference on 60 strand-sorted anchor segments:
random graphs with breaks and shortcuts, hop limits 2-4, lookbacks 1-64,
every AGNES trust decision, the legacy linear blend, duplicated anchor keys
and learned-transition entries outside the segment or the window.  The
weights and bonus rows of ``graphmambaformer_b200.hybrid`` must equal them
bit for bit (they feed a float64 DP whose scores are compared exactly)."""

from __future__ import annotations

import os
import pickle
from dataclasses import replace

import numpy as np
import pytest

from conftest import GOLDEN


def _cases():
    with open(os.path.join(GOLDEN, "hybrid_inputs_golden.pkl"), "rb") as fh:
        return pickle.load(fh)["cases"]


@pytest.mark.parametrize("k", range(60))
def test_weights_and_bonus_rows_match_reference(k):
    from graphmambaformer_b200.config import ChainingConfig
    from graphmambaformer_b200.hybrid import (ChainingContext, GraphDistanceOracle, Segment, anchor_weights,
                                              bonus_rows)

    c = _cases()[k]
    cfg = replace(ChainingConfig(), **c["cfg"])
    seg = Segment(c["read_pos"], c["ref_pos"], c["length"], c["strand"], c["node_id"], c["score"])
    graph = GraphDistanceOracle(c["edges"], c["n_nodes"], max_hops=c["max_hops"]) if c["use_oracle"] else None
    ctx = ChainingContext(oracle=graph, backbone=c["backbone"], trust_neural=c["trust"],
                          learned_transitions=c["transitions"])
    w = anchor_weights(cfg, seg, ctx)
    assert w.dtype == np.float64
    assert np.array_equal(w.view(np.int64), np.asarray(c["weight"], np.float64).view(np.int64))
    b = bonus_rows(cfg, seg, ctx)
    if c["bonus"] is None:
        assert b is None
    else:
        assert b is not None and b.shape == c["bonus"].shape
        assert np.array_equal(b.view(np.int64), c["bonus"].view(np.int64))


def test_hop_table_matches_breadth_first_search():
    """The all-sources frontier BFS against a plain queue BFS per source on a
    random graph with self loops, repeated edges and isolated nodes."""
    from collections import deque

    from graphmambaformer_b200.hybrid import GraphDistanceOracle

    rng = np.random.default_rng(3)
    n = 300
    edges = rng.integers(0, n - 20, size=(2, 500))
    edges[:, :5] = [[7, 7, 8, 9, 9], [7, 8, 7, 10, 10]]
    for hops in (0, 1, 2, 3, 5):
        g = GraphDistanceOracle(edges, n, max_hops=hops)
        nodes = rng.integers(0, n, size=60)
        table, index = g.hop_matrix(nodes)
        adj = [[] for _ in range(n)]
        for a, b in edges.T:
            adj[a].append(b)
            adj[b].append(a)
        for u, row in index.items():
            dist = {u: 0}
            q = deque([u])
            while q:
                x = q.popleft()
                if dist[x] == hops:
                    continue
                for y in adj[x]:
                    if y not in dist:
                        dist[y] = dist[x] + 1
                        q.append(y)
            for v, col in index.items():
                assert table[row, col] == dist.get(v, -1), (hops, u, v)
