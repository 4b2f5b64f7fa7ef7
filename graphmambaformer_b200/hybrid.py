"""Hybrid-mode chaining inputs: gated anchor weights and DP bonus rows.

In the reference's ``hybrid`` pipeline the scoring model runs first, and its
outputs reach the chaining DP through two host-side inputs
(graphmambaformer/alignment/chaining.py L307-481; the graph distances are
L60-114):

* a per-anchor **weight**: the match length, raised by ``ref_path_bias`` on
  the graph backbone, then scaled by an AGNES confidence gate of the neural
  seed score (or by the older linear blend when adaptive scoring is off);
* an optional ``(n, max_lookback)`` **bonus** row per anchor: a decay in the
  hop distance between the two anchors' graph nodes, plus a clipped logit of
  the learned transition probability between the two anchors.

This module computes both for each strand segment in the order the device
sort produces, and the batch driver hands them to the same device DP, peel
and select kernels as fast mode.  The design:

* hop distances come from one frontier BFS that runs from all of a
  segment's distinct nodes at once, on (source, node) pairs held as int64
  keys in sorted arrays;
* the bonus rows are filled by array lookups into the resulting hop table;
* learned transitions are joined to the segment through a table of the
  segment's distinct anchor keys, so each learned entry is looked up once
  instead of every (predecessor, anchor) pair of the window.

Only the floating-point arithmetic is the reference's, in its operation
order and dtypes, because bit-exact DP scores depend on it: the f64 weight
``length (+ bias)`` times the gate ``clip(1 + gain * log(p / (1 - p)))``, the
legacy blend ``0.5 + score`` in the score's own dtype, the decay
``bonus * (1 - hop / max_hops)`` added to zero, and the transition term
``gnn_bonus * clip(log(p / (1 - p)))`` added after it.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import _native
from .config import ChainingConfig

_P_LO = 1e-4
_P_HI = 1.0 - 1e-4


# --------------------------------------------------------------------------- #
# pangenome graph distances
# --------------------------------------------------------------------------- #
def undirected_csr(edge_index: np.ndarray, num_nodes: int) -> tuple[np.ndarray, np.ndarray]:
    """(indptr, neighbours) of the graph with every edge taken both ways."""
    e = np.asarray(edge_index, dtype=np.int64).reshape(2, -1)
    n = max(int(num_nodes), int(e.max()) + 1 if e.size else 0)  # ids past num_nodes still get rows
    ends = np.concatenate([e, e[::-1]], axis=1)  # row 0: from, row 1: to
    by_from = np.argsort(ends[0], kind="stable")
    indptr = np.searchsorted(ends[0][by_from], np.arange(n + 1), side="left").astype(np.int64)
    return indptr, ends[1][by_from]


def pairwise_hops(graph, nodes: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Hop distances among the distinct non-negative ``nodes``.

    ``graph`` is any object with ``indptr``, ``neighbours`` and ``max_hops``
    (this module's :class:`GraphDistanceOracle` or the reference's own).
    Returns (sorted distinct nodes, int16 table): entry [a, b] is the number
    of edges on a shortest path from node a to node b, or -1 when there is
    none of at most ``max_hops`` edges.  All sources advance together, level
    by level, over (source, node) pairs encoded as ``source * N + node``.
    """
    distinct = np.unique(np.asarray(nodes, dtype=np.int64))
    distinct = distinct[distinct >= 0]
    k = len(distinct)
    table = np.full((k, k), -1, dtype=np.int16)
    if k == 0:
        return distinct, table
    indptr = np.asarray(graph.indptr, dtype=np.int64)
    nbr = np.asarray(graph.neighbours, dtype=np.int64)
    n_graph = max(len(indptr) - 1, int(distinct[-1]) + 1)
    table[np.arange(k), np.arange(k)] = 0
    src = np.arange(k, dtype=np.int64)
    at = distinct.copy()
    seen = np.sort(src * n_graph + at)
    for depth in range(1, int(graph.max_hops) + 1):
        inside = at < len(indptr) - 1
        src, at = src[inside], at[inside]
        first = indptr[at]
        deg = indptr[at + 1] - first
        total = int(deg.sum())
        if total == 0:
            break
        # the neighbours of every frontier pair, flattened
        base = np.repeat(first - (np.cumsum(deg) - deg), deg)
        reach_src = np.repeat(src, deg)
        reach = nbr[base + np.arange(total)]
        keys = np.unique(reach_src * n_graph + reach)
        keys = keys[~np.isin(keys, seen, assume_unique=True)]
        if len(keys) == 0:
            break
        seen = np.union1d(seen, keys)
        src, at = keys // n_graph, keys % n_graph
        col = np.searchsorted(distinct, at)
        hit = col < k
        hit[hit] = distinct[col[hit]] == at[hit]
        table[src[hit], col[hit]] = depth
    return distinct, table


class GraphDistanceOracle:
    """Bounded hop distances between pangenome nodes, the interface of the
    reference's ``GraphDistanceOracle`` (chaining.py L60-114): built from an
    edge list, edges usable in both directions, distances up to
    ``max_hops``."""

    def __init__(self, edge_index: np.ndarray, num_nodes: int, max_hops: int = 3):
        self.num_nodes = int(num_nodes)
        self.max_hops = int(max_hops)
        self.indptr, self.neighbours = undirected_csr(edge_index, self.num_nodes)

    def hop_matrix(self, nodes) -> tuple[np.ndarray, dict]:
        """(hop table, node -> row) over the distinct nodes of ``nodes``."""
        distinct, table = pairwise_hops(self, np.asarray(list(nodes), dtype=np.int64))
        return table, {int(v): i for i, v in enumerate(distinct)}


@dataclass
class ChainingContext:
    """Pangenome / AGNES context of one read (chaining.py L264-289)."""

    oracle: Optional[object] = None
    backbone: Optional[np.ndarray] = None
    trust_neural: Optional[bool] = None
    learned_transitions: Optional[dict] = None


# --------------------------------------------------------------------------- #
# one strand segment of a read, in DP order
# --------------------------------------------------------------------------- #
@dataclass
class Segment:
    """Columns of one read's anchors on one strand, sorted by (ref_end,
    read_end): the rows of one DP."""

    read_pos: np.ndarray
    ref_pos: np.ndarray
    length: np.ndarray
    strand: np.ndarray
    node_id: np.ndarray
    score: np.ndarray

    @staticmethod
    def of(anchors, idx: np.ndarray) -> "Segment":
        n = len(anchors.read_pos)
        node = getattr(anchors, "node_id", None)
        score = getattr(anchors, "score", None)
        col = lambda a, fill, dt: (np.asarray(a)[idx] if a is not None and len(a) == n
                                   else np.full(len(idx), fill, dt))
        return Segment(np.asarray(anchors.read_pos)[idx], np.asarray(anchors.ref_pos)[idx],
                       np.asarray(anchors.length)[idx], np.asarray(anchors.strand)[idx],
                       col(node, -1, np.int64), col(score, np.nan, np.float32))

    def __len__(self) -> int:
        return len(self.read_pos)


def sorted_layout(anchors) -> tuple[np.ndarray, int, int]:
    """The device sort's permutation of a read's anchors: + strand, then -
    strand, each by (ref_end, read_end) with ties in input order (types.py
    L144-152 ``for_strand`` + ``sorted_by_ref``); and the two segment sizes."""
    strand = np.asarray(anchors.strand)
    ln = np.asarray(anchors.length, dtype=np.int64)
    read_end = np.asarray(anchors.read_pos, dtype=np.int64) + ln
    ref_end = np.asarray(anchors.ref_pos, dtype=np.int64) + ln
    # one stable sort on (strand group, ref_end, read_end): - strand anchors
    # and strands other than +-1 sort after the + strand ones
    group = np.where(strand == 1, 0, np.where(strand == -1, 1, 2))
    order = np.lexsort((read_end, ref_end, group))
    n_plus = int((strand == 1).sum())
    n_minus = int((strand == -1).sum())
    return order[: n_plus + n_minus].astype(np.int64), n_plus, n_minus


# --------------------------------------------------------------------------- #
# anchor weights (chaining.py L307-412)
# --------------------------------------------------------------------------- #
def confidence_metric(cfg: ChainingConfig, scores: np.ndarray) -> float:
    """AGNES separation of the scored seeds: (mean of confident-good minus
    mean of confident-bad) over the spread of all of them; 0 when the
    spread vanishes."""
    s = np.asarray(scores, dtype=np.float64)
    if s.size == 0:
        return 0.0
    spread = float(s.std())
    if spread <= 1e-6:
        return 0.0
    good = s[s > cfg.high_confidence_prob]
    bad = s[s < cfg.low_confidence_prob]
    mean_good = float(good.mean()) if good.size else 0.0
    mean_bad = float(bad.mean()) if bad.size else 0.0
    return (mean_good - mean_bad) / spread


def trusts_scores(cfg: ChainingConfig, score: np.ndarray) -> bool:
    """The AGNES decision for one segment: adaptive scoring on, a scored-seed
    count within the configured range, and a separation above threshold."""
    if not cfg.adaptive_seed_scoring:
        return False
    scored = np.asarray(score)[np.isfinite(score)]
    if not cfg.min_confidence_anchors <= scored.size <= cfg.max_confidence_anchors:
        return False
    return confidence_metric(cfg, scored) > cfg.confidence_threshold


def gate_factors(cfg: ChainingConfig, score: np.ndarray, scored: np.ndarray) -> np.ndarray:
    """Multiplicative weight gate: clip(1 + gain * logit(p)) for scored seeds,
    1 for the others."""
    p = np.clip(np.asarray(score)[scored].astype(np.float64), _P_LO, _P_HI)
    gate = np.ones(len(score), dtype=np.float64)
    gate[scored] = np.clip(1.0 + cfg.logit_gate_gain * np.log(p / (1.0 - p)), cfg.logit_gate_min,
                           cfg.logit_gate_max)
    return gate


def anchor_weights(cfg: ChainingConfig, seg: Segment, ctx: Optional[ChainingContext]) -> np.ndarray:
    """f64 DP weight of every anchor of the segment."""
    w = np.asarray(seg.length).astype(np.float64)
    if ctx is not None and ctx.backbone is not None:
        backbone = np.asarray(ctx.backbone)
        node = np.asarray(seg.node_id)
        on_path = (node >= 0) & backbone[np.clip(node, 0, len(backbone) - 1)]
        w = w + np.where(on_path, cfg.ref_path_bias, 0.0)
    score = np.asarray(seg.score)
    scored = np.isfinite(score)
    trust = None if ctx is None else ctx.trust_neural
    if not scored.any() or trust is False:
        return w
    if not cfg.adaptive_seed_scoring:  # the older linear blend, in the score's dtype
        blend = score.copy()
        blend[~scored] = 1.0
        return w * (0.5 + blend)
    if trust is True or trusts_scores(cfg, score):
        return w * gate_factors(cfg, score, scored)
    return w


# --------------------------------------------------------------------------- #
# bonus rows (chaining.py L414-481)
# --------------------------------------------------------------------------- #
def _window_pairs(n: int, lookback: int):
    """(anchor, predecessor, column) of every in-range window cell: column c
    of anchor i holds predecessor i - lookback + c."""
    i = np.repeat(np.arange(n, dtype=np.int64), lookback)
    c = np.tile(np.arange(lookback, dtype=np.int64), n)
    j = i - lookback + c
    keep = j >= 0
    return i[keep], j[keep], c[keep]


def _graph_rows(cfg: ChainingConfig, seg: Segment, graph, lookback: int, rows: np.ndarray) -> bool:
    """Adds the hop-distance decay into ``rows``; True when some pair is
    within the graph's hop limit."""
    node = np.asarray(seg.node_id, dtype=np.int64)
    distinct, table = pairwise_hops(graph, node)
    if table.size == 0:
        return False
    local = np.where(node >= 0, np.searchsorted(distinct, np.maximum(node, 0)), -1)
    i, j, c = _window_pairs(len(seg), lookback)
    both = (local[i] >= 0) & (local[j] >= 0)
    hop = np.full(rows.shape, -1, dtype=np.int16)
    hop[i[both], c[both]] = table[local[i[both]], local[j[both]]]
    near = hop >= 0
    decay = 1.0 - np.maximum(hop, 0) / max(cfg.graph_max_hops, 1)
    rows += np.where(near, cfg.graph_bonus * decay, 0.0)
    return bool(near.any())


def _transition_rows(cfg: ChainingConfig, seg: Segment, learned: dict, lookback: int,
                     rows: np.ndarray) -> bool:
    """Adds the learned-transition logits into ``rows`` by joining the
    learned (source key, target key) entries to the segment's anchor keys;
    True when some entry falls inside the window."""
    cols = np.stack([np.asarray(seg.read_pos, np.int64), np.asarray(seg.ref_pos, np.int64),
                     np.asarray(seg.length, np.int64), np.asarray(seg.strand).astype(np.int64)], axis=1)
    uniq, key_of = np.unique(cols, axis=0, return_inverse=True)
    key_of = key_of.reshape(-1)
    slot = {tuple(int(v) for v in row): g for g, row in enumerate(uniq)}
    # anchors of each distinct key, in order (CSR over keys)
    members = np.argsort(key_of, kind="stable")
    first = np.searchsorted(key_of[members], np.arange(len(uniq) + 1))
    src_key, dst_key, prob = [], [], []
    for (ks, kd), p in learned.items():
        a, b = slot.get(tuple(ks)), slot.get(tuple(kd))
        if a is not None and b is not None:
            src_key.append(a)
            dst_key.append(b)
            prob.append(float(p))
    if not prob:
        return False
    # every (source anchor, target anchor) of every matched entry
    sk, dk = np.asarray(src_key), np.asarray(dst_key)
    n_src = first[sk + 1] - first[sk]
    n_dst = first[dk + 1] - first[dk]
    per = n_src * n_dst
    entry = np.repeat(np.arange(len(prob)), per)
    r = np.arange(int(per.sum())) - np.repeat(np.cumsum(per) - per, per)
    src = members[first[sk[entry]] + r // n_dst[entry]]
    dst = members[first[dk[entry]] + r % n_dst[entry]]
    gap = dst - src
    inside = (gap > 0) & (gap <= lookback)
    if not inside.any():
        return False
    p = np.clip(np.asarray(prob, dtype=np.float64)[entry[inside]], _P_LO, _P_HI)
    logit = np.clip(np.log(p / (1.0 - p)), -cfg.gnn_transition_logit_clip, cfg.gnn_transition_logit_clip)
    rows[dst[inside], lookback - gap[inside]] += cfg.gnn_transition_bonus * logit
    return True


def bonus_rows(cfg: ChainingConfig, seg: Segment, ctx: Optional[ChainingContext]) -> Optional[np.ndarray]:
    """The segment's ``(n, max_lookback)`` f64 bonus, or None when neither
    term applies to any window cell."""
    if ctx is None:
        return None
    lookback = max(1, int(cfg.max_lookback))
    rows = np.zeros((len(seg), lookback), dtype=np.float64)
    used = False
    node = np.asarray(seg.node_id)
    if ctx.oracle is not None and cfg.graph_bonus != 0.0 and (node >= 0).any():
        used = _graph_rows(cfg, seg, ctx.oracle, lookback, rows)
    if ctx.trust_neural is True and ctx.learned_transitions and cfg.gnn_transition_bonus != 0.0:
        used = _transition_rows(cfg, seg, ctx.learned_transitions, lookback, rows) or used
    return rows if used else None


# --------------------------------------------------------------------------- #
# batch driver
# --------------------------------------------------------------------------- #
def needs_host_inputs(cfg: ChainingConfig, anchor_sets: Sequence, contexts: Sequence) -> bool:
    """True when some read's weights differ from its anchor lengths or it has
    a bonus (backbone bias, finite neural scores, graph context, learned
    transitions); fast mode runs entirely on the device otherwise."""
    for a, ctx in zip(anchor_sets, contexts):
        if ctx is not None and (ctx.backbone is not None or ctx.oracle is not None
                                or (ctx.trust_neural is True and ctx.learned_transitions)):
            return True
        score = getattr(a, "score", None)
        if score is not None and len(score) and np.isfinite(score).any():
            return True
    return False


def chain_batch_hybrid(chainer, anchor_sets: Sequence, contexts: Sequence, dev: torch.device) -> list:
    """Hybrid-mode chain_batch: weights and bonus rows per strand segment on
    the host, laid out as the device sort would lay them out, then the
    device DP, peel and select."""
    from .chaining import AnchorCSR, fetch_chains, launch_chain_batch, upload_anchors
    from .device import to_device

    cfg = chainer.cfg
    lookback = max(1, int(cfg.max_lookback))
    csr = AnchorCSR.from_sets(anchor_sets)
    A = max(int(csr.read_off[-1]), 1)
    perm = np.zeros(A, np.int32)
    read_end = np.zeros(A, np.int32)
    ref_end = np.zeros(A, np.int32)
    weight = np.zeros(A, np.float64)
    bonus = None
    n_plus = np.zeros(len(anchor_sets), np.int32)
    n_minus = np.zeros(len(anchor_sets), np.int32)
    for r, (a, ctx) in enumerate(zip(anchor_sets, contexts)):
        base = int(csr.read_off[r])
        order, n_plus[r], n_minus[r] = sorted_layout(a)
        at = slice(base, base + len(order))
        perm[at] = order
        ln = np.asarray(a.length)
        read_end[at] = (np.asarray(a.read_pos) + ln)[order]
        ref_end[at] = (np.asarray(a.ref_pos) + ln)[order]
        for lo, hi in ((0, int(n_plus[r])), (int(n_plus[r]), len(order))):
            if hi == lo:
                continue
            seg = Segment.of(a, order[lo:hi])
            weight[base + lo: base + hi] = anchor_weights(cfg, seg, ctx)
            rows = bonus_rows(cfg, seg, ctx)
            if rows is not None:
                if bonus is None:
                    bonus = np.zeros((A, lookback), np.float64)
                bonus[base + lo: base + hi] = rows
    da = upload_anchors(csr, dev)
    keep = [to_device(x, dev) for x in (perm, n_plus, n_minus, read_end, ref_end)]
    layout = _native.GmfSortedAnchors(*[t.data_ptr() for t in keep])
    out = launch_chain_batch(da, cfg, sorted_layout=layout, sorted_weight=to_device(weight, dev),
                             sorted_bonus=None if bonus is None else to_device(bonus, dev))
    res = fetch_chains(out, csr.read_off)
    del keep
    return [res.chains(r) for r in range(len(anchor_sets))]
