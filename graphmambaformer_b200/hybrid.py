"""Hybrid-mode chaining inputs: gated anchor weights and DP bonus terms.

In the reference's ``hybrid`` pipeline the model runs first and its outputs
change only two DP inputs, both computed on the host before the DP
(graphmambaformer/alignment/chaining.py L307-481):

* the per-anchor **weight** -- match length, plus ``ref_path_bias`` on the
  graph backbone, times an AGNES confidence gate of the neural seed score;
* an optional ``(n, max_lookback)`` **bonus** -- graph-distance decay between
  anchor nodes plus learned transition logits.

They are evaluated here with numpy in the reference's order of operations and
dtypes, in the per-strand sorted order the device sort produces, and handed to
the same device DP / peel / select kernels as fast mode.
"""

from __future__ import annotations

from collections import deque
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import _native
from .config import ChainingConfig


class GraphDistanceOracle:
    """Bounded hop distances between pangenome nodes (chaining.py L60-114):
    depth-limited BFS over an undirected CSR adjacency."""

    def __init__(self, edge_index: np.ndarray, num_nodes: int, max_hops: int = 3):
        self.num_nodes = int(num_nodes)
        self.max_hops = int(max_hops)
        e = np.asarray(edge_index, dtype=np.int64).reshape(2, -1)
        src = np.concatenate([e[0], e[1]])
        dst = np.concatenate([e[1], e[0]])
        order = np.argsort(src, kind="stable")
        self.neighbours = dst[order]
        counts = np.bincount(src, minlength=self.num_nodes)
        self.indptr = np.zeros(self.num_nodes + 1, dtype=np.int64)
        np.cumsum(counts, out=self.indptr[1:])

    def _bfs(self, source: int) -> dict:
        seen = {source: 0}
        queue = deque([source])
        while queue:
            node = queue.popleft()
            depth = seen[node]
            if depth >= self.max_hops:
                continue
            for nbr in self.neighbours[self.indptr[node]: self.indptr[node + 1]]:
                nbr = int(nbr)
                if nbr not in seen:
                    seen[nbr] = depth + 1
                    queue.append(nbr)
        return seen

    def hop_matrix(self, nodes) -> tuple[np.ndarray, dict]:
        distinct = sorted({int(n) for n in nodes if n >= 0})
        index = {node: i for i, node in enumerate(distinct)}
        hops = np.full((len(distinct), len(distinct)), -1, dtype=np.int16)
        for node, row in index.items():
            for reached, depth in self._bfs(node).items():
                col = index.get(reached)
                if col is not None:
                    hops[row, col] = depth
        return hops, index


@dataclass
class ChainingContext:
    """Pangenome / AGNES context of one read (chaining.py L264-289)."""

    oracle: Optional[GraphDistanceOracle] = None
    backbone: Optional[np.ndarray] = None
    trust_neural: Optional[bool] = None
    learned_transitions: Optional[dict] = None


# --------------------------------------------------------------------------- #
# weights (chaining.py L307-412)
# --------------------------------------------------------------------------- #
def seed_confidence(cfg: ChainingConfig, scores: np.ndarray) -> float:
    if scores.size == 0:
        return 0.0
    scores = np.asarray(scores, dtype=np.float64)
    high = scores[scores > cfg.high_confidence_prob]
    low = scores[scores < cfg.low_confidence_prob]
    mu_high = float(high.mean()) if high.size else 0.0
    mu_low = float(low.mean()) if low.size else 0.0
    sigma = float(scores.std())
    if sigma <= 1e-6:
        return 0.0
    return (mu_high - mu_low) / sigma


def trust_neural_scores(cfg: ChainingConfig, anchors) -> bool:
    if not cfg.adaptive_seed_scoring:
        return False
    finite = np.isfinite(anchors.score)
    n = int(finite.sum())
    if not (cfg.min_confidence_anchors <= n <= cfg.max_confidence_anchors):
        return False
    return seed_confidence(cfg, anchors.score[finite]) > cfg.confidence_threshold


def logit_gate(cfg: ChainingConfig, score: np.ndarray, finite: np.ndarray) -> np.ndarray:
    gate = np.ones(len(score), dtype=np.float64)
    p = np.clip(score[finite].astype(np.float64), 1e-4, 1.0 - 1e-4)
    logit = np.log(p / (1.0 - p))
    gate[finite] = np.clip(1.0 + cfg.logit_gate_gain * logit, cfg.logit_gate_min, cfg.logit_gate_max)
    return gate


def weights(cfg: ChainingConfig, anchors, ctx: Optional[ChainingContext]) -> np.ndarray:
    """Per-anchor chain weight of already strand-split, sorted anchors."""
    weight = anchors.length.astype(np.float64)
    if ctx is not None and ctx.backbone is not None:
        on_path = (anchors.node_id >= 0) & ctx.backbone[np.clip(anchors.node_id, 0, len(ctx.backbone) - 1)]
        weight = weight + on_path * cfg.ref_path_bias
    finite = np.isfinite(anchors.score)
    if not finite.any():
        return weight
    trust = None if ctx is None else ctx.trust_neural
    if trust is False:
        return weight
    if cfg.adaptive_seed_scoring:
        if trust is True:
            return weight * logit_gate(cfg, anchors.score, finite)
        if trust_neural_scores(cfg, anchors):
            return weight * logit_gate(cfg, anchors.score, finite)
        return weight
    scores = np.where(finite, anchors.score, 1.0)
    return weight * (0.5 + scores)


# --------------------------------------------------------------------------- #
# bonus (chaining.py L414-481)
# --------------------------------------------------------------------------- #
def graph_bonus(cfg: ChainingConfig, anchors, ctx: Optional[ChainingContext]) -> Optional[np.ndarray]:
    if ctx is None:
        return None
    n = len(anchors)
    lookback = max(1, cfg.max_lookback)
    rows = np.arange(n)[:, None]
    cols = rows - lookback + np.arange(lookback)[None, :]
    bonus = np.zeros((n, lookback), dtype=np.float64)
    has_bonus = False
    if ctx.oracle is not None and cfg.graph_bonus != 0.0 and (anchors.node_id >= 0).any():
        hops, index = ctx.oracle.hop_matrix(anchors.node_id)
        if hops.size:
            local = np.array([index.get(int(node), -1) for node in anchors.node_id], dtype=np.int64)
            ccols = np.clip(cols, 0, n - 1)
            valid = (cols >= 0) & (local[rows] >= 0) & (local[ccols] >= 0)
            hop = np.full((n, lookback), -1, dtype=np.int16)
            src = local[rows.repeat(lookback, axis=1)][valid]
            dst = local[ccols][valid]
            hop[valid] = hops[src, dst]
            decay = 1.0 - np.clip(hop, 0, None) / max(cfg.graph_max_hops, 1)
            bonus += np.where(hop >= 0, cfg.graph_bonus * decay, 0.0)
            has_bonus = bool((hop >= 0).any())
    if ctx.trust_neural is True and ctx.learned_transitions and cfg.gnn_transition_bonus != 0.0:
        keys = [(int(anchors.read_pos[i]), int(anchors.ref_pos[i]), int(anchors.length[i]),
                 int(anchors.strand[i])) for i in range(n)]
        for dst in range(n):
            lo = max(0, dst - lookback)
            offset = lookback - (dst - lo)
            for slot, src in enumerate(range(lo, dst), start=offset):
                probability = ctx.learned_transitions.get((keys[src], keys[dst]))
                if probability is None:
                    continue
                p = np.clip(float(probability), 1e-4, 1.0 - 1e-4)
                logit = np.clip(np.log(p / (1.0 - p)), -cfg.gnn_transition_logit_clip,
                                cfg.gnn_transition_logit_clip)
                bonus[dst, slot] += cfg.gnn_transition_bonus * logit
                has_bonus = True
    return bonus if has_bonus else None


# --------------------------------------------------------------------------- #
# batch driver
# --------------------------------------------------------------------------- #
def needs_host_inputs(cfg: ChainingConfig, anchor_sets: Sequence, contexts: Sequence) -> bool:
    """True when some read's weights differ from its anchor lengths or it has
    a bonus term (backbone bias, finite neural scores, graph oracle, learned
    transitions)."""
    for a, ctx in zip(anchor_sets, contexts):
        if ctx is not None and (ctx.backbone is not None or ctx.oracle is not None
                                or (ctx.trust_neural is True and ctx.learned_transitions)):
            return True
        score = getattr(a, "score", None)
        if score is not None and len(score) and np.isfinite(score).any():
            return True
    return False


class _Sub:
    """Minimal AnchorSet view (columns re-indexed) accepted by weights/bonus."""

    def __init__(self, a, idx):
        self.read_pos = np.asarray(a.read_pos)[idx]
        self.ref_pos = np.asarray(a.ref_pos)[idx]
        self.length = np.asarray(a.length)[idx]
        self.strand = np.asarray(a.strand)[idx]
        self.node_id = np.asarray(a.node_id)[idx]
        self.score = np.asarray(a.score)[idx]

    def __len__(self) -> int:
        return len(self.read_pos)


def sorted_layout(a) -> tuple[np.ndarray, int, int]:
    """for_strand(+1), for_strand(-1), each sorted_by_ref: the permutation of
    the read's anchors the device sort produces, and the two segment sizes."""
    strand = np.asarray(a.strand)
    read_end = np.asarray(a.read_pos).astype(np.int64) + np.asarray(a.length)
    ref_end = np.asarray(a.ref_pos).astype(np.int64) + np.asarray(a.length)
    parts = []
    for s in (1, -1):
        idx = np.flatnonzero(strand == s)
        order = np.lexsort((read_end[idx], ref_end[idx]))
        parts.append(idx[order])
    return np.concatenate(parts).astype(np.int64), len(parts[0]), len(parts[1])


def chain_batch_hybrid(chainer, anchor_sets: Sequence, contexts: Sequence, dev: torch.device) -> list:
    from .chaining import AnchorCSR, fetch_chains, launch_chain_batch, upload_anchors
    from .device import to_device

    cfg = chainer.cfg
    lb = max(1, int(cfg.max_lookback))
    csr = AnchorCSR.from_sets(anchor_sets)
    A = int(csr.read_off[-1])
    perm = np.zeros(max(A, 1), np.int32)
    re_s = np.zeros(max(A, 1), np.int32)
    fe_s = np.zeros(max(A, 1), np.int32)
    w_s = np.zeros(max(A, 1), np.float64)
    bonus = np.zeros((max(A, 1), lb), np.float64)
    n_plus = np.zeros(len(anchor_sets), np.int32)
    n_minus = np.zeros(len(anchor_sets), np.int32)
    any_bonus = False
    for r, (a, ctx) in enumerate(zip(anchor_sets, contexts)):
        a0 = int(csr.read_off[r])
        order, npl, nmi = sorted_layout(a)
        n_plus[r], n_minus[r] = npl, nmi
        perm[a0: a0 + len(order)] = order
        re_s[a0: a0 + len(order)] = (np.asarray(a.read_pos) + np.asarray(a.length))[order]
        fe_s[a0: a0 + len(order)] = (np.asarray(a.ref_pos) + np.asarray(a.length))[order]
        for seg0, seg_n in ((0, npl), (npl, nmi)):
            if seg_n == 0:
                continue
            sub = _Sub(a, order[seg0: seg0 + seg_n])
            w_s[a0 + seg0: a0 + seg0 + seg_n] = weights(cfg, sub, ctx)
            b = graph_bonus(cfg, sub, ctx)
            if b is not None:
                bonus[a0 + seg0: a0 + seg0 + seg_n] = b
                any_bonus = True
    da = upload_anchors(csr, dev)
    keep = [to_device(x, dev) for x in (perm, n_plus, n_minus, re_s, fe_s)]
    layout = _native.GmfSortedAnchors(*[t.data_ptr() for t in keep])
    w_dev = to_device(w_s, dev)
    b_dev = to_device(bonus, dev) if any_bonus else None
    out = launch_chain_batch(da, cfg, sorted_layout=layout, sorted_weight=w_dev, sorted_bonus=b_dev)
    res = fetch_chains(out, csr.read_off)
    del keep
    return [res.chains(r) for r in range(len(anchor_sets))]
