"""Stage configuration, field for field the reference's dataclasses.

``ChainingConfig`` mirrors graphmambaformer/config.py L661-736 and
``ExtensionConfig`` mirrors L739-767 (same names, same defaults), so a
reference config object can be passed wherever these are accepted (the
engines only read attributes).
"""

from __future__ import annotations

from dataclasses import dataclass


@dataclass
class ChainingConfig:
    max_lookback: int = 64
    max_gap: int = 5_000
    gap_open: float = 6.0
    gap_extend: float = 0.05
    log_coeff: float = 0.5

    graph_bonus: float = 4.0
    graph_max_hops: int = 3
    ref_path_bias: float = 1.5

    adaptive_seed_scoring: bool = True
    confidence_threshold: float = 0.7
    high_confidence_prob: float = 0.7
    low_confidence_prob: float = 0.3
    min_confidence_anchors: int = 5
    max_confidence_anchors: int = 1000
    logit_gate_gain: float = 0.25
    logit_gate_min: float = 0.1
    logit_gate_max: float = 3.0

    gnn_transition_bonus: float = 2.0
    gnn_transition_logit_clip: float = 3.0

    min_chain_score: float = 20.0
    min_chain_anchors: int = 1
    max_chains: int = 8
    secondary_overlap: float = 0.5
    secondary_score_ratio: float = 0.6


@dataclass
class ExtensionConfig:
    algorithm: str = "banded_sw"

    match_score: float = 2.0
    mismatch_penalty: float = 4.0
    gap_open: float = 6.0
    gap_extend: float = 2.0
    x_drop: float = 600.0

    half_band: int = 64
    max_half_band: int = 512

    flank: int = 100
    max_window: int = 32_768
    wfa_max_distance: int = 4_096
