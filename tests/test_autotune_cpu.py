"""Host logic of the batched-form autotuner: the descent over scheduling
knobs, the C struct round trip, the workload signature and the JSON cache."""

from __future__ import annotations

import numpy as np

from graphmambaformer_b200 import autotune
from graphmambaformer_b200.autotune import DEFAULT, SwTuning


def test_coordinate_descent_finds_the_cheapest_valid_setting():
    # a fake cost with its minimum at (29, 253, (2, 4, 8), 2, 1); one setting is rejected
    target = SwTuning(29, 253, (2, 4, 8), 2, 1)

    def evaluate(t: SwTuning):
        if t.l8_max_w == 125 and t.l16_max_w == 125:
            return None  # rejected (e.g. results differed)
        cost = 10.0
        cost += abs(t.l8_max_w - target.l8_max_w) / 10 + abs(t.l16_max_w - target.l16_max_w) / 100
        cost += 0 if t.coop_min_strips == target.coop_min_strips else 3
        cost += 0 if t.warps_per_block == target.warps_per_block else 1
        return cost

    best, ms, trials = autotune.coordinate_descent(DEFAULT, evaluate, passes=3)
    assert best == target and ms == 10.0
    assert all(t.valid() for t, _ in trials)
    assert len({t for t, _ in trials}) == len(trials)  # each setting evaluated once


def test_invalid_settings_are_never_tried():
    seen = []

    def evaluate(t):
        seen.append(t)
        return 1.0

    autotune.coordinate_descent(SwTuning(61, 61, (4, 8, 16), 4, 1), evaluate, passes=1)
    assert all(t.l8_max_w <= t.l16_max_w for t in seen)


def test_struct_round_trip():
    t = SwTuning(29, 253, (2, 0, 8), 3, 0)
    assert SwTuning.from_c(t.to_c()) == t
    assert not SwTuning(130, 125).valid() and not SwTuning(warps_per_block=5).valid()


def test_signature_is_coarse_and_stable():
    rng = np.random.default_rng(0)
    ql = rng.integers(150, 20_000, size=5000)
    hb = np.clip(32 + ql // 50, 32, 500)
    s1 = autotune.signature(ql, hb)
    s2 = autotune.signature(ql[rng.permutation(len(ql))], hb[rng.permutation(len(hb))] * 0 + hb)
    assert s1 == autotune.signature(ql.copy(), hb.copy())
    assert isinstance(s2, str) and s1


def test_cache_round_trip(tmp_path):
    path = str(tmp_path / "tune.json")
    c = autotune.TuningCache(path)
    assert c.get("B200", "sig") is None
    t = SwTuning(29, 253, (2, 4, 8), 2, 1)
    c.put("B200", "sig", t)
    assert autotune.TuningCache(path).get("B200", "sig") == t
