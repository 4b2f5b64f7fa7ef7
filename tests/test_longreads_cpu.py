"""The long-read segmentation rule (`longreads.segment_chain`), checked on
the CPU against its statement: kept anchors at least `min_spacing` apart
(the last member always kept), segments tiling the query between the first
and the last anchor, targets padded and clipped to the reference, band
offset at the first anchor, half band clip(32 + |drift| + qlen * b //
1000, 32, 2000), in both modes (fine: 1 kb spacing, b = 20; wide: 8 kb
spacing, b = 250)."""

from __future__ import annotations

import numpy as np
import pytest


@pytest.mark.parametrize("mode", ["fine", "wide"])
def test_segments_follow_the_rule(mode):
    from graphmambaformer_b200.longreads import BASE_BAND, FINE, MAX_BAND, PAD, WIDE, segment_chain

    spacing, per_kb = FINE if mode == "fine" else WIDE
    rng = np.random.default_rng(4)
    for t in range(300):
        n = int(rng.integers(0, 400))
        rp = np.cumsum(rng.integers(1, 300 if mode == "fine" else 900, n))
        fp = rp + int(rng.integers(0, 50_000)) + np.cumsum(rng.integers(-20, 21, n))
        ref_len = int(fp.max() + rng.integers(-100, 1000)) if n else 1000
        segs = segment_chain(rp, fp, ref_len, min_spacing=spacing, band_per_kb=per_kb)
        if n < 2:
            assert segs == []
            continue
        # kept anchors: the starts of the segments, plus the last member
        starts = [s[0] for s in segs]
        assert starts[0] == rp[0]
        assert all(b - a >= spacing for a, b in zip(starts[:-1], starts[1:]))
        for (qs, ql, ts, tl, hb, off), nxt in zip(segs, segs[1:] + [None]):
            qe = qs + ql
            assert ql > 0
            assert qe == (nxt[0] if nxt else rp[-1])  # tiles the query
            u = int(np.flatnonzero(rp == qs)[0])
            v = int(np.flatnonzero(rp == qe)[0])
            assert ts == max(0, fp[u] - PAD) and ts + tl == max(ts, min(ref_len, fp[v] + PAD))
            assert off == fp[u] - ts
            drift = (fp[v] - fp[u]) - ql
            assert hb == int(np.clip(BASE_BAND + abs(drift) + ql * per_kb // 1000, BASE_BAND, MAX_BAND))
