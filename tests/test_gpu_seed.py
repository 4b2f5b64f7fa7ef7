"""Device minimizer seeding (gmf_seed_count / gmf_seed_fill) against the
reference's MinimizerIndex golden anchors -- every case, both orientations,
reads shorter than k, N runs, max_occ -- and against the host seeding of a
mixed-profile read pool."""

from __future__ import annotations

import numpy as np
import pytest

from test_seed_cpu import golden_cases

pytestmark = pytest.mark.gpu


def test_device_seeding_matches_reference_golden():
    from graphmambaformer_b200.seeding import DeviceMinimizerIndex

    g, refs, reads = golden_cases()
    for case in range(len(refs)):
        k, w, mo = (int(x) for x in g["ref_kw"][case])
        idx = DeviceMinimizerIndex(refs[case], k=k, w=w, max_occ=mo, device="cuda:0")
        qs = [(q, ri, st) for q, (c, ri, st) in enumerate(g["query"]) if c == case]
        rids = sorted({ri for _, ri, _ in qs})
        got = idx.seed([reads[ri] for ri in rids])
        for q, ri, st in qs:
            r = rids.index(ri)
            lo, hi = got.read_off[r], got.read_off[r + 1]
            sel = np.arange(lo, hi)[got.strand[lo:hi] == st]
            s, e = g["anchor_off"][q], g["anchor_off"][q + 1]
            assert np.array_equal(got.read_pos[sel], g["read_pos"][s:e]), (case, q)
            assert np.array_equal(got.ref_pos[sel], g["ref_pos"][s:e]), (case, q)
            assert np.all(got.length[sel] == k)
            # forward anchors come first
            if st > 0 and len(sel):
                assert sel[-1] - lo == len(sel) - 1


def test_device_seeding_matches_host_on_read_pool():
    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.seeding import DeviceMinimizerIndex

    pool = synth.mixed_read_pool(n_reads=150, seed=21, ref_len=2_000_000, max_len=12_000)
    idx = DeviceMinimizerIndex(pool.ref, k=15, w=10, max_occ=200, device="cuda:0")
    got = idx.seed(pool.reads)
    a = pool.anchors
    assert np.array_equal(got.read_off, a.read_off)
    for name in ("read_pos", "ref_pos", "length", "strand"):
        assert np.array_equal(getattr(got, name), getattr(a, name)), name
