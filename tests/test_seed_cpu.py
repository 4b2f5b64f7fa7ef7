"""The host minimizer table and query (synth.MinimizerSketch, the index
builder of the device seeding path) against golden anchors produced by the
reference's own MinimizerIndex (tests/golden/seed_golden.npz)."""

from __future__ import annotations

import numpy as np

from helpers import load


def golden_cases():
    g = load("seed_golden.npz")
    refs = [g["ref"][g["ref_off"][i]: g["ref_off"][i + 1]] for i in range(len(g["ref_off"]) - 1)]
    reads = [g["reads"][g["read_off"][i]: g["read_off"][i + 1]] for i in range(len(g["read_off"]) - 1)]
    return g, refs, reads


def test_host_sketch_matches_reference_minimizer_index():
    from graphmambaformer_b200 import synth

    g, refs, reads = golden_cases()
    sketches = {}
    for q, (case, ri, strand) in enumerate(g["query"]):
        k, w, mo = (int(x) for x in g["ref_kw"][case])
        sk = sketches.setdefault(case, synth.MinimizerSketch(refs[case], k=k, w=w, max_occ=mo))
        codes = reads[ri] if strand > 0 else synth.reverse_complement(reads[ri])
        rp, fp = sk.query(codes)
        s, e = g["anchor_off"][q], g["anchor_off"][q + 1]
        assert np.array_equal(rp, g["read_pos"][s:e]), q
        assert np.array_equal(fp, g["ref_pos"][s:e]), q
        assert np.all(g["length"][s:e] == k)
    assert int(g["anchor_off"][-1]) > 5000
