"""The stage-level drop-in against the reference pipeline's own output.

``pipeline_golden.pkl`` holds what the reference's
``FastAlignmentPipeline.align`` (graphmambaformer/alignment/pipeline.py
L438-512) returned with its stock CPU stage objects, in both extension
algorithms: per read the seed stage's anchors, the chains, and the records.
Here the B200 stage objects take the place of ``pipeline.chainer`` and
``pipeline.extender`` (pipeline.py L222-231) and run the fast pipeline's
steps on those anchors -- ``chain_batch`` over the batch (L344-351), one
``extend_chains`` per read (L353-363), margin MAPQ and records per read
(L486-511) -- and every chain and record must equal the reference's: f64
chain scores, spans, anchor indices, primary flags, CIGARs, MAPQs."""

from __future__ import annotations

import os
import pickle
from dataclasses import fields

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(GOLDEN, "pipeline_golden.pkl"), "rb") as fh:
        return pickle.load(fh)


def _configs(run):
    from graphmambaformer_b200.config import ChainingConfig, ExtensionConfig

    cc = ChainingConfig(**{f.name: run["config"]["chaining"][f.name] for f in fields(ChainingConfig)
                           if f.name in run["config"]["chaining"]})
    ec = ExtensionConfig(**{f.name: run["config"]["extension"][f.name] for f in fields(ExtensionConfig)
                            if f.name in run["config"]["extension"]})
    return cc, ec


@pytest.mark.parametrize("algorithm", ["banded_sw", "wfa"])
def test_fast_pipeline_with_b200_stages_matches_reference_records(golden, algorithm):
    from graphmambaformer_b200.chaining import AffineChainer
    from graphmambaformer_b200.extension import ExtensionEngine
    from graphmambaformer_b200.records import read_alignments
    from graphmambaformer_b200.synth import decode_bases
    from graphmambaformer_b200.types import AnchorSet

    run = golden["runs"][algorithm]
    cc, ec = _configs(run)
    ref_str = decode_bases(golden["ref"])
    reads, ids = golden["reads"], golden["ids"]
    sets = []
    for read, g in zip(reads, run["reads"]):
        a = g["anchors"]
        sets.append(AnchorSet.from_lists(a[:, 0], a[:, 1], a[:, 2], a[:, 3], read_len=len(read),
                                         ref_len=len(ref_str)))
    chainer = AffineChainer(cc, backend="b200", device="cuda:0")
    extender = ExtensionEngine(ec, device="cuda:0")
    chains = chainer.chain_batch(sets, [None] * len(sets), device="cuda:0")
    checked = 0
    for r, (read, g) in enumerate(zip(reads, run["reads"])):
        assert len(chains[r]) == len(g["chains"]), r
        for c, w in zip(chains[r], g["chains"]):
            assert c.score == w["score"] and c.strand == w["strand"] and c.is_primary == w["is_primary"], r
            assert (c.read_start, c.read_end, c.ref_start, c.ref_end) == w["span"], r
            assert np.array_equal(np.asarray(c.anchor_idx, np.int64), w["anchor_idx"]), r
        exts = extender.extend_chains(read, chains[r], sets[r], ref_str) if chains[r] else []
        got = read_alignments(ids[r], len(read), sets[r], chains[r], exts, ref_id=0, max_mapq=60).records
        assert len(got) == len(g["records"]), r
        for x, w in zip(got, g["records"]):
            have = dict(ref_id=x.ref_id, ref_start=x.ref_start, ref_end=x.ref_end, strand=x.strand, mapq=x.mapq,
                        chain_score=x.chain_score, alignment_score=x.alignment_score,
                        cigar=[(op, int(n)) for op, n in x.cigar], is_mapped=x.is_mapped, is_primary=x.is_primary,
                        is_supplementary=x.is_supplementary, n_anchors=x.n_anchors, n_chains=x.n_chains,
                        node_id=x.node_id)
            if not w["is_mapped"]:  # the unmapped record's span and id fields are the dataclass defaults
                have = {k: v for k, v in have.items() if k in ("mapq", "cigar", "is_mapped", "is_primary")}
                w = {k: w[k] for k in have}
            assert have == w, (r, have, w)
            checked += 1
    assert checked == sum(len(g["records"]) for g in run["reads"])
    assert sum(len(c) > 1 for c in chains) > 0  # secondary chains were exercised


def test_batched_extension_equals_per_read_calls_on_pipeline_reads(golden):
    """extend_batch (one launch for the batch) gives what the pipeline's
    per-read extend_chains calls give."""
    from graphmambaformer_b200.chaining import AffineChainer
    from graphmambaformer_b200.extension import ExtensionEngine
    from graphmambaformer_b200.synth import decode_bases
    from graphmambaformer_b200.types import AnchorSet

    run = golden["runs"]["banded_sw"]
    cc, ec = _configs(run)
    ref_str = decode_bases(golden["ref"])
    sets = [AnchorSet.from_lists(g["anchors"][:, 0], g["anchors"][:, 1], g["anchors"][:, 2], g["anchors"][:, 3],
                                 read_len=len(rd), ref_len=len(ref_str)) for rd, g in zip(golden["reads"], run["reads"])]
    chains = AffineChainer(cc, backend="b200", device="cuda:0").chain_batch(sets, device="cuda:0")
    eng = ExtensionEngine(ec, device="cuda:0")
    batched = eng.extend_batch(golden["reads"], chains, sets, ref_str)
    for r, rd in enumerate(golden["reads"]):
        one = eng.extend_chains(rd, chains[r], sets[r], ref_str) if chains[r] else []
        assert [(e.score, e.cigar, e.ref_start, e.ref_end) for e in batched[r]] == \
            [(e.score, e.cigar, e.ref_start, e.ref_end) for e in one], r
