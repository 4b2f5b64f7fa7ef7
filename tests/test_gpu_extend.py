"""Stage-level parity of ExtensionEngine.extend_chains (window placement, band
widening, strand handling, soft clips, forward-reference coordinates)."""

from __future__ import annotations

import numpy as np
import pytest

from helpers import load, words_to_cigar

pytestmark = pytest.mark.gpu


def test_extend_chains_matches_reference_golden():
    from graphmambaformer_b200.config import ExtensionConfig
    from graphmambaformer_b200.extension import ExtensionEngine
    from graphmambaformer_b200.synth import decode_bases
    from graphmambaformer_b200.types import AnchorSet, Chain

    g = load("extend_golden.npz")
    ref = decode_bases(g["ref"])
    eng = ExtensionEngine(ExtensionConfig())
    off = g["read_off"]
    reads, chains, anchors = [], [], []
    for k in range(len(off) - 1):
        read = decode_bases(g["reads"][off[k]: off[k + 1]])
        row = g["chains"][k]
        rp, fp, ln, strand = row[0:3], row[3:6], row[6:9], int(row[9])
        a = AnchorSet.from_lists(rp, fp, ln, np.full(3, strand, np.int8))
        c = Chain(anchor_idx=np.arange(3), score=40.0, strand=strand, read_start=int(rp.min()),
                  read_end=int((rp + ln).max()), ref_start=int(fp.min()), ref_end=int((fp + ln).max()))
        reads.append(read)
        chains.append([c])
        anchors.append(a)
    # one call per read (the reference's own call shape) ...
    single = [eng.extend_chains(r, c, a, ref)[0] for r, c, a in zip(reads, chains, anchors)]
    # ... and all reads in one device launch
    batched = [x[0] for x in eng.extend_batch(reads, chains, anchors, ref)]
    for k, res in enumerate(single):
        want_cigar = words_to_cigar(g["cigar"][g["cigar_off"][k]: g["cigar_off"][k + 1]])
        for got in (res, batched[k]):
            assert got.score == g["score"][k], k
            assert got.cigar == want_cigar, (k, got.cigar_string)
            assert (got.read_start, got.read_end, got.ref_start, got.ref_end) == (
                g["read_start"][k], g["read_end"][k], g["ref_start"][k], g["ref_end"][k])
            assert [got.n_match, got.n_mismatch, got.n_insertion, got.n_deletion] == list(g["counts"][k])


def test_banded_affine_sw_batch_and_traceback_signature():
    """The reference's own identical-sequence check (tests/test_alignment_stages.py
    L1029-1048) through banded_affine_sw_batch + traceback_banded."""
    import torch

    from graphmambaformer_b200.config import ExtensionConfig
    from graphmambaformer_b200.extension import banded_affine_sw_batch, traceback_banded

    rng = np.random.default_rng(3)
    codes = rng.integers(1, 5, size=40).astype(np.int16)
    cfg = ExtensionConfig()
    res = banded_affine_sw_batch(torch.as_tensor(codes, device="cuda")[None],
                                 torch.as_tensor(codes, device="cuda")[None], torch.tensor([40]),
                                 torch.tensor([40]), cfg, half_band=8, return_matrices=True)
    assert float(res.score[0]) == 80.0
    ext = traceback_banded(res, 0, codes, codes, cfg)
    assert ext.cigar == [("=", 40)] and ext.edit_distance == 0
    with pytest.raises(ValueError):
        traceback_banded(banded_affine_sw_batch(torch.as_tensor(codes, device="cuda")[None],
                                                torch.as_tensor(codes, device="cuda")[None],
                                                torch.tensor([40]), torch.tensor([40]), cfg, 8),
                         0, codes, codes, cfg)
