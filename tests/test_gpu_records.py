"""SAM text rendered on the device (gmf_sam_count / gmf_sam_fill) against the
reference's segment fields (sam_golden.pkl) through the pinned oracle, and
the whole step after extension -- our extend_chains, record assembly, device
SAM -- against the reference on the same reads."""

from __future__ import annotations

import os
import pickle
from types import SimpleNamespace

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _golden():
    with open(os.path.join(GOLDEN, "sam_golden.pkl"), "rb") as fh:
        return pickle.load(fh)


def _reads(g):
    return [c["seq"] if c["modality"] is None else
            SimpleNamespace(read_id=c["read_id"], seq=c["seq"], quals=c["quals"], modality=c["modality"])
            for c in g["calls"]]


def _check_lines(text: bytes, segments, contigs):
    from oracle import sam

    lines = text.decode().split("\n")
    assert lines[-1] == ""
    lines = lines[:-1]
    assert len(lines) == len(segments)
    for k, (line, seg) in enumerate(zip(lines, segments)):
        assert line == sam.render(seg, contigs), k


def test_device_sam_matches_reference_segments():
    from graphmambaformer_b200.records import AlignmentRecord, ReadAlignments, render_sam, sam_records

    g = _golden()
    results = [ReadAlignments(read_id=c["read_id"], read_len=len(c["seq"]),
                              records=[AlignmentRecord(**{k: v for k, v in r.items() if k != "extension"})
                                       for r in c["records"]]) for c in g["calls"]]
    for (inc, names), want in g["outputs"].items():
        b = sam_records(results, _reads(g), "pacbio_hifi", inc, {0: len(g["ref"])},
                        None if names is None else {0: names})
        _check_lines(render_sam(b, "cuda:0"), want["segments"], [names or "ref0"])


def test_extension_records_and_sam_end_to_end(tmp_path):
    """Our extend_chains (banded SW or WFA, as each golden read used), record
    assembly and device SAM on the reference's reads give the reference's
    SAM fields; write_sam produces the header and the same lines."""
    from graphmambaformer_b200.config import ExtensionConfig
    from graphmambaformer_b200.extension import ExtensionEngine
    from graphmambaformer_b200.records import AlignmentRecord, read_alignments, render_sam, sam_records, write_sam
    from graphmambaformer_b200.synth import decode_bases
    from graphmambaformer_b200.types import AnchorSet, Chain

    g = _golden()
    ref = decode_bases(g["ref"])
    engines = {a: ExtensionEngine(ExtensionConfig(algorithm="wfa" if a else "banded_sw")) for a in (0, 1)}
    results = []
    for c in g["calls"]:
        a = c["anchors"]
        anchors = AnchorSet.from_lists(a[:, 0], a[:, 1], a[:, 2], a[:, 3].astype(np.int8)) if len(a) else \
            AnchorSet.from_lists([], [], [], [])
        chains = []
        for lo, hi, cs, score, prim in c["chains"]:
            rp, fp, ln = a[lo:hi, 0], a[lo:hi, 1], a[lo:hi, 2]
            chains.append(Chain(anchor_idx=np.arange(lo, hi), score=score, strand=int(cs),
                                read_start=int(rp.min()), read_end=int((rp + ln).max()), ref_start=int(fp.min()),
                                ref_end=int((fp + ln).max()), is_primary=prim))
        exts = engines[c["algo"]].extend_chains(c["seq"], chains, anchors, ref) if chains else []
        exts = exts[: c["n_ext"]]
        ra = read_alignments(c["read_id"], len(c["seq"]), anchors, chains, exts, node_starts=g["node_starts"],
                             node_ids=g["node_ids"])
        extra = c["records"][len(ra.records):]  # the generator's hand-made edge records
        ra.records += [AlignmentRecord(**{k: v for k, v in r.items() if k != "extension"}) for r in extra]
        results.append(ra)
    want = g["outputs"][(True, None)]["segments"]
    b = sam_records(results, _reads(g), "pacbio_hifi", True, {0: len(g["ref"])})
    text = render_sam(b, "cuda:0")
    _check_lines(text, want, ["ref0"])
    path = write_sam(results, _reads(g), str(tmp_path / "out.sam"), references={0: len(g["ref"])},
                     include_secondary=True, device="cuda:0")
    body = open(path, "rb").read()
    head = [ln for ln in body.split(b"\n") if ln.startswith(b"@")]
    assert head[0] == b"@HD\tVN:1.6\tSO:unsorted" and head[1] == b"@SQ\tSN:ref0\tLN:300000"
    assert body.endswith(text)


def test_device_sam_at_scale_matches_oracle():
    """20,000 synthetic records of 150 bp - 20 kb (both strands, clipped and
    unclipped CIGARs, unmapped and length-mismatched ones) against the oracle."""
    from oracle import sam

    from graphmambaformer_b200.records import AlignmentRecord, ReadAlignments, render_sam, sam_records

    rng = np.random.default_rng(5)
    results, reads = [], []
    for i in range(20_000):
        L = int(np.clip(rng.lognormal(7.0, 1.2), 150, 20_000))
        seq = "".join(rng.choice(list("ACGTN"), size=L, p=[0.249, 0.249, 0.249, 0.249, 0.004]))
        cl = int(rng.integers(0, min(50, L // 4)))
        cr = int(rng.integers(0, min(50, L // 4)))
        mid = L - cl - cr
        core = [("=", mid // 2), ("X", 1), ("I", 2), ("=", mid - mid // 2 - 3), ("D", 4)]
        cigar = ([("S", cl)] if cl else []) + [x for x in core if x[1] > 0] + ([("S", cr)] if cr else [])
        if i % 97 == 0:
            cigar = cigar[:-1] + [("S", cr + 1)]  # query length off by one: written unmapped
        mapped = i % 31 != 0
        rec = AlignmentRecord(read_id=f"r{i}", read_len=L, ref_id=0, ref_start=int(rng.integers(0, 10**7)),
                              ref_end=0, strand=1 if rng.random() < 0.5 else -1, mapq=int(rng.integers(0, 61)),
                              cigar=cigar, is_mapped=mapped)
        rec.ref_end = rec.ref_start + mid
        results.append(ReadAlignments(read_id=rec.read_id, read_len=L, records=[rec]))
        quals = [int(x) for x in rng.integers(0, 60, size=L)] if i % 2 else None
        reads.append(SimpleNamespace(read_id=rec.read_id, seq=seq, quals=quals, modality="ont"))
    b = sam_records(results, reads, "ont", False, {0: 10**8})
    text = render_sam(b, "cuda:0")
    segs = [sam.segment(vars(r.records[0]), rd.seq, rd.quals, "ont", {0: 0}) for r, rd in zip(results, reads)]
    _check_lines(text, segs, ["ref0"])
    # the length hint only splits the work: none, too low and too high give the same bytes
    for hint in (0, 5000, 10**6):
        assert render_sam(b, "cuda:0", max_seq_len=hint) == text, hint
