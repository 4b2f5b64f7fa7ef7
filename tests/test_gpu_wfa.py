"""Wavefront alignment on the device against the reference's own outputs
(golden vectors of WavefrontAligner.align and of extend_chains in both
modes) and against the oracle at sizes where the history spills out of
shared memory."""

from __future__ import annotations

import numpy as np
import pytest

from helpers import load, words_to_cigar

pytestmark = pytest.mark.gpu


def _golden_cases():
    g = load("wfa_golden.npz")
    for i in range(len(g["distance"])):
        q = g["q"][g["q_off"][i]: g["q_off"][i + 1]]
        t = g["t"][g["t_off"][i]: g["t_off"][i + 1]]
        yield q, t, int(g["max_distance"][i]), int(g["distance"][i]), \
            words_to_cigar(g["cigar"][g["cigar_off"][i]: g["cigar_off"][i + 1]])


def test_wavefront_aligner_matches_reference_golden():
    from graphmambaformer_b200.config import ExtensionConfig
    from graphmambaformer_b200.wfa import WavefrontAligner

    for q, t, md, d, cigar in _golden_cases():
        wfa = WavefrontAligner(ExtensionConfig(algorithm="wfa", wfa_max_distance=md))
        if d < 0:
            with pytest.raises(RuntimeError, match="wfa_max_distance"):
                wfa.align(q, t)
        else:
            assert wfa.align(q, t) == (d, cigar)


def test_batched_wfa_matches_reference_golden():
    """All golden pairs in one call per bound (and one call for every bound at
    its largest, checked through the distances), including empty sides."""
    from graphmambaformer_b200.wfa import align_wfa_pairs

    cases = list(_golden_cases())
    for md in sorted({c[2] for c in cases}):
        sel = [c for c in cases if c[2] == md]
        r = align_wfa_pairs([c[0] for c in sel], [c[1] for c in sel], md)
        for b, (_, _, _, d, cigar) in enumerate(sel):
            assert int(r.distance[b]) == d, (md, b)
            if d >= 0:
                assert r.cigar(b) == cigar, (md, b)
                counts = [sum(n for op, n in cigar if op == o) for o in "=XID"]
                assert list(r.op_counts[b]) == counts
            else:
                assert r.cigar_len[b] == -1


def test_wfa_distance_padded_signature():
    """accel/cuda_kernels.py L569-600 shape: padded int8 tensors; the
    reference's own check (tests/test_accel.py L336-345) included."""
    import torch

    from graphmambaformer_b200.synth import encode_bases
    from graphmambaformer_b200.wfa import wfa_distance

    q = torch.as_tensor(encode_bases("ACGTAC"), dtype=torch.int8, device="cuda")[None]
    t = torch.as_tensor(encode_bases("ACGTTAC"), dtype=torch.int8, device="cuda")[None]
    got = wfa_distance(q, t, torch.tensor([6], device="cuda"), torch.tensor([7], device="cuda"), max_distance=4)
    assert int(got[0]) == 1
    cases = list(_golden_cases())
    B = len(cases)
    M = max(len(c[0]) for c in cases)
    N = max(len(c[1]) for c in cases)
    qp = np.full((B, max(M, 1)), -1, np.int8)
    tp = np.full((B, max(N, 1)), -1, np.int8)
    for b, c in enumerate(cases):
        qp[b, : len(c[0])] = c[0]
        tp[b, : len(c[1])] = c[1]
    ql = torch.tensor([len(c[0]) for c in cases], device="cuda")
    tl = torch.tensor([len(c[1]) for c in cases], device="cuda")
    got = wfa_distance(torch.as_tensor(qp, device="cuda"), torch.as_tensor(tp, device="cuda"), ql, tl, 4096)
    want = [c[3] if c[2] == 4096 else None for c in cases]
    for b, w in enumerate(want):
        if w is not None:
            assert int(got[b]) == w, b


def _engine_calls(g):
    from graphmambaformer_b200.synth import decode_bases
    from graphmambaformer_b200.types import AnchorSet, Chain

    calls = []
    for c in range(len(g["calls"])):
        read = decode_bases(g["reads"][g["read_off"][c]: g["read_off"][c + 1]])
        a = g["anchors"][g["anchor_off"][c]: g["anchor_off"][c + 1]]
        rp, fp, ln, st = a[:, 0], a[:, 1], a[:, 2], a[:, 3].astype(np.int8)
        anchors = AnchorSet.from_lists(rp, fp, ln, st)
        chains = []
        for call, lo, hi, cs in g["chains"]:
            if call != c:
                continue
            chains.append(Chain(anchor_idx=np.arange(lo, hi), score=30.0, strand=int(cs),
                                read_start=int(rp[lo:hi].min()), read_end=int((rp[lo:hi] + ln[lo:hi]).max()),
                                ref_start=int(fp[lo:hi].min()), ref_end=int((fp[lo:hi] + ln[lo:hi]).max())))
        calls.append((int(g["calls"][c][0]), int(g["calls"][c][1]), read, chains, anchors))
    return calls


def _check_ext(got, g, k):
    want_cigar = words_to_cigar(g["x_cigar"][g["x_cigar_off"][k]: g["x_cigar_off"][k + 1]])
    assert got.cigar == want_cigar, (k, got.cigar_string)
    assert got.score == g["x_score"][k], k
    assert [got.read_start, got.read_end, got.ref_start, got.ref_end] == list(g["x_span"][k]), k
    assert [got.n_match, got.n_mismatch, got.n_insertion, got.n_deletion] == list(g["x_counts"][k]), k


def test_extend_chains_multi_chain_both_modes():
    """Several chains per read: banded_sw mode (one band per read, the widest
    of its chains) and wfa mode (window from the diagonal and net indel,
    banded-SW fallback beyond the bound) -- one call per read and all reads
    of a mode in one batch."""
    from graphmambaformer_b200.config import ExtensionConfig
    from graphmambaformer_b200.extension import ExtensionEngine
    from graphmambaformer_b200.synth import decode_bases

    g = load("wfa_golden.npz")
    ref = decode_bases(g["ref"])
    calls = _engine_calls(g)
    k = 0
    groups: dict = {}
    for algo, md, read, chains, anchors in calls:
        cfg = ExtensionConfig(algorithm="wfa" if algo else "banded_sw", wfa_max_distance=md)
        out = ExtensionEngine(cfg).extend_chains(read, chains, anchors, ref)
        assert len(out) == len(chains)
        groups.setdefault((algo, md), []).append((read, chains, anchors, k))
        for got in out:
            _check_ext(got, g, k)
            k += 1
    assert k == len(g["x_score"])
    for (algo, md), items in groups.items():
        cfg = ExtensionConfig(algorithm="wfa" if algo else "banded_sw", wfa_max_distance=md)
        out = ExtensionEngine(cfg).extend_batch([x[0] for x in items], [x[1] for x in items],
                                                [x[2] for x in items], ref)
        for (_, chains, _, k0), res in zip(items, out):
            for j, got in enumerate(res):
                _check_ext(got, g, k0 + j)


def test_wfa_spilled_wavefronts_and_chunked_histories_match_oracle():
    """Distances above 255 move the live wavefronts to global memory; a small
    history budget splits the batch over several calls.  Both against the
    oracle, with the Levenshtein properties of the reference's own test
    (tests/test_alignment_stages.py L1063-1091) checked on every pair."""
    from oracle import oracle

    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.wfa import align_wfa_pairs

    rng = np.random.default_rng(17)
    qs, ts = [], []
    for L, prof in ((6000, synth.ONT), (3000, synth.ONT), (2000, synth.HIFI), (400, synth.ILLUMINA),
                    (900, synth.ErrorProfile(0.1, 0.05, 0.05)), (50, synth.ONT)):
        for _ in range(3):
            a = synth.random_reference(L, rng).astype(np.int8)
            qs.append(a)
            ts.append(synth.apply_errors(a, prof, rng).astype(np.int8))
    want = [oracle.wfa_align(q, t, 4096) for q, t in zip(qs, ts)]
    assert max(d for d, _ in want) > 255, "the case must exercise the spilled wavefronts"
    for budget in (1 << 29, 300_000):
        r = align_wfa_pairs(qs, ts, 4096, history_budget=budget)
        for b, (d, cigar) in enumerate(want):
            assert int(r.distance[b]) == d, (budget, b)
            got = r.cigar(b)
            assert got == cigar, (budget, b)
            assert sum(n for op, n in got if op in "=XI") == len(qs[b])
            assert sum(n for op, n in got if op in "=XD") == len(ts[b])
            assert sum(n for op, n in got if op in "XID") == d


@pytest.mark.parametrize("pinned", [False, True])
def test_csr_batch_matches_list_form_and_oracle(pinned):
    """align_wfa_batch on the pairs as CSR arrays (plain, or page-locked and
    copied to the device directly) gives the list form's distances and
    CIGARs, and the oracle's; empty sides and a bound some pairs exceed
    included."""
    from oracle import oracle

    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.wfa import WfaBatch, align_wfa_batch, align_wfa_pairs

    rng = np.random.default_rng(23)
    qs, ts = [], []
    for L in (0, 1, 7, 150, 600, 2500):
        for _ in range(2):
            a = synth.random_reference(L, rng).astype(np.int8)
            qs.append(a)
            ts.append(synth.apply_errors(a, synth.ONT, rng).astype(np.int8) if L else a.copy())
    qs.append(np.zeros(0, np.int8))
    ts.append(synth.random_reference(30, rng).astype(np.int8))
    md = 90
    batch = WfaBatch.of(qs, ts)
    if pinned:
        batch = batch.pinned()
    got = align_wfa_batch(batch, md)
    ref = align_wfa_pairs(qs, ts, md)
    assert np.array_equal(got.distance, ref.distance)
    assert (got.distance < 0).any() and (got.distance >= 0).any()
    for b in range(len(qs)):
        d, cigar = oracle.wfa_align(qs[b], ts[b], md)
        assert int(got.distance[b]) == d, b
        if d >= 0:
            assert got.cigar(b) == ref.cigar(b) == cigar, b
