"""The host half of `ExtensionEngine` on the CPU: the DP windows, bands and
band offsets `_pairs` derives from each chain, and the soft clips and
reference offsets put on the results, reproduce the reference's
`extend_chains` outputs (extend_golden.npz) when the DP itself is the
oracle's.  The GPU suite checks the same fixture through the device."""

from __future__ import annotations

import numpy as np

from helpers import load, words_to_cigar
from oracle import oracle


def test_extension_windows_through_the_oracle_match_reference_golden():
    from graphmambaformer_b200.config import ExtensionConfig
    from graphmambaformer_b200.extension import ExtensionEngine
    from graphmambaformer_b200.synth import decode_bases, encode_bases
    from graphmambaformer_b200.types import AnchorSet, Chain, add_soft_clips

    g = load("extend_golden.npz")
    cfg = ExtensionConfig()
    eng = ExtensionEngine.__new__(ExtensionEngine)  # the host logic only: no device
    eng.cfg = cfg
    ref_codes = encode_bases(decode_bases(g["ref"]))
    off = g["read_off"]
    items = []
    for k in range(len(off) - 1):
        row = g["chains"][k]
        rp, fp, ln, strand = row[0:3], row[3:6], row[6:9], int(row[9])
        a = AnchorSet.from_lists(rp, fp, ln, np.full(3, strand, np.int8))
        c = Chain(anchor_idx=np.arange(3), score=40.0, strand=strand, read_start=int(rp.min()),
                  read_end=int((rp + ln).max()), ref_start=int(fp.min()), ref_end=int((fp + ln).max()))
        items.append((encode_bases(decode_bases(g["reads"][off[k]: off[k + 1]])), [c], a, ref_codes))
    ps, meta = eng._pairs(items)
    assert len(ps) == len(items) and np.array_equal(np.diff(ps.xdrop_group_off), np.ones(len(items)))
    out = oracle.sw_batch([ps.q(b) for b in range(len(ps))], [ps.t(b) for b in range(len(ps))],
                          ps.half_band, ps.band_offset, cfg.match_score, cfg.mismatch_penalty, cfg.gap_open,
                          cfg.gap_extend, cfg.x_drop)
    for b, (k, start, read_len) in enumerate(meta):
        assert float(out.score[b]) == g["score"][k], k
        cigar = add_soft_clips(out.cigars[b], int(out.query_start[b]), read_len - int(out.query_end[b]))
        assert cigar == words_to_cigar(g["cigar"][g["cigar_off"][k]: g["cigar_off"][k + 1]]), k
        assert (int(out.query_start[b]), int(out.query_end[b]), int(out.target_start[b]) + start,
                int(out.target_end[b]) + start) == (g["read_start"][k], g["read_end"][k],
                                                     g["ref_start"][k], g["ref_end"][k]), k
        assert list(out.counts[b]) == list(g["counts"][k]), k


def test_multi_chain_reads_share_the_xdrop_stop_through_the_oracle():
    """Reads whose chains drop on different rows (xdrop_golden.npz): `_pairs`
    makes one x-drop group and one band per read, and the oracle's grouped SW
    reproduces the reference's `extend_chains` results for every chain."""
    from graphmambaformer_b200.config import ExtensionConfig
    from graphmambaformer_b200.extension import ExtensionEngine
    from graphmambaformer_b200.synth import decode_bases, encode_bases
    from graphmambaformer_b200.types import AnchorSet, Chain, add_soft_clips

    g = load("xdrop_golden.npz")
    cfg = ExtensionConfig()
    eng = ExtensionEngine.__new__(ExtensionEngine)
    eng.cfg = cfg
    ref_codes = encode_bases(decode_bases(g["ref"]))
    items = []
    for c in range(len(g["read_off"]) - 1):
        read = encode_bases(decode_bases(g["reads"][g["read_off"][c]: g["read_off"][c + 1]]))
        a = g["anchors"][g["anchor_off"][c]: g["anchor_off"][c + 1]]
        rp, fp, ln = a[:, 0], a[:, 1], a[:, 2]
        anchors = AnchorSet.from_lists(rp, fp, ln, a[:, 3].astype(np.int8))
        chains = [Chain(anchor_idx=np.arange(lo, hi), score=30.0, strand=int(cs), read_start=int(rp[lo:hi].min()),
                        read_end=int((rp[lo:hi] + ln[lo:hi]).max()), ref_start=int(fp[lo:hi].min()),
                        ref_end=int((fp[lo:hi] + ln[lo:hi]).max()))
                   for call, lo, hi, cs in g["chains"] if call == c]
        items.append((read, chains, anchors, ref_codes))
    ps, meta = eng._pairs(items)
    out = oracle.sw_batch([ps.q(b) for b in range(len(ps))], [ps.t(b) for b in range(len(ps))], ps.half_band,
                          ps.band_offset, cfg.match_score, cfg.mismatch_penalty, cfg.gap_open, cfg.gap_extend,
                          cfg.x_drop, group_off=ps.xdrop_group_off)
    assert len(meta) == len(g["x_score"]) and np.diff(ps.xdrop_group_off).max() > 1
    for b, (_, start, read_len) in enumerate(meta):
        qs0, qe0 = int(out.query_start[b]), int(out.query_end[b])
        assert float(out.score[b]) == g["x_score"][b], b
        assert add_soft_clips(out.cigars[b], qs0, read_len - qe0) == words_to_cigar(
            g["x_cigar"][g["x_cigar_off"][b]: g["x_cigar_off"][b + 1]]), b
        assert [qs0, qe0, int(out.target_start[b]) + start, int(out.target_end[b]) + start] == list(g["x_span"][b])
        assert list(out.counts[b]) == list(g["x_counts"][b]), b
