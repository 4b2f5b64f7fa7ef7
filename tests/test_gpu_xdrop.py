"""The reference's batch x-drop rule on the device: a batch's row loop stops
only after every member dropped (extension.py L190-193).  Golden vectors
from banded_affine_sw_batch on batches whose members drop on different
rows, and from extend_chains on reads whose chains drop at different rows."""

from __future__ import annotations

import numpy as np
import pytest

from helpers import load, words_to_cigar

pytestmark = pytest.mark.gpu


def _batches(g):
    for b in range(len(g["batch_off"]) - 1):
        lo, hi = int(g["batch_off"][b]), int(g["batch_off"][b + 1])
        qs = [g["query"][g["query_off"][p]: g["query_off"][p + 1]] for p in range(lo, hi)]
        ts = [g["target"][g["target_off"][p]: g["target_off"][p + 1]] for p in range(lo, hi)]
        yield lo, hi, float(g["x_drop"][b]), qs, ts


def _check_pair(g, p, score, qe, te, qs=None, ts=None, cigar=None):
    assert (score, qe, te) == (g["score"][p], g["qe"][p], g["te"][p]), p
    if cigar is not None:
        assert (qs, ts) == (g["qs"][p], g["ts"][p]), p
        assert cigar == words_to_cigar(g["cigar"][g["cigar_off"][p]: g["cigar_off"][p + 1]]), p


def test_banded_affine_sw_batch_stops_the_batch_together():
    import torch

    from graphmambaformer_b200.config import ExtensionConfig
    from graphmambaformer_b200.extension import banded_affine_sw_batch, traceback_banded

    g = load("xdrop_golden.npz")
    for lo, hi, xd, qs, ts in _batches(g):
        B = hi - lo
        M, N = max(len(x) for x in qs), max(len(x) for x in ts)
        qt = torch.full((B, M), -1, dtype=torch.int16)
        tt = torch.full((B, N), -1, dtype=torch.int16)
        for b in range(B):
            qt[b, : len(qs[b])] = torch.as_tensor(qs[b].astype(np.int16))
            tt[b, : len(ts[b])] = torch.as_tensor(ts[b].astype(np.int16))
        cfg = ExtensionConfig(x_drop=xd)
        res = banded_affine_sw_batch(qt.cuda(), tt.cuda(), torch.tensor([len(x) for x in qs]),
                                     torch.tensor([len(x) for x in ts]), cfg,
                                     half_band=int(g["half_band"][lo]),
                                     band_offset=torch.as_tensor(g["band_offset"][lo:hi].astype(np.int64)),
                                     return_matrices=True)
        for b in range(B):
            ext = traceback_banded(res, b, qs[b], ts[b], cfg)
            _check_pair(g, lo + b, float(res.score[b]), int(res.query_end[b]), int(res.target_end[b]),
                        ext.read_start, ext.ref_start, ext.cigar)


@pytest.mark.parametrize("form", ["batched", "plain"])
def test_groups_in_one_launch_both_forms(form):
    """Every golden batch as one x-drop group of a single launch, in both
    entry points (the plain form defers its walk behind the group pass)."""
    from graphmambaformer_b200.extension import align_pairs, sw_params
    from graphmambaformer_b200.synth import PairSet

    g = load("xdrop_golden.npz")
    for xd in sorted(set(float(x) for x in g["x_drop"])):
        qs, ts, hb, off, goff, idx = [], [], [], [], [0], []
        for lo, hi, x, q, t in _batches(g):
            if x != xd:
                continue
            qs += q
            ts += t
            hb += list(g["half_band"][lo:hi])
            off += list(g["band_offset"][lo:hi])
            goff.append(goff[-1] + hi - lo)
            idx += list(range(lo, hi))
        ps = PairSet.from_lists(qs, ts, np.array(hb, np.int32), np.array(off, np.int32))
        ps.xdrop_group_off = np.array(goff, np.int32)
        res = align_pairs(ps, sw_params(2, 4, 6, 2, xd), traceback=True, form=form)
        for b, p in enumerate(idx):
            _check_pair(g, p, int(res.score[b]), int(res.query_end[b]), int(res.target_end[b]),
                        int(res.query_start[b]), int(res.target_start[b]), res.cigar(b))
        # and without groups every pair stops on its own rows: some results differ
        ps.xdrop_group_off = None
        alone = align_pairs(ps, sw_params(2, 4, 6, 2, xd), traceback=False, form=form)
        assert np.all(alone.score <= res.score)


def test_graphed_and_session_paths_take_groups():
    from graphmambaformer_b200.extension import sw_params
    from graphmambaformer_b200.graphs import GraphedAligner
    from graphmambaformer_b200.session import ExtensionSession
    from graphmambaformer_b200.synth import PairSet

    g = load("xdrop_golden.npz")
    xd = 35.0
    qs, ts, hb, off, goff, idx = [], [], [], [], [0], []
    for lo, hi, x, q, t in _batches(g):
        if x != xd:
            continue
        qs += q
        ts += t
        hb += list(g["half_band"][lo:hi])
        off += list(g["band_offset"][lo:hi])
        goff.append(goff[-1] + hi - lo)
        idx += list(range(lo, hi))
    ps = PairSet.from_lists(qs, ts, np.array(hb, np.int32), np.array(off, np.int32))
    ps.xdrop_group_off = np.array(goff, np.int32)
    params = sw_params(2, 4, 6, 2, xd)
    ga = GraphedAligner("cuda:0", params, cap_pairs=len(ps) + 3, cap_query=int(ps.query_off[-1]) + 64,
                        cap_target=int(ps.target_off[-1]) + 64, max_half_band=int(max(hb)))
    sess = ExtensionSession("cuda:0", x_drop=xd)
    for res in (ga.align(ps), ga.align(ps), sess.align(ps)):
        for b, p in enumerate(idx):
            _check_pair(g, p, int(res.score[b]), int(res.query_end[b]), int(res.target_end[b]),
                        int(res.query_start[b]), int(res.target_start[b]), res.cigar(b))


def test_extend_chains_reads_with_unalignable_blocks():
    from graphmambaformer_b200.config import ExtensionConfig
    from graphmambaformer_b200.extension import ExtensionEngine
    from graphmambaformer_b200.synth import decode_bases
    from graphmambaformer_b200.types import AnchorSet, Chain

    g = load("xdrop_golden.npz")
    ref = decode_bases(g["ref"])
    eng = ExtensionEngine(ExtensionConfig())
    k = 0
    reads, chains_all, anchors_all = [], [], []
    for c in range(len(g["read_off"]) - 1):
        read = decode_bases(g["reads"][g["read_off"][c]: g["read_off"][c + 1]])
        a = g["anchors"][g["anchor_off"][c]: g["anchor_off"][c + 1]]
        rp, fp, ln = a[:, 0], a[:, 1], a[:, 2]
        anchors = AnchorSet.from_lists(rp, fp, ln, a[:, 3].astype(np.int8))
        chains = [Chain(anchor_idx=np.arange(lo, hi), score=30.0, strand=int(cs), read_start=int(rp[lo:hi].min()),
                        read_end=int((rp[lo:hi] + ln[lo:hi]).max()), ref_start=int(fp[lo:hi].min()),
                        ref_end=int((fp[lo:hi] + ln[lo:hi]).max()))
                  for call, lo, hi, cs in g["chains"] if call == c]
        reads.append(read)
        chains_all.append(chains)
        anchors_all.append(anchors)
    out_single = [eng.extend_chains(r, c, a, ref) for r, c, a in zip(reads, chains_all, anchors_all)]
    out_batch = eng.extend_batch(reads, chains_all, anchors_all, ref)
    for res_s, res_b in zip(out_single, out_batch):
        for got_s, got_b in zip(res_s, res_b):
            want = words_to_cigar(g["x_cigar"][g["x_cigar_off"][k]: g["x_cigar_off"][k + 1]])
            for got in (got_s, got_b):
                assert got.score == g["x_score"][k], k
                assert got.cigar == want, (k, got.cigar_string)
                assert [got.read_start, got.read_end, got.ref_start, got.ref_end] == list(g["x_span"][k])
                assert [got.n_match, got.n_mismatch, got.n_insertion, got.n_deletion] == list(g["x_counts"][k])
            k += 1
    assert k == len(g["x_score"])
