"""Banded SW replayed from a captured CUDA graph: every batch (padded to the
aligner's capacity with empty pairs) gives exactly the results of the
eager call, batch after batch, with one capture."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b, n):
    assert np.array_equal(a.score, b.score) and np.array_equal(a.query_end, b.query_end)
    assert np.array_equal(a.target_end, b.target_end) and np.array_equal(a.query_start, b.query_start)
    assert np.array_equal(a.target_start, b.target_start) and np.array_equal(a.op_counts, b.op_counts)
    assert all(a.cigar(k) == b.cigar(k) for k in range(n))


def test_graph_replays_match_eager_calls():
    from graphmambaformer_b200 import extension, synth
    from graphmambaformer_b200.graphs import GraphedAligner

    prm = extension.sw_params(2, 4, 4, 2, 0)
    big = synth.extension_pairs_mixed(n_pairs=400, seed=51, ref_len=2_000_000, max_len=8000, log_mean=7.0,
                                      log_sigma=1.0, band_slope=0.04)
    small = [big.subset(np.arange(k, len(big), 3)) for k in range(3)]
    al = GraphedAligner("cuda:0", prm, cap_pairs=400, cap_query=int(big.query_off[-1]),
                        cap_target=int(big.target_off[-1]), max_half_band=int(big.half_band.max()))
    for ps in [big] + small + [big]:
        got = al.align(ps)
        want = extension.align_pairs(ps, prm, device="cuda:0")
        _same(got, want, len(ps))
    assert al.replays == 5 and al.captures == 1  # the first batch sized the workspace for the rest


def test_graph_handles_empty_and_oversized_batches():
    from graphmambaformer_b200 import extension, synth
    from graphmambaformer_b200.graphs import GraphedAligner

    prm = extension.sw_params(2, 4, 4, 2, 0)
    ps = synth.extension_pairs_150bp(n_pairs=50, seed=3, ref_len=100_000)
    al = GraphedAligner("cuda:0", prm, cap_pairs=64, cap_query=64 * 200, cap_target=64 * 300, max_half_band=32)
    empty = ps.subset(np.zeros(0, np.int64))
    assert len(al.align(empty)) == 0
    _same(al.align(ps), extension.align_pairs(ps, prm, device="cuda:0"), len(ps))
    with pytest.raises(ValueError):
        al.align(synth.extension_pairs_150bp(n_pairs=65, seed=4, ref_len=100_000))
