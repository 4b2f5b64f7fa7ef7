"""The C ABI's asynchronous host-buffer form (gmf_ctx_* / gmf_batch_*)
against the device-buffer form on the same pairs: several batches in flight,
polling, slot reuse, x-drop groups, a budget that refuses an oversized
batch, and an empty batch."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b, traceback=True):
    assert np.array_equal(a.score, b.score)
    assert np.array_equal(a.query_end, b.query_end)
    assert np.array_equal(a.target_end, b.target_end)
    if traceback:
        assert np.array_equal(a.query_start, b.query_start)
        assert np.array_equal(a.target_start, b.target_start)
        assert np.array_equal(a.op_counts, b.op_counts)
        for k in range(len(a.score)):
            assert a.cigar(k) == b.cigar(k), k


def test_context_matches_device_form_with_batches_in_flight():
    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.context import AlignContext
    from graphmambaformer_b200.extension import align_pairs, sw_params

    params = sw_params(2, 4, 4, 2, 0)
    batches = [synth.extension_pairs_mixed(n_pairs=n, seed=s, ref_len=300_000, max_len=5000)
               for n, s in ((300, 1), (50, 2), (700, 3), (1, 4), (400, 5))]
    want = [align_pairs(ps, params) for ps in batches]
    with AlignContext(0) as ctx:
        tickets = [ctx.submit(ps, params) for ps in batches]  # five batches on three slots
        got = [None] * len(batches)
        for _ in range(100000):
            for i, t in enumerate(tickets):
                if got[i] is None:
                    got[i] = ctx.poll(t)
            if all(g is not None for g in got):
                break
        for g, w in zip(got, want):
            assert g is not None and g.error_flags == 0
            _same(g, w)
        # score-only batches and synchronous use
        r = ctx.align(batches[0], params, traceback=False)
        _same(r, want[0], traceback=False)
        # an empty batch
        empty = synth.PairSet.from_lists([], [], np.zeros(0, np.int32), 0)
        assert len(ctx.align(empty, params).score) == 0


def test_context_groups_and_budget():
    from graphmambaformer_b200 import _native, synth
    from graphmambaformer_b200.context import AlignContext
    from graphmambaformer_b200.extension import align_pairs, sw_params

    ps = synth.extension_pairs_mixed(n_pairs=200, seed=9, ref_len=300_000, max_len=3000)
    ps.xdrop_group_off = np.array([0, 3, 3, 50, 51, 200], np.int32)
    params = sw_params(2, 4, 4, 2, 40)
    want = align_pairs(ps, params)
    with AlignContext(0) as ctx:
        _same(ctx.align(ps, params), want)
    with AlignContext(0, slots=3, memory_budget=3 * 4096) as small:
        with pytest.raises(_native.GmfError, match="limit"):
            small.submit(ps, params)
