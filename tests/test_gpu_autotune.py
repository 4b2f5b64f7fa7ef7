"""The batched-form autotuner on the GPU: its knobs change scheduling only,
so the tuned setting gives results identical to the default on every field,
and out-of-range settings are refused by the C ABI."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_keeps_results_identical():
    from graphmambaformer_b200 import autotune, extension, synth

    ps = synth.extension_pairs_mixed(n_pairs=300, seed=41, ref_len=2_000_000, max_len=9000,
                                     log_mean=7.5, log_sigma=1.0, band_slope=0.05)
    prm = extension.sw_params(2, 4, 4, 2, 0)
    try:
        autotune.set_tuning(autotune.DEFAULT, "cuda:0")
        ref = extension.align_pairs(ps, prm, device="cuda:0")
        rep = autotune.autotune_sw(ps, prm, "cuda:0", reps=1, passes=1)
        assert rep.best.valid() and rep.best_ms <= rep.default_ms
        assert autotune.get_tuning("cuda:0") == rep.best
        got = extension.align_pairs(ps, prm, device="cuda:0")
        assert np.array_equal(got.score, ref.score) and np.array_equal(got.query_end, ref.query_end)
        assert np.array_equal(got.target_start, ref.target_start)
        assert all(got.cigar(b) == ref.cigar(b) for b in range(len(ps)))
        # every knob extreme still gives the same answers
        for t in (autotune.SwTuning(0, 0, (0, 0, 0), 1, 0), autotune.SwTuning(125, 509, (2, 4, 8), 2, 1)):
            autotune.set_tuning(t, "cuda:0")
            got = extension.align_pairs(ps, prm, device="cuda:0")
            assert np.array_equal(got.score, ref.score), t
            assert all(got.cigar(b) == ref.cigar(b) for b in range(len(ps))), t
    finally:
        autotune.set_tuning(autotune.DEFAULT, "cuda:0")


def test_set_tuning_rejects_out_of_range_values():
    from graphmambaformer_b200 import _native, autotune

    autotune.set_tuning(autotune.DEFAULT, "cuda:0")
    bad = autotune.SwTuning(200, 100).to_c()
    assert _native.lib().gmf_sw_set_tuning(ctypes.byref(bad)) == _native.GMF_ERR_INVALID_ARGUMENT
    bad = autotune.SwTuning(warps_per_block=9).to_c()
    assert _native.lib().gmf_sw_set_tuning(ctypes.byref(bad)) == _native.GMF_ERR_INVALID_ARGUMENT
    assert autotune.get_tuning("cuda:0") == autotune.DEFAULT
