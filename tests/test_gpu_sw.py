"""GPU parity of the banded SW + traceback kernel: bit-exact scores, end and
start coordinates, op counts and CIGARs against the reference's golden
vectors and the CPU oracle; plus size-independent properties at full size."""

from __future__ import annotations

import numpy as np
import pytest

from helpers import assert_sw_equal, cigar_score, golden_sw_pairs, words_to_cigar

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ext():
    from graphmambaformer_b200 import extension

    return extension


@pytest.mark.parametrize("form", ["batched", "plain"])
def test_sw_matches_reference_golden(ext, form):
    n = 0
    for p, idx, ps, g in golden_sw_pairs():
        res = ext.align_pairs(ps, ext.sw_params(*p), traceback=True, form=form)
        for k, b in enumerate(idx):
            tag = str(g["tag"][b])
            assert res.score[k] == g["score"][b], (tag, b, res.score[k], g["score"][b])
            assert res.query_end[k] == g["query_end"][b], (tag, b)
            assert res.target_end[k] == g["target_end"][b], (tag, b)
            assert res.query_start[k] == g["query_start"][b], (tag, b)
            assert res.target_start[k] == g["target_start"][b], (tag, b)
            assert list(res.op_counts[k]) == list(g["counts"][b]), (tag, b)
            want = words_to_cigar(g["cigar"][g["cigar_off"][b]: g["cigar_off"][b + 1]])
            assert res.cigar(k) == want, (tag, b, res.cigar(k), want)
            n += 1
    assert n == len(np.load(__import__("conftest").GOLDEN + "/sw_golden.npz")["half_band"])


def test_sw_known_answer_acgt(ext):
    """tests/test_accel.py L306-334 of the reference."""
    from graphmambaformer_b200.synth import PairSet, encode_bases

    ps = PairSet.from_lists([encode_bases("ACGT")], [encode_bases("TTACGTAA")], 2, 2)
    res = ext.align_pairs(ps, ext.sw_params(2, 4, 6, 2, 600))
    assert int(res.score[0]) == 8 and res.query_end[0] == 4 and res.target_end[0] == 6
    assert res.cigar(0) == [("=", 4)]


def test_sw_matches_oracle_150bp_workload(ext):
    """All 10,000 pairs of the 150 bp extension workload, bit for bit."""
    from graphmambaformer_b200 import synth
    from oracle import oracle

    ps = synth.extension_pairs_150bp(n_pairs=10_000, seed=1)
    res = ext.align_pairs(ps, ext.sw_params(2, 4, 4, 2, 0))
    qs = [ps.q(b) for b in range(len(ps))]
    ts = [ps.t(b) for b in range(len(ps))]
    want = oracle.sw_batch(qs, ts, ps.half_band, ps.band_offset, 2, 4, 4, 2, 0, threads=8)
    assert_sw_equal(res, want, label="150bp")


def test_sw_matches_oracle_mixed_profiles(ext):
    from graphmambaformer_b200 import synth
    from oracle import oracle

    ps = synth.extension_pairs_mixed(n_pairs=400, seed=7, ref_len=2_000_000, max_len=4000,
                                     log_mean=6.5, log_sigma=0.8)
    for params in ((2, 4, 4, 2, 0), (2, 4, 6, 2, 600), (1, 3, 5, 1, 40), (3, 2, 2, 2, 25), (2, 5, 1, 3, 0),
                   (3, 6, 9, 3, 0), (4, 6, 10, 2, 301), (6, 6, 6, 6, 0)):
        res = ext.align_pairs(ps, ext.sw_params(*params))
        want = oracle.sw_batch([ps.q(b) for b in range(len(ps))], [ps.t(b) for b in range(len(ps))],
                               ps.half_band, ps.band_offset, *params, threads=8)
        assert_sw_equal(res, want, label=str(params))


def test_sw_wide_bands_match_oracle(ext):
    """Bands of 500..2000 (W up to 4001) on ONT-like pairs."""
    from graphmambaformer_b200 import synth
    from oracle import oracle

    rng = np.random.default_rng(5)
    ref = synth.random_reference(200_000, rng)
    qs, ts, hbs = [], [], []
    for hb, L in ((500, 1500), (1000, 1200), (2000, 900), (64, 3000), (4096, 300)):
        s = int(rng.integers(3000, 150_000))
        qs.append(synth.apply_errors(ref[s: s + L], synth.ONT, rng))
        ts.append(ref[s - 200: s + L + 200])
        hbs.append(hb)
    ps = synth.PairSet.from_lists(qs, ts, np.array(hbs, np.int32), 200)
    res = ext.align_pairs(ps, ext.sw_params(2, 4, 4, 2, 0))
    want = oracle.sw_batch(qs, ts, ps.half_band, ps.band_offset, 2, 4, 4, 2, 0, threads=5)
    assert_sw_equal(res, want, label="wide")


def test_cooperative_classes_match_oracle(ext):
    """Long pairs with wide bands are shared by 2, 4 or 8 warps of one CTA
    (strip by strip, the row above passed between warps through shared
    memory).  Pairs sized for each of those classes, plus the one-warp cases
    just below their thresholds, match the oracle bit for bit with x-drop off
    and on and under each gap-tie mode (open > ext, open == ext, open < ext)."""
    from graphmambaformer_b200 import synth
    from oracle import oracle

    rng = np.random.default_rng(31)
    ref = synth.random_reference(400_000, rng)
    qs, ts, hbs = [], [], []
    #  (length, half band): C2 (P >= 264), C4 (P >= 528), C8 (P >= 1056), and
    #  one-warp fallbacks (too few strips, or period below the C2 threshold)
    for L, hb in ((2000, 150), (900, 200), (3000, 300), (4200, 264), (5000, 600), (6000, 1000),
                  (500, 300), (200, 600), (3000, 128)):
        for prof in (synth.ONT, synth.HIFI):
            s = int(rng.integers(2000, 390_000 - L))
            qs.append(synth.apply_errors(ref[s: s + L], prof, rng))
            ts.append(ref[s - 150: s + L + 150])
            hbs.append(hb)
    ps = synth.PairSet.from_lists(qs, ts, np.array(hbs, np.int32), 150)
    for params in ((2, 4, 4, 2, 0), (2, 4, 6, 2, 300), (2, 4, 4, 4, 0), (1, 3, 2, 3, 0)):
        res = ext.align_pairs(ps, ext.sw_params(*params))
        want = oracle.sw_batch(qs, ts, ps.half_band, ps.band_offset, *params, threads=8)
        assert_sw_equal(res, want, label=str(params))
        plain = ext.align_pairs(ps, ext.sw_params(*params), form="plain")
        assert np.array_equal(res.score, plain.score) and all(
            res.cigar(k) == plain.cigar(k) for k in range(len(ps))), params


def test_sw_same_result_alone_and_in_the_mix(ext):
    from graphmambaformer_b200 import synth

    ps = synth.extension_pairs_mixed(n_pairs=300, seed=9, ref_len=2_000_000, max_len=3000,
                                     log_mean=6.0, log_sigma=1.0)
    params = ext.sw_params(2, 4, 6, 2, 600)
    mix = ext.align_pairs(ps, params)
    for b in (0, 17, 101, 299):
        alone = ext.align_pairs(ps.subset([b]), params)
        assert alone.score[0] == mix.score[b]
        assert alone.query_end[0] == mix.query_end[b] and alone.target_end[0] == mix.target_end[b]
        assert alone.query_start[0] == mix.query_start[b]
        assert alone.cigar(0) == mix.cigar(b)
    # and a shuffled processing order changes nothing
    order = np.random.default_rng(0).permutation(len(ps)).astype(np.int32)
    shuf = ext.align_pairs(ps, params, order=order)
    assert np.array_equal(shuf.score, mix.score)
    assert all(shuf.cigar(b) == mix.cigar(b) for b in range(len(ps)))


def test_sw_cigar_invariants_full_workload(ext):
    """Size-independent properties on the full 150 bp workload: each CIGAR
    consumes exactly the aligned read and reference spans, and re-scoring the
    CIGAR reproduces the alignment score."""
    from graphmambaformer_b200 import synth

    ps = synth.extension_pairs_150bp(n_pairs=10_000, seed=4)
    res = ext.align_pairs(ps, ext.sw_params(2, 4, 4, 2, 0))
    for b in range(len(ps)):
        c = res.cigar(b)
        assert sum(n for op, n in c if op in "=XI") == res.query_end[b] - res.query_start[b]
        assert sum(n for op, n in c if op in "=XD") == res.target_end[b] - res.target_start[b]
        assert cigar_score(c, 2, 4, 4, 2) == res.score[b]
        if res.score[b] > 0:
            assert c[0][0] in "=X" and c[-1][0] in "=X"


def test_sw_score_only_mode_matches_traceback_mode(ext):
    from graphmambaformer_b200 import synth

    ps = synth.extension_pairs_mixed(n_pairs=200, seed=2, ref_len=1_000_000, max_len=2000)
    a = ext.align_pairs(ps, ext.sw_params(2, 4, 6, 2, 600), traceback=True)
    b = ext.align_pairs(ps, ext.sw_params(2, 4, 6, 2, 600), traceback=False)
    assert np.array_equal(a.score, b.score)
    assert np.array_equal(a.query_end, b.query_end) and np.array_equal(a.target_end, b.target_end)


def test_banded_sw_primitive_matches_reference_signature(ext):
    import torch

    from graphmambaformer_b200.synth import encode_bases

    q = torch.as_tensor(encode_bases("ACGT"), dtype=torch.int8, device="cuda")[None]
    t = torch.as_tensor(encode_bases("TTACGTAA"), dtype=torch.int8, device="cuda")[None]
    score, qe, te = ext.banded_sw(q, t, torch.tensor([4]), torch.tensor([8]), 2, 2.0, 4.0, 6.0, 2.0,
                                  band_offset=torch.tensor([2]))
    assert score.dtype == torch.float32 and float(score[0]) == 8.0
    assert int(qe[0]) == 4 and int(te[0]) == 6


def test_empty_and_degenerate_inputs(ext):
    from graphmambaformer_b200.synth import PairSet

    empty = PairSet.from_lists([], [], np.zeros(0, np.int32), np.zeros(0, np.int32))
    res = ext.align_pairs(empty, ext.sw_params())
    assert len(res.score) == 0
    ps = PairSet.from_lists([np.zeros(0, np.int8), np.array([1, 2, 3], np.int8)],
                            [np.array([1, 2], np.int8), np.zeros(0, np.int8)], 3, 0)
    res = ext.align_pairs(ps, ext.sw_params())
    assert list(res.score) == [0, 0] and res.cigar(0) == [] and res.cigar(1) == []


def test_rejects_band_beyond_limit(ext):
    from graphmambaformer_b200.synth import PairSet

    ps = PairSet.from_lists([np.ones(5, np.int8)], [np.ones(5, np.int8)], 5000, 0)
    with pytest.raises(ValueError):
        ext.align_pairs(ps, ext.sw_params())
    with pytest.raises(ValueError):
        ext.sw_params(2.5, 4, 6, 2, 0)


def test_batched_and_plain_forms_agree_on_every_class(ext):
    """16x2 cells with 8/16/32 lanes, int32 (scores beyond the 16-bit range),
    x-drop on and off: the batched form equals the plain int32 form field for
    field."""
    from graphmambaformer_b200 import synth

    rng = np.random.default_rng(21)
    ref = synth.random_reference(400_000, rng)
    qs, ts, hbs = [], [], []
    for L, hb in ((80, 5), (300, 20), (900, 45), (600, 90), (2000, 200), (17_000, 40), (33_000, 30),
                  (300, 0), (50, 300)):
        for _ in range(6):
            s = int(rng.integers(500, 350_000 - L))
            qs.append(synth.apply_errors(ref[s: s + L], synth.ONT, rng))
            ts.append(ref[s - 100: s + L + 100])
            hbs.append(hb)
    ps = synth.PairSet.from_lists(qs, ts, np.array(hbs, np.int32), 100)
    for params in ((2, 4, 4, 2, 0), (2, 4, 6, 2, 600), (2, 4, 4, 4, 30)):
        a = ext.align_pairs(ps, ext.sw_params(*params), form="batched")
        b = ext.align_pairs(ps, ext.sw_params(*params), form="plain")
        assert np.array_equal(a.score, b.score), params
        assert np.array_equal(a.query_end, b.query_end) and np.array_equal(a.target_end, b.target_end)
        assert np.array_equal(a.query_start, b.query_start) and np.array_equal(a.target_start, b.target_start)
        assert np.array_equal(a.op_counts, b.op_counts)
        assert all(a.cigar(k) == b.cigar(k) for k in range(len(ps))), params


@pytest.mark.parametrize("params", [(2, 4, 6, 2, 0), (2, 3, 5, 1, 0)])
def test_int16_eligibility_boundary(ext, params):
    """Identical sequences whose lengths sit just inside and just outside the
    16x2 form's range -- on the scoring divided by g = gcd(match, mismatch,
    open, extend): m * (len + 1) + 4 * p + 2 + m <= 32768, p the largest
    scaled penalty (32,752 bases at 2/4/6/2, where g = 2; 16,371 at 2/3/5/1)
    -- agree with the plain int32 form and with the closed-form score."""
    from math import gcd

    from graphmambaformer_b200 import synth

    g = gcd(gcd(params[0], params[1]), gcd(params[2], params[3]))
    m, p = params[0] // g, max(params[1], params[2], params[3]) // g
    last = (32768 - 4 * p - 2 - m) // m - 1
    rng = np.random.default_rng(77)
    qs, ts = [], []
    for n in (last - 1, last, last + 1, last + 40):
        s = synth.random_reference(n, rng)
        qs.append(s)
        ts.append(s.copy())
    ps = synth.PairSet.from_lists(qs, ts, 8, 0)
    a = ext.align_pairs(ps, ext.sw_params(*params), form="batched")
    b = ext.align_pairs(ps, ext.sw_params(*params), form="plain")
    assert list(a.score) == [params[0] * len(x) for x in qs]
    assert np.array_equal(a.score, b.score) and np.array_equal(a.query_end, b.query_end)
    assert all(a.cigar(k) == [("=", len(qs[k]))] for k in range(len(qs)))


def test_long_noisy_pairs_near_the_16x2_limit_match_oracle(ext):
    """ONT-like pairs whose lengths approach the 16x2 range on the scaled
    scoring (at 2/4/4/2, g = 2: up to 32,756 bases), so traceback
    differences come close to their 15-bit bound, plus pairs just beyond it
    (int32 class); bands wide enough for the cooperative classes."""
    from graphmambaformer_b200 import synth
    from oracle import oracle

    rng = np.random.default_rng(12)
    ref = synth.random_reference(200_000, rng)
    qs, ts, hbs = [], [], []
    for L, hb in ((32_700, 300), (32_400, 200), (31_000, 600), (33_500, 300)):
        s = int(rng.integers(1000, 200_000 - L - 1000))
        qs.append(synth.apply_errors(ref[s: s + L], synth.ONT, rng)[:32_756])
        ts.append(ref[s: s + L])
        hbs.append(hb)
    qs[-1] = ref[5000: 5000 + 33_500].copy()  # identical: its score leaves the 16x2 range
    ts[-1] = qs[-1].copy()
    ps = synth.PairSet.from_lists(qs, ts, np.array(hbs, np.int32), 0)
    for params in ((2, 4, 4, 2, 0), (2, 4, 6, 2, 0)):
        res = ext.align_pairs(ps, ext.sw_params(*params))
        want = oracle.sw_batch(qs, ts, ps.half_band, ps.band_offset, *params, threads=4)
        assert_sw_equal(res, want, label=str(params))


def test_bounded_cooperative_wait_gives_up_then_recovers(ext):
    """The waits between the warps of a cooperative class are bounded.  With
    the test hook making every writer keep its progress to itself, each wait
    runs out after 256 polls: the call still returns, its error flags carry
    GMF_SWF_TIMEOUT and the host API raises.  The next normal call on the
    same device is bit-exact with the oracle again."""
    import torch

    from graphmambaformer_b200 import _native, autotune, synth
    from oracle import oracle

    rng = np.random.default_rng(41)
    ref = synth.random_reference(100_000, rng)
    qs, ts, hbs = [], [], []
    for L, hb in ((3000, 300), (3000, 150)):  # a 4-warp and a 2-warp cooperative pair
        s = int(rng.integers(1000, 90_000))
        qs.append(synth.apply_errors(ref[s: s + L], synth.ONT, rng))
        ts.append(ref[s - 100: s + L + 100])
        hbs.append(hb)
    ps = synth.PairSet.from_lists(qs, ts, np.array(hbs, np.int32), 100)
    params = ext.sw_params(2, 4, 4, 2, 0)
    autotune.set_tuning(autotune.DEFAULT, "cuda:0")
    lib = _native.lib()
    assert lib.gmf_sw_test_coop_wait(256, 1) == _native.GMF_OK
    try:
        dp = ext.upload_pairs(ps, "cuda:0")
        out = ext.launch_banded_sw(dp, params)
        torch.cuda.synchronize()
        assert int(out.error_flags.item()) & _native.GMF_SWF_TIMEOUT
        with pytest.raises(RuntimeError, match="bounded wait"):
            ext.align_pairs(ps, params)
    finally:
        assert lib.gmf_sw_test_coop_wait(0, 0) == _native.GMF_OK
    res = ext.align_pairs(ps, params)
    want = oracle.sw_batch(qs, ts, ps.half_band, ps.band_offset, 2, 4, 4, 2, 0, threads=2)
    assert_sw_equal(res, want, label="after the timeout")
