"""Generate golden vectors by running the reference implementation itself.

Run in a container that has the reference checked out (read-only), naming
its root in ``$GMF_REFERENCE`` or with ``--reference PATH``::

    GMF_REFERENCE=<reference root> PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py [which ...]

It imports ``graphmambaformer.alignment`` from the reference, feeds it seeded
synthetic inputs, and stores inputs + outputs as small compressed ``.npz``
fixtures next to this script.  The GPU test suite and the oracle tests read
only these fixtures; nothing at test time imports the reference.

Fixtures:

* ``sw_golden.npz``     -- ``banded_affine_sw_batch`` (B=1 per pair) +
  ``traceback_banded``: the reference's known-answer pairs
  (tests/test_accel.py L306-334, tests/test_alignment_stages.py L1029-1048),
  edge cases (empty query, band outside the target, N bases, negative
  offsets, x-drop cut-offs, half band 0) and seeded random pairs.
* ``chain_golden.npz``  -- ``chain_dp_numpy`` on random inputs (with and
  without a bonus, several lookbacks) including the known-answer anchors of
  tests/test_accel.py L347-370, plus ``AffineChainer.chain`` on minimizer
  anchors of simulated HiFi reads.
* ``extend_golden.npz`` -- ``ExtensionEngine.extend_chains`` on single-chain
  calls (window, band widening, soft clips).
* ``seed_golden.npz``   -- ``MinimizerIndex`` (build + ``query``) on seeded
  references with N runs and a repeated block, reads of many lengths (shorter
  than k, with N bases, mutated copies) in both orientations, ``max_occ`` 0
  and 5.
* ``wfa_golden.npz``    -- ``WavefrontAligner.align`` (distance + CIGAR, or
  the over-budget signal) on the reference's own cases
  (tests/test_alignment_stages.py L1063-1111, tests/test_accel.py L336-345)
  and seeded pairs (empty sides, N bases, every error profile, lengths up to
  3000, several distance budgets), plus ``ExtensionEngine.extend_chains``
  calls with several chains per read, in ``banded_sw`` mode (one band shared
  by the read's chains) and in ``wfa`` mode (window from the chain's
  diagonal and net indel, banded-SW fallback beyond ``wfa_max_distance``).
* ``xdrop_golden.npz``  -- the batch x-drop rule: ``banded_affine_sw_batch``
  batches whose members drop on different rows (small ``x_drop``), and
  ``extend_chains`` on reads with unalignable blocks next to secondary
  chains, where a chain keeps extending while another has not dropped.
* ``sam_golden.pkl``    -- record assembly and SAM fields: the pipeline's
  ``_margin_mapq`` and ``_records`` on ``extend_chains`` results (both
  algorithms, both strands, reads without chains), then
  ``alignments_to_records`` and the field assignments of ``_make_segment``
  (data/formats.py L343-397) captured on a stand-in segment object, since
  pysam is not installed here.  Edge records cover a CIGAR that does not
  match the read, an empty span, qualities out of range or short, bases
  outside ACGTN and contig-name overrides.
* ``hybrid_golden.pkl`` -- ``AffineChainer.chain`` with a ``ChainingContext``
  (graph-distance oracle, backbone bias, neural seed scores with each AGNES
  trust decision, learned transitions).
* ``hybrid_inputs_golden.pkl`` -- the two hybrid-mode DP inputs alone,
  ``AffineChainer._weights`` and ``AffineChainer._graph_bonus``, on strand-
  sorted anchor segments over random graphs (several hop limits, lookbacks,
  bonus weights, the legacy linear blend, duplicated anchor keys, transition
  keys that are not in the segment).
* ``pipeline_golden.pkl`` -- ``FastAlignmentPipeline.align`` end to end
  with its stock CPU stage objects (minimizer seeding, ``AffineChainer``,
  ``ExtensionEngine`` in both algorithms, margin MAPQ, records) on seeded
  reads: HiFi, ONT and 150 bp reads on both strands, chimeric and repeated
  reads with secondary chains, unmappable reads, a reference with an N run.
  Stored per read: the seed stage's anchors, the chains and the records.
"""

from __future__ import annotations

import os
import sys

import numpy as np

def _reference_root() -> str:
    args = sys.argv[1:]
    if "--reference" in args:
        i = args.index("--reference")
        root = args[i + 1]
        del sys.argv[i + 1: i + 3]
        return root
    root = os.environ.get("GMF_REFERENCE")
    if not root:
        sys.exit("make_golden.py: name the reference checkout with $GMF_REFERENCE or --reference PATH")
    return root


REF = _reference_root()
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))  # repo root
sys.path.insert(0, REF)
sys.dont_write_bytecode = True

import torch  # noqa: E402

torch.set_num_threads(1)

from graphmambaformer.alignment.chaining import AffineChainer, chain_dp_numpy  # noqa: E402
from graphmambaformer.alignment.extension import (  # noqa: E402
    ExtensionEngine,
    banded_affine_sw_batch,
    traceback_banded,
)
from graphmambaformer.alignment.seeding import encode_bases  # noqa: E402
from graphmambaformer.alignment.types import AnchorSet, Chain  # noqa: E402
from graphmambaformer.config import ChainingConfig, ExtensionConfig  # noqa: E402

from graphmambaformer_b200 import synth  # noqa: E402

OPS = "=XIDS"


def cigar_words(cigar):
    return np.array([(n << 4) | OPS.index(op) for op, n in cigar], dtype=np.uint32)


def ragged(arrs, dtype):
    off = np.zeros(len(arrs) + 1, dtype=np.int64)
    np.cumsum([len(a) for a in arrs], out=off[1:])
    flat = np.concatenate([np.asarray(a, dtype=dtype) for a in arrs]) if off[-1] else np.zeros(0, dtype)
    return flat, off


# --------------------------------------------------------------------------- #
# Banded SW
# --------------------------------------------------------------------------- #
def sw_case(q, t, hb, off, params):
    cfg = ExtensionConfig(match_score=params[0], mismatch_penalty=params[1],
                          gap_open=params[2], gap_extend=params[3], x_drop=params[4])
    qt = torch.as_tensor(np.asarray(q, dtype=np.int16))[None]
    tt = torch.as_tensor(np.asarray(t, dtype=np.int16))[None]
    res = banded_affine_sw_batch(qt, tt, torch.tensor([len(q)]), torch.tensor([len(t)]), cfg,
                                 half_band=hb, band_offset=torch.tensor([off]),
                                 return_matrices=True)
    ext = traceback_banded(res, 0, np.asarray(q), np.asarray(t), cfg)
    return dict(score=float(res.score[0]), qe=int(res.query_end[0]), te=int(res.target_end[0]),
                qs=int(ext.read_start), ts=int(ext.ref_start), cigar=cigar_words(ext.cigar),
                counts=[ext.n_match, ext.n_mismatch, ext.n_insertion, ext.n_deletion])


def make_sw(rng):
    cases = []  # (q, t, hb, off, params, tag)
    default = (2.0, 4.0, 6.0, 2.0, 600.0)
    cfg1 = (2.0, 4.0, 4.0, 2.0, 0.0)
    # known answers from the reference's own tests
    cases.append((encode_bases("ACGT"), encode_bases("TTACGTAA"), 2, 2, default, "ka_acgt"))
    s40 = "".join(rng.choice(list("ACGT"), size=40))
    cases.append((encode_bases(s40), encode_bases(s40), 8, 0, default, "ka_identical40"))
    # edge cases
    r = lambda n: rng.integers(1, 5, size=n).astype(np.int8)  # noqa: E731
    cases.append((np.zeros(0, np.int8), r(10), 3, 0, default, "empty_query"))
    cases.append((r(1), r(1), 0, 0, default, "one_base_hb0"))
    x = r(30)
    cases.append((x, x.copy(), 0, 0, default, "hb0_identical"))
    cases.append((r(20), r(20), 5, 40, default, "band_right_of_target"))
    cases.append((r(20), r(20), 5, -40, default, "band_left_of_target"))
    y = r(50)
    cases.append((y[5:45], y, 4, -3, default, "negative_offset"))
    yn = y.copy()
    yn[[3, 10, 22]] = 5
    cases.append((yn, y, 6, 0, default, "query_N"))
    cases.append((y, yn, 6, 0, default, "target_N"))
    cases.append((yn, yn.copy(), 6, 0, default, "both_N"))
    cases.append((r(25), r(60), 40, 10, default, "band_wider_than_target"))
    # x-drop: a matching prefix followed by random sequence
    base = r(200)
    qx = np.concatenate([base[:80], r(120)])
    for xd in (5.0, 10.0, 20.0, 40.0):
        cases.append((qx, base, 10, 0, (2.0, 4.0, 6.0, 2.0, xd), f"xdrop_{int(xd)}"))
    # gap-heavy pairs: insertions and deletions of several lengths
    for L in (1, 2, 3, 5, 8):
        t0 = r(120)
        q_ins = np.concatenate([t0[:60], r(L), t0[60:]])
        q_del = np.concatenate([t0[:60], t0[60 + L:]])
        cases.append((q_ins, t0, 12, 0, default, f"ins_{L}"))
        cases.append((q_del, t0, 12, 0, default, f"del_{L}"))
        cases.append((q_ins, t0, 12, 0, cfg1, f"ins_{L}_cfg1"))
        cases.append((q_del, t0, 12, 0, cfg1, f"del_{L}_cfg1"))
    # exhaustive-ish tiny cases: every small band / offset / length combination
    for hb in (0, 1, 2, 3):
        for off in range(-3, 6):
            for ql in (1, 2, 4, 7):
                for tl in (1, 3, 6, 9):
                    cases.append((r(ql), r(tl), hb, off, default, "tiny"))
    # random scoring parameters (integers, including open < extend)
    for k in range(40):
        ql = int(rng.integers(5, 60))
        t0 = r(ql + int(rng.integers(0, 20)))
        q0 = synth.apply_errors(t0[: ql], synth.ONT, rng)
        params = (float(rng.integers(1, 5)), float(rng.integers(1, 7)), float(rng.integers(0, 9)),
                  float(rng.integers(0, 5)), float(rng.choice([0, 0, 7, 15, 600])))
        cases.append((q0, t0, int(rng.integers(0, 12)), int(rng.integers(-5, 10)), params, "randparams"))
    # the 150 bp extension workload, first 150 pairs
    ps = synth.extension_pairs_150bp(n_pairs=150, seed=11, ref_len=200_000)
    for b in range(len(ps)):
        cases.append((ps.q(b), ps.t(b), 32, 32, cfg1, "cfg1"))
    # mixed-profile medium pairs with widened bands
    mixed = synth.extension_pairs_mixed(n_pairs=24, seed=5, ref_len=400_000, max_len=1500,
                                        log_mean=6.0, log_sigma=0.6)
    for b in range(len(mixed)):
        cases.append((mixed.q(b), mixed.t(b), int(mixed.half_band[b]), 32, default, "mixed"))
    out = [sw_case(q, t, hb, off, p) for (q, t, hb, off, p, _) in cases]
    q_flat, q_off = ragged([c[0] for c in cases], np.int8)
    t_flat, t_off = ragged([c[1] for c in cases], np.int8)
    cg_flat, cg_off = ragged([o["cigar"] for o in out], np.uint32)
    np.savez_compressed(
        os.path.join(HERE, "sw_golden.npz"),
        query=q_flat, query_off=q_off, target=t_flat, target_off=t_off,
        half_band=np.array([c[2] for c in cases], np.int32),
        band_offset=np.array([c[3] for c in cases], np.int32),
        params=np.array([c[4] for c in cases], np.float64),
        tag=np.array([c[5] for c in cases]),
        score=np.array([o["score"] for o in out], np.float32),
        query_end=np.array([o["qe"] for o in out], np.int64),
        target_end=np.array([o["te"] for o in out], np.int64),
        query_start=np.array([o["qs"] for o in out], np.int64),
        target_start=np.array([o["ts"] for o in out], np.int64),
        counts=np.array([o["counts"] for o in out], np.int64),
        cigar=cg_flat, cigar_off=cg_off,
    )
    print(f"sw_golden.npz: {len(cases)} pairs")


# --------------------------------------------------------------------------- #
# Chaining
# --------------------------------------------------------------------------- #
def lut_for(cfg: ChainingConfig) -> np.ndarray:
    gap = np.arange(cfg.max_gap + 1, dtype=np.int64)
    return np.where(gap > 0, cfg.gap_open + cfg.gap_extend * gap + cfg.log_coeff * np.log2(gap + 1.0), 0.0)


def chimeric_batch(rng, n_reads=10):
    """Reads stitched from 2-3 segments (either strand) of a reference that
    also carries a diverged copy of one region, so reads have several chains
    on both strands, secondary candidates and overlapping repeats."""
    ref = synth.random_reference(600_000, rng)
    src = ref[100_000:104_000].copy()
    dup = synth.apply_errors(src, synth.ErrorProfile(0.01, 0.0, 0.0), rng)[:4000]
    ref[400_000:400_000 + len(dup)] = dup
    sketch = synth.MinimizerSketch(ref, k=15, w=10)
    rp, fp, ln, st, counts, rl = [], [], [], [], [], []
    for r in range(n_reads):
        parts = []
        for s in range(int(rng.integers(2, 4))):
            L = int(rng.integers(600, 2500))
            if r % 3 == 0 and s == 0:
                start = 100_000 + int(rng.integers(0, 1000))  # lands in the repeat
            else:
                start = int(rng.integers(0, len(ref) - L))
            seg = ref[start:start + L]
            if rng.random() < 0.5:
                seg = synth.reverse_complement(seg)
            parts.append(synth.apply_errors(seg, synth.HIFI, rng))
        read = np.concatenate(parts)
        n = 0
        for strand, codes in ((1, read), (-1, synth.reverse_complement(read))):
            a, b = sketch.query(codes)
            rp.append(a); fp.append(b)
            ln.append(np.full(len(a), 15, np.int64)); st.append(np.full(len(a), strand, np.int8))
            n += len(a)
        counts.append(n)
        rl.append(len(read))
    off = np.zeros(n_reads + 1, np.int64)
    np.cumsum(counts, out=off[1:])
    return synth.AnchorBatch(off, np.concatenate(rp).astype(np.int32), np.concatenate(fp).astype(np.int32),
                             np.concatenate(ln).astype(np.int32), np.concatenate(st).astype(np.int8),
                             np.array(rl, np.int64))


def group_batch(rng, n_reads=8):
    """Hand-built anchor sets: many collinear groups with distinct or
    overlapping read spans and random strands, to exercise the score cutoff,
    the overlap filter and the max_chains cap of select()."""
    rp, fp, ln, st, counts = [], [], [], [], []
    for r in range(n_reads):
        n_groups = int(rng.integers(3, 14))
        n = 0
        for g in range(n_groups):
            k = int(rng.integers(2, 40))
            start = int(rng.integers(0, 20_000)) if r % 2 else g * 1500
            diag = int(rng.integers(0, 5_000_000))
            pos = start + np.cumsum(rng.integers(10, 40, size=k))
            drift = np.cumsum(rng.integers(-2, 3, size=k)) if r % 4 == 3 else 0
            rp.append(pos)
            fp.append(pos + diag + drift)
            ln.append(rng.integers(12, 25, size=k))
            st.append(np.full(k, 1 if rng.random() < 0.6 else -1, np.int8))
            n += k
        counts.append(n)
    off = np.zeros(n_reads + 1, np.int64)
    np.cumsum(counts, out=off[1:])
    return synth.AnchorBatch(off, np.concatenate(rp).astype(np.int32), np.concatenate(fp).astype(np.int32),
                             np.concatenate(ln).astype(np.int32), np.concatenate(st).astype(np.int8),
                             np.full(n_reads, 30_000, np.int64))


def make_chain(rng):
    # --- DP level ---
    dp_cases = []  # (read_end, ref_end, weight, bonus or None, lookback, max_gap)
    dp_cases.append((np.array([10, 20, 30]), np.array([10, 20, 31]), np.array([10.5, 9.25, 8.75]),
                     None, 64, 5000))
    for trial in range(40):
        n = int(rng.integers(1, 120))
        re = np.sort(rng.integers(1, 2000, size=n)).astype(np.int64)
        fe = np.sort(rng.integers(1, 2000, size=n)).astype(np.int64)
        w = rng.integers(5, 40, size=n).astype(np.float64)
        if trial % 3 == 0:
            w = w + rng.random(n)  # fractional weights (hybrid gate)
        lb = int(rng.choice([1, 4, 16, 50, 64, 200]))
        mg = int(rng.choice([100, 500, 5000]))
        bonus = None
        if trial % 4 == 1:
            bonus = rng.normal(0, 3, size=(n, lb))
        dp_cases.append((re, fe, w, bonus, lb, mg))
    # ties: equal scores from several predecessors (collinear grid)
    re = np.repeat(np.arange(1, 21) * 10, 1)
    dp_cases.append((re, re.copy(), np.full(20, 15.0), None, 8, 5000))
    grid = np.array([10, 10, 20, 20, 30, 30, 40, 40])
    dp_cases.append((grid, np.array([10, 12, 20, 22, 30, 32, 40, 42]), np.full(8, 12.0), None, 4, 5000))
    f_all, p_all = [], []
    for (re, fe, w, bonus, lb, mg) in dp_cases:
        cfg = ChainingConfig(max_lookback=lb, max_gap=mg)
        f, p = chain_dp_numpy(re, fe, w, cfg, bonus=bonus)
        f_all.append(f)
        p_all.append(p)
    re_flat, dp_off = ragged([c[0] for c in dp_cases], np.int64)
    fe_flat, _ = ragged([c[1] for c in dp_cases], np.int64)
    w_flat, _ = ragged([c[2] for c in dp_cases], np.float64)
    has_bonus = np.array([c[3] is not None for c in dp_cases])
    bonus_flat, bonus_off = ragged([np.asarray(c[3]).ravel() if c[3] is not None else np.zeros(0)
                                    for c in dp_cases], np.float64)
    f_flat, _ = ragged(f_all, np.float64)
    p_flat, _ = ragged(p_all, np.int64)

    # --- chain() level on simulated minimizer anchors ---
    batches = [
        synth.chaining_reads_hifi(n_reads=24, seed=21, ref_len=1_000_000, mean_len=3000),
        synth.chaining_reads_hifi(n_reads=4, seed=22, ref_len=2_000_000, mean_len=15_000),
        synth.chaining_reads_hifi(n_reads=6, seed=23, ref_len=500_000, mean_len=4000,
                                  profile=synth.ONT),
    ]
    lookbacks = [50, 50, 200]
    batches.append(chimeric_batch(rng))
    lookbacks.append(50)
    batches.append(group_batch(rng))
    lookbacks.append(64)
    reads_rp, reads_fp, reads_ln, reads_st, read_lb = [], [], [], [], []
    ch_score, ch_strand, ch_span, ch_primary, ch_members, ch_count = [], [], [], [], [], []
    for batch, lb in zip(batches, lookbacks):
        cfg = ChainingConfig(max_lookback=lb, max_gap=5000)
        chainer = AffineChainer(cfg, backend="torch", workers=1)
        for r in range(len(batch)):
            rp, fp, ln, st = batch.read(r)
            anchors = AnchorSet.from_lists(rp.astype(np.int64), fp.astype(np.int64),
                                           ln.astype(np.int64), st.astype(np.int8))
            chains = chainer.chain(anchors, device="cpu")
            reads_rp.append(rp)
            reads_fp.append(fp)
            reads_ln.append(ln)
            reads_st.append(st)
            read_lb.append(lb)
            ch_count.append(len(chains))
            for c in chains:
                ch_score.append(c.score)
                ch_strand.append(c.strand)
                ch_span.append([c.read_start, c.read_end, c.ref_start, c.ref_end])
                ch_primary.append(c.is_primary)
                ch_members.append(np.asarray(c.anchor_idx, np.int64))
    rp_flat, read_off = ragged(reads_rp, np.int64)
    fp_flat, _ = ragged(reads_fp, np.int64)
    ln_flat, _ = ragged(reads_ln, np.int64)
    st_flat, _ = ragged(reads_st, np.int8)
    mem_flat, mem_off = ragged(ch_members, np.int64)
    np.savez_compressed(
        os.path.join(HERE, "chain_golden.npz"),
        lut_default=lut_for(ChainingConfig()),
        dp_read_end=re_flat, dp_ref_end=fe_flat, dp_weight=w_flat, dp_off=dp_off,
        dp_has_bonus=has_bonus, dp_bonus=bonus_flat, dp_bonus_off=bonus_off,
        dp_lookback=np.array([c[4] for c in dp_cases], np.int32),
        dp_max_gap=np.array([c[5] for c in dp_cases], np.int64),
        dp_f=f_flat, dp_parent=p_flat,
        read_pos=rp_flat, ref_pos=fp_flat, length=ln_flat, strand=st_flat, read_off=read_off,
        read_lookback=np.array(read_lb, np.int32),
        n_chains=np.array(ch_count, np.int32), chain_score=np.array(ch_score, np.float64),
        chain_strand=np.array(ch_strand, np.int32), chain_span=np.array(ch_span, np.int64).reshape(-1, 4),
        chain_primary=np.array(ch_primary, bool), chain_members=mem_flat, chain_members_off=mem_off,
    )
    print(f"chain_golden.npz: {len(dp_cases)} DP cases, {len(reads_rp)} reads, {len(ch_score)} chains")


# --------------------------------------------------------------------------- #
# extend_chains (stage level)
# --------------------------------------------------------------------------- #
def make_extend(rng):
    ref = synth.random_reference(300_000, rng)
    ref_str = synth.decode_bases(ref)
    cfg = ExtensionConfig()
    eng = ExtensionEngine(cfg, device="cpu", backend="torch")
    reads, chain_rows, results = [], [], []
    for k in range(30):
        L = int(rng.integers(120, 900))
        s = int(rng.integers(200, len(ref) - L - 200))
        prof = (synth.ILLUMINA, synth.HIFI, synth.ONT)[k % 3]
        tmpl = ref[s: s + L]
        strand = 1 if k % 2 == 0 else -1
        if strand < 0:
            tmpl = synth.reverse_complement(tmpl)
        read = synth.apply_errors(tmpl, prof, rng)
        oriented = read if strand > 0 else synth.reverse_complement(read)
        # a chain of 3 anchors along the true diagonal, with a jittered diagonal
        n = len(oriented)
        rp = np.array([5, n // 2, max(n - 40, 6)], np.int64)
        jit = rng.integers(-6, 7, size=3)
        fp = s + rp + jit
        ln = np.array([15, 15, 15], np.int64)
        anchors = AnchorSet.from_lists(rp, fp, ln, np.full(3, strand, np.int8))
        chain = Chain(anchor_idx=np.arange(3), score=40.0, strand=strand,
                      read_start=int(rp.min()), read_end=int((rp + ln).max()),
                      ref_start=int(fp.min()), ref_end=int((fp + ln).max()))
        res = eng.extend_chains(synth.decode_bases(read), [chain], anchors, ref_str)[0]
        reads.append(read)
        chain_rows.append(np.concatenate([rp, fp, ln, [strand]]))
        results.append(res)
    r_flat, r_off = ragged(reads, np.int8)
    cg_flat, cg_off = ragged([cigar_words(x.cigar) for x in results], np.uint32)
    np.savez_compressed(
        os.path.join(HERE, "extend_golden.npz"),
        ref=ref, reads=r_flat, read_off=r_off, chains=np.array(chain_rows, np.int64),
        score=np.array([x.score for x in results], np.float64),
        read_start=np.array([x.read_start for x in results], np.int64),
        read_end=np.array([x.read_end for x in results], np.int64),
        ref_start=np.array([x.ref_start for x in results], np.int64),
        ref_end=np.array([x.ref_end for x in results], np.int64),
        counts=np.array([[x.n_match, x.n_mismatch, x.n_insertion, x.n_deletion] for x in results]),
        cigar=cg_flat, cigar_off=cg_off,
        cfg=np.array([cfg.match_score, cfg.mismatch_penalty, cfg.gap_open, cfg.gap_extend,
                      cfg.x_drop, cfg.half_band, cfg.max_half_band, cfg.flank, cfg.max_window]),
    )
    print(f"extend_golden.npz: {len(results)} single-chain extensions")


# --------------------------------------------------------------------------- #
# hybrid-mode chain() (gated weights, graph + learned-transition bonus)
# --------------------------------------------------------------------------- #
def make_hybrid(rng):
    from graphmambaformer.alignment.chaining import ChainingContext, GraphDistanceOracle

    n_nodes = 60
    edges = np.array([[i, i + 1] for i in range(n_nodes - 1)] + [[3, 10], [20, 35], [40, 41]]).T
    oracle = GraphDistanceOracle(edges, n_nodes, max_hops=3)
    backbone = np.zeros(n_nodes, dtype=bool)
    backbone[::2] = True
    reads = []
    for r in range(16):
        n_groups = int(rng.integers(1, 4))
        rp, fp, ln, st, nid, sc = [], [], [], [], [], []
        for g in range(n_groups):
            k = int(rng.integers(3, 30))
            start = int(rng.integers(0, 8000))
            diag = int(rng.integers(0, 200_000))
            pos = start + np.cumsum(rng.integers(8, 40, size=k))
            rp.append(pos)
            fp.append(pos + diag + np.cumsum(rng.integers(-3, 4, size=k)))
            ln.append(rng.integers(12, 30, size=k))
            st.append(np.full(k, 1 if rng.random() < 0.7 else -1, np.int8))
            nid.append(np.where(rng.random(k) < 0.8, rng.integers(0, n_nodes, size=k), -1))
            sc.append(rng.random(k).astype(np.float32) if r % 3 else np.full(k, np.nan, np.float32))
        rp, fp, ln = (np.concatenate(x).astype(np.int64) for x in (rp, fp, ln))
        a = AnchorSet.from_lists(rp, fp, ln, np.concatenate(st), node_id=np.concatenate(nid))
        a.score = np.concatenate(sc)
        if r % 4 == 1:  # decisive scores: high for group anchors, low for a few
            a.score = np.where(rng.random(len(a)) < 0.8, 0.95, 0.05).astype(np.float32)
        trust = [None, True, False, None][r % 4]
        trans = None
        if trust:
            keys = [(int(a.read_pos[i]), int(a.ref_pos[i]), int(a.length[i]), int(a.strand[i]))
                    for i in range(len(a))]
            trans = {(keys[i], keys[i + 1]): float(rng.random()) for i in range(0, len(a) - 1, 2)}
        ctx = ChainingContext(oracle=oracle if r % 2 == 0 else None,
                              backbone=backbone if r % 3 != 2 else None,
                              trust_neural=trust, learned_transitions=trans)
        reads.append((a, ctx))
    cfg = ChainingConfig(max_lookback=16, max_gap=5000)
    chainer = AffineChainer(cfg, backend="torch", workers=1)
    out = [chainer.chain(a, ctx, device="cpu") for a, ctx in reads]
    import pickle

    payload = dict(
        edges=edges, n_nodes=n_nodes, backbone=backbone,
        reads=[dict(read_pos=a.read_pos, ref_pos=a.ref_pos, length=a.length, strand=a.strand,
                    node_id=a.node_id, score=a.score, use_oracle=ctx.oracle is not None,
                    use_backbone=ctx.backbone is not None, trust=ctx.trust_neural,
                    transitions=ctx.learned_transitions) for a, ctx in reads],
        chains=[[dict(score=c.score, strand=c.strand, span=(c.read_start, c.read_end, c.ref_start,
                                                             c.ref_end), primary=c.is_primary,
                      members=np.asarray(c.anchor_idx)) for c in chains] for chains in out],
        lookback=16,
    )
    with open(os.path.join(HERE, "hybrid_golden.pkl"), "wb") as fh:
        pickle.dump(payload, fh, protocol=4)
    print(f"hybrid_golden.pkl: {len(reads)} reads, {sum(len(c) for c in out)} chains")


def make_hybrid_inputs(rng):
    """The reference's hybrid-mode weight and bonus rows on strand-sorted
    anchor segments: each case keeps the segment's columns, the context and
    the config overrides, and the reference's outputs."""
    import pickle
    from dataclasses import replace

    from graphmambaformer.alignment.chaining import ChainingContext, GraphDistanceOracle

    graphs = []
    for n_nodes, extra in ((50, 6), (400, 120), (1500, 40)):
        chain = [[i, i + 1] for i in range(n_nodes - 1) if rng.random() < 0.92]  # some breaks: components
        more = rng.integers(0, n_nodes, size=(extra, 2)).tolist()
        edges = np.array(chain + more, dtype=np.int64).T
        graphs.append((edges, n_nodes))
    cases = []
    for c in range(60):
        edges, n_nodes = graphs[c % 3]
        hops = int((2, 3, 4)[c % 3])
        oracle = GraphDistanceOracle(edges, n_nodes, max_hops=hops)
        n = int(rng.integers(1, 90))
        rp = np.sort(rng.integers(0, 20_000, size=n)).astype(np.int64)
        fp = (rp + 1000 + rng.integers(-40, 40, size=n)).astype(np.int64)
        ln = rng.integers(10, 30, size=n).astype(np.int64)
        strand = 1 if c % 2 else -1
        if c % 7 == 3 and n > 4:  # duplicated anchor keys
            rp[1], fp[1], ln[1] = rp[0], fp[0], ln[0]
            rp[3], fp[3], ln[3] = rp[2], fp[2], ln[2]
        nid = np.where(rng.random(n) < 0.85, rng.integers(0, n_nodes, size=n), -1).astype(np.int64)
        a = AnchorSet.from_lists(rp, fp, ln, np.full(n, strand, np.int8), node_id=nid)
        kind = c % 5
        if kind == 0:
            a.score = np.full(n, np.nan, np.float32)
        elif kind == 1:
            a.score = np.where(rng.random(n) < 0.75, 0.97, 0.02).astype(np.float32)
        else:
            sc = rng.random(n).astype(np.float32)
            sc[rng.random(n) < 0.2] = np.nan
            a.score = sc
        sub, _ = a.for_strand(strand)
        sub, _ = sub.sorted_by_ref()
        trust = [None, True, False, True, None][c % 5]
        trans = None
        if trust is True:
            keys = [(int(sub.read_pos[i]), int(sub.ref_pos[i]), int(sub.length[i]), int(sub.strand[i]))
                    for i in range(len(sub))]
            trans = {}
            for i in range(len(sub)):
                for j in rng.integers(max(0, i - 40), i + 1, size=3):
                    if j < i:
                        trans[(keys[int(j)], keys[i])] = float(rng.random())
            trans[((-1, -1, 1, 1), keys[0])] = 0.5  # a key the segment does not have
            if len(sub) > 2:
                trans[(keys[0], keys[-1])] = float(rng.random())  # beyond most lookbacks
        backbone = (rng.random(n_nodes) < 0.5) if c % 3 != 1 else None
        ctx = ChainingContext(oracle=oracle if c % 4 != 2 else None, backbone=backbone, trust_neural=trust,
                              learned_transitions=trans)
        over = dict(max_lookback=int((1, 16, 50, 64, 7)[c % 5]),
                    graph_bonus=float((4.0, 2.5, 0.0, 4.0, 1.25)[c % 5]),
                    graph_max_hops=int((3, 2, 4, 1, 3)[c % 5]),
                    adaptive_seed_scoring=c % 6 != 5)
        cfg = replace(ChainingConfig(), **over)
        chainer = AffineChainer(cfg, backend="torch", workers=1)
        w = chainer._weights(sub, ctx)
        b = chainer._graph_bonus(sub, ctx)
        cases.append(dict(read_pos=sub.read_pos, ref_pos=sub.ref_pos, length=sub.length, strand=sub.strand,
                          node_id=sub.node_id, score=sub.score, edges=edges, n_nodes=n_nodes, max_hops=hops,
                          use_oracle=ctx.oracle is not None, backbone=backbone, trust=trust, transitions=trans,
                          cfg=over, weight=w, bonus=b))
    with open(os.path.join(HERE, "hybrid_inputs_golden.pkl"), "wb") as fh:
        pickle.dump(dict(cases=cases), fh, protocol=4)
    print(f"hybrid_inputs_golden.pkl: {len(cases)} segments, "
          f"{sum(c['bonus'] is not None for c in cases)} with a bonus")


def make_seed(rng):
    from graphmambaformer.alignment.seeding import MinimizerIndex, reverse_complement_codes

    cases = {}
    refs, reads_all, params, out = [], [], [], {"read_pos": [], "ref_pos": [], "length": []}
    for case, (ref_len, k, w, max_occ) in enumerate(((200_000, 15, 10, 0), (120_000, 11, 5, 5),
                                                      (150_000, 19, 12, 0))):
        ref = synth.random_reference(ref_len, rng)
        ref[5000:5040] = 5  # an N run
        blk = ref[20_000:20_400].copy()
        for s0 in (40_000, 60_000, 80_000, 100_000, 110_000, 115_000):
            ref[s0: s0 + 400] = blk  # a repeated block (caught by max_occ)
        idx = MinimizerIndex(ref, k=k, window=w, max_occ=max_occ)
        reads = [ref[1000:1010].copy(), ref[300:300 + k].copy()]
        for L in (150, 1000, 5000, 20_000):
            st = int(rng.integers(0, ref_len - L))
            reads.append(synth.apply_errors(ref[st: st + L], synth.ONT, rng))
        r = ref[20_000:20_600].copy()
        r[100:103] = 5
        reads.append(r)
        for read in reads:
            for strand, codes in ((1, read), (-1, reverse_complement_codes(read))):
                a, b, c = idx.query(codes)
                out["read_pos"].append(np.asarray(a, np.int64))
                out["ref_pos"].append(np.asarray(b, np.int64))
                out["length"].append(np.asarray(c, np.int64))
                params.append((case, len(reads_all), strand))
            reads_all.append(read)
        refs.append((ref, k, w, max_occ))
    cnt = np.array([len(x) for x in out["read_pos"]], np.int64)
    aoff = np.zeros(len(cnt) + 1, np.int64)
    np.cumsum(cnt, out=aoff[1:])
    rq, roff = ragged(reads_all, np.int8)
    fr, foff = ragged([x[0] for x in refs], np.int8)
    np.savez_compressed(
        os.path.join(HERE, "seed_golden.npz"),
        ref=fr, ref_off=foff, ref_kw=np.array([[k, w, mo] for _, k, w, mo in refs], np.int64),
        reads=rq, read_off=roff, query=np.array(params, np.int64), anchor_off=aoff,
        read_pos=np.concatenate(out["read_pos"]), ref_pos=np.concatenate(out["ref_pos"]),
        length=np.concatenate(out["length"]))


# --------------------------------------------------------------------------- #
# WavefrontAligner + multi-chain extend_chains (both algorithms)
# --------------------------------------------------------------------------- #
def make_wfa(rng):
    from graphmambaformer.alignment.extension import WavefrontAligner

    # ---- aligner cases: (query, target, max_distance) ----
    cases = [("ACGTACGTACGT", "ACGTACGTACGT", 4096), ("ACGT", "TGCA", 4096), ("AN", "AN", 4096),
             ("ACGTAC", "ACGTTAC", 4), ("", "", 4096), ("", "ACG", 4096), ("ACGTA", "", 4096),
             ("NNNN", "NNNN", 4096), ("A", "C", 0), ("A", "A", 0), ("ACGT", "ACGA", 1)]
    cases = [(encode_bases(a), encode_bases(b), d) for a, b, d in cases]
    for _ in range(3):  # unrelated sequences past a small budget (L1094-1103)
        cases.append((synth.random_reference(60, rng).astype(np.int8),
                       synth.random_reference(60, rng).astype(np.int8), 2))
    profiles = (synth.ILLUMINA, synth.HIFI, synth.ONT)
    for c in range(150):
        L = int(rng.choice([int(rng.integers(1, 40)), int(rng.integers(40, 400)), int(rng.integers(400, 3000))]))
        a = synth.random_reference(L, rng).astype(np.int8)
        b = synth.apply_errors(a, profiles[c % 3], rng).astype(np.int8)
        if c % 7 == 0 and L > 10:
            a[rng.integers(0, L, size=max(1, L // 50))] = 5
        if c % 5 == 0:
            b = np.concatenate([b, synth.random_reference(int(rng.integers(1, 30)), rng).astype(np.int8)])
        if c % 9 == 0:
            a, b = b, a
        md = int(rng.choice([4096, 4096, 50, 8]))
        cases.append((a, b, md))
    qs, ts, mds, dist, cig = [], [], [], [], []
    for a, b, md in cases:
        wfa = WavefrontAligner(ExtensionConfig(algorithm="wfa", wfa_max_distance=md))
        try:
            d, cigar = wfa.align(np.asarray(a, np.int8), np.asarray(b, np.int8))
        except RuntimeError:
            d, cigar = -1, []
        qs.append(a)
        ts.append(b)
        mds.append(md)
        dist.append(d)
        cig.append(cigar_words(cigar))
    q_flat, q_off = ragged(qs, np.int8)
    t_flat, t_off = ragged(ts, np.int8)
    c_flat, c_off = ragged(cig, np.uint32)

    # ---- extend_chains with several chains per read ----
    ref = synth.random_reference(400_000, rng)
    ref_str = synth.decode_bases(ref)
    reads, anc, chain_rows, call_rows, results = [], [], [], [], []
    for call in range(48):
        algo = call % 2  # 0 banded_sw, 1 wfa
        prof = profiles[(call // 2) % 3]
        L = int(rng.integers(100, 2500 if prof is synth.ILLUMINA else 4000))
        s0 = int(rng.integers(300, len(ref) - L - 300))
        strand = 1 if (call // 6) % 2 == 0 else -1
        tmpl = ref[s0: s0 + L]
        read = synth.apply_errors(tmpl if strand > 0 else synth.reverse_complement(tmpl), prof, rng)
        oriented = read if strand > 0 else synth.reverse_complement(read)
        n = len(oriented)
        rp_l, fp_l, ln_l, st_l, rows = [], [], [], [], []
        n_chains = int(rng.integers(1, 4))
        for c in range(n_chains):
            if c == 0:  # the true chain: anchors along the true diagonal
                k = int(rng.integers(2, 6))
                rp = np.sort(rng.choice(np.arange(0, max(n - 20, 1)), size=min(k, max(n - 20, 1)), replace=False))
                fp = s0 + rp + rng.integers(-4, 5, size=len(rp))
                cs = strand
            else:  # a secondary chain elsewhere, possibly the other strand, wider spread
                k = int(rng.integers(2, 5))
                rp = np.sort(rng.choice(np.arange(0, max(n - 20, 1)), size=min(k, max(n - 20, 1)), replace=False))
                base = int(rng.integers(500, len(ref) - n - 500))
                fp = base + rp + rng.integers(-40, 41, size=len(rp))
                cs = strand if rng.random() < 0.5 else -strand
            lo = len(np.concatenate(rp_l)) if rp_l else 0
            rp_l.append(rp.astype(np.int64))
            fp_l.append(fp.astype(np.int64))
            ln_l.append(np.full(len(rp), 15, np.int64))
            st_l.append(np.full(len(rp), cs, np.int8))
            rows.append((call, lo, lo + len(rp), cs))
        rp, fp, ln, st = (np.concatenate(x) for x in (rp_l, fp_l, ln_l, st_l))
        anchors = AnchorSet.from_lists(rp, fp, ln, st)
        chains = [Chain(anchor_idx=np.arange(lo, hi), score=30.0, strand=cs,
                        read_start=int(rp[lo:hi].min()), read_end=int((rp[lo:hi] + ln[lo:hi]).max()),
                        ref_start=int(fp[lo:hi].min()), ref_end=int((fp[lo:hi] + ln[lo:hi]).max()))
                  for (_, lo, hi, cs) in rows]
        md = int(rng.choice([4096, 4096, 30]))
        cfg = ExtensionConfig(algorithm="wfa" if algo else "banded_sw", wfa_max_distance=md)
        eng = ExtensionEngine(cfg, device="cpu", backend="torch")
        out = eng.extend_chains(synth.decode_bases(read), chains, anchors, ref_str)
        reads.append(read)
        anc.append(np.stack([rp, fp, ln, st.astype(np.int64)], 1))
        chain_rows.extend(rows)
        call_rows.append((algo, md))
        results.extend(out)
    r_flat, r_off = ragged(reads, np.int8)
    a_flat = np.concatenate(anc)
    a_off = np.zeros(len(anc) + 1, np.int64)
    np.cumsum([len(x) for x in anc], out=a_off[1:])
    x_flat, x_off = ragged([cigar_words(x.cigar) for x in results], np.uint32)
    np.savez_compressed(
        os.path.join(HERE, "wfa_golden.npz"),
        q=q_flat, q_off=q_off, t=t_flat, t_off=t_off, max_distance=np.array(mds, np.int64),
        distance=np.array(dist, np.int64), cigar=c_flat, cigar_off=c_off,
        ref=ref, reads=r_flat, read_off=r_off, anchors=a_flat, anchor_off=a_off,
        chains=np.array(chain_rows, np.int64), calls=np.array(call_rows, np.int64),
        x_score=np.array([x.score for x in results], np.float64),
        x_span=np.array([[x.read_start, x.read_end, x.ref_start, x.ref_end] for x in results], np.int64),
        x_counts=np.array([[x.n_match, x.n_mismatch, x.n_insertion, x.n_deletion] for x in results], np.int64),
        x_cigar=x_flat, x_cigar_off=x_off,
    )
    print(f"wfa_golden.npz: {len(cases)} aligner cases ({sum(d < 0 for d in dist)} over budget), "
          f"{len(call_rows)} extend calls, {len(results)} chains")


# --------------------------------------------------------------------------- #
# x-drop over a batch (all members must have dropped)
# --------------------------------------------------------------------------- #
def make_xdrop(rng):
    # ---- banded_affine_sw_batch: batches of 2-5 pairs, x_drop 20..60 ----
    bq, bt, bhb, boff, bgrp, bxd, out = [], [], [], [], [0], [], []
    for batch in range(24):
        B = int(rng.integers(2, 6))
        xd = float(rng.choice([20.0, 35.0, 60.0]))
        hb = int(rng.integers(4, 24))
        qs, ts, offs = [], [], []
        for _ in range(B):
            L = int(rng.integers(60, 400))
            t = synth.random_reference(L + 40, rng).astype(np.int8)
            q = t[20: 20 + L].copy()
            # a block of junk of random length somewhere: the pair drops there
            if rng.random() < 0.8:
                a0 = int(rng.integers(0, L))
                jl = len(q[a0: a0 + int(rng.integers(10, 80))])
                q[a0: a0 + jl] = synth.random_reference(jl, rng)
            q = synth.apply_errors(q, synth.ILLUMINA, rng).astype(np.int8)
            qs.append(q)
            ts.append(t)
            offs.append(20)
        M = max(len(x) for x in qs)
        N = max(len(x) for x in ts)
        qt = torch.full((B, M), -1, dtype=torch.int16)
        tt = torch.full((B, N), -1, dtype=torch.int16)
        for b in range(B):
            qt[b, : len(qs[b])] = torch.as_tensor(qs[b].astype(np.int16))
            tt[b, : len(ts[b])] = torch.as_tensor(ts[b].astype(np.int16))
        cfg = ExtensionConfig(x_drop=xd)
        res = banded_affine_sw_batch(qt, tt, torch.tensor([len(x) for x in qs]), torch.tensor([len(x) for x in ts]),
                                     cfg, half_band=hb, band_offset=torch.tensor(offs), return_matrices=True)
        for b in range(B):
            ext = traceback_banded(res, b, qs[b], ts[b], cfg)
            out.append(dict(score=float(res.score[b]), qe=int(res.query_end[b]), te=int(res.target_end[b]),
                            qs=int(ext.read_start), ts=int(ext.ref_start), cigar=cigar_words(ext.cigar)))
        bq += qs
        bt += ts
        bhb += [hb] * B
        boff += offs
        bgrp.append(bgrp[-1] + B)
        bxd.append(xd)

    # ---- extend_chains: reads with unalignable blocks + secondary chains ----
    ref = synth.random_reference(200_000, rng)
    ref_str = synth.decode_bases(ref)
    eng = ExtensionEngine(ExtensionConfig(), device="cpu", backend="torch")  # x_drop 600
    reads, anc, chain_rows, results = [], [], [], []
    for call in range(10):
        A = int(rng.integers(300, 700))
        J = int(rng.integers(900, 1600))
        Bn = int(rng.integers(300, 900))
        s0 = int(rng.integers(1000, len(ref) - 5000))
        read = ref[s0: s0 + A + J + Bn].copy()
        read[A: A + J] = synth.random_reference(J, rng)
        read = synth.apply_errors(read, synth.HIFI, rng).astype(np.int8)
        n = len(read)
        rp = np.array([5, A // 2, A + J + 10, n - 40], np.int64)
        fp = s0 + rp
        rows = [(call, 0, 4, 1)]
        n_sec = int(rng.integers(1, 3))
        rp_l, fp_l = [rp], [fp]
        for c in range(n_sec):
            r2 = np.sort(rng.choice(np.arange(0, n - 20), size=2, replace=False)).astype(np.int64)
            base = int(rng.integers(500, len(ref) - n - 500))
            f2 = base + r2 + rng.integers(-20, 21, size=2)
            lo = sum(len(x) for x in rp_l)
            rp_l.append(r2)
            fp_l.append(f2)
            rows.append((call, lo, lo + 2, 1))
        if call % 3 == 2:  # the read alone, one chain (the pair's own stop)
            rows = rows[:1]
            rp_l, fp_l = rp_l[:1], fp_l[:1]
        rpa, fpa = np.concatenate(rp_l), np.concatenate(fp_l)
        ln = np.full(len(rpa), 15, np.int64)
        st = np.ones(len(rpa), np.int8)
        anchors = AnchorSet.from_lists(rpa, fpa, ln, st)
        chains = [Chain(anchor_idx=np.arange(lo, hi), score=30.0, strand=1,
                        read_start=int(rpa[lo:hi].min()), read_end=int((rpa[lo:hi] + 15).max()),
                        ref_start=int(fpa[lo:hi].min()), ref_end=int((fpa[lo:hi] + 15).max()))
                  for (_, lo, hi, _) in rows]
        res = eng.extend_chains(synth.decode_bases(read), chains, anchors, ref_str)
        reads.append(read)
        anc.append(np.stack([rpa, fpa, ln, st.astype(np.int64)], 1))
        chain_rows.extend(rows)
        results.extend(res)
    q_flat, q_off = ragged(bq, np.int8)
    t_flat, t_off = ragged(bt, np.int8)
    c_flat, c_off = ragged([o["cigar"] for o in out], np.uint32)
    r_flat, r_off = ragged(reads, np.int8)
    a_flat = np.concatenate(anc)
    a_off = np.zeros(len(anc) + 1, np.int64)
    np.cumsum([len(x) for x in anc], out=a_off[1:])
    x_flat, x_off = ragged([cigar_words(x.cigar) for x in results], np.uint32)
    np.savez_compressed(
        os.path.join(HERE, "xdrop_golden.npz"),
        query=q_flat, query_off=q_off, target=t_flat, target_off=t_off, half_band=np.array(bhb, np.int32),
        band_offset=np.array(boff, np.int32), batch_off=np.array(bgrp, np.int64), x_drop=np.array(bxd),
        score=np.array([o["score"] for o in out]), qe=np.array([o["qe"] for o in out]),
        te=np.array([o["te"] for o in out]), qs=np.array([o["qs"] for o in out]),
        ts=np.array([o["ts"] for o in out]), cigar=c_flat, cigar_off=c_off,
        ref=ref, reads=r_flat, read_off=r_off, anchors=a_flat, anchor_off=a_off,
        chains=np.array(chain_rows, np.int64),
        x_score=np.array([x.score for x in results], np.float64),
        x_span=np.array([[x.read_start, x.read_end, x.ref_start, x.ref_end] for x in results], np.int64),
        x_counts=np.array([[x.n_match, x.n_mismatch, x.n_insertion, x.n_deletion] for x in results], np.int64),
        x_cigar=x_flat, x_cigar_off=x_off,
    )
    print(f"xdrop_golden.npz: {len(bgrp) - 1} batches ({len(out)} pairs), {len(reads)} reads, "
          f"{len(results)} chains")


# --------------------------------------------------------------------------- #
# record assembly + SAM segment fields
# --------------------------------------------------------------------------- #
class _Segment:
    """Stand-in for pysam.AlignedSegment: keeps every field assigned."""

    def __init__(self):
        self.query_name = None
        self.flag = 0
        self.reference_id = -1
        self.reference_start = -1
        self.mapping_quality = 255
        self.cigartuples = None
        self.next_reference_id = -1
        self.next_reference_start = -1
        self.template_length = 0
        self.query_sequence = None
        self.query_qualities = None
        self.tags = []

    def set_tag(self, key, value):
        self.tags.append((key, value))


class _Pysam:
    AlignedSegment = _Segment


def make_sam(rng):
    import pickle
    from types import SimpleNamespace

    from graphmambaformer.alignment.pipeline import AlignmentPipeline
    from graphmambaformer.alignment.seeding import SeedIndexBundle
    from graphmambaformer.alignment.types import AlignmentRecord, ReadAlignments
    from graphmambaformer.data import alignment_io, formats

    ref = synth.random_reference(300_000, rng)
    ref_str = synth.decode_bases(ref)
    bundle = object.__new__(SeedIndexBundle)
    bundle.node_starts = np.arange(0, len(ref), 1000, dtype=np.int64)
    bundle.node_ids = np.arange(len(bundle.node_starts), dtype=np.int64) * 3 + 7
    reference = SimpleNamespace(ref_id=0, bundle=bundle)
    stub = SimpleNamespace(uses_neural_scoring=False, mode="fast",
                           cfg=SimpleNamespace(scoring=SimpleNamespace(max_mapq=60)))
    profiles = (synth.ILLUMINA, synth.HIFI, synth.ONT)
    modalities = ("illumina", "pacbio_hifi", "ont")
    reads_in, results, calls = [], [], []
    for r in range(36):
        algo = r % 2
        prof = profiles[(r // 2) % 3]
        L = int(rng.integers(80, 1500))
        s0 = int(rng.integers(500, len(ref) - L - 500))
        strand = 1 if (r // 4) % 2 == 0 else -1
        tmpl = ref[s0: s0 + L]
        read = synth.apply_errors(tmpl if strand > 0 else synth.reverse_complement(tmpl), prof, rng)
        seq = synth.decode_bases(read)
        if r % 9 == 4:  # bases outside ACGTN ride along in SEQ
            seq = seq[:10] + "R" + seq[11:20] + "a" + seq[21:]
        oriented = read if strand > 0 else synth.reverse_complement(read)
        n = len(oriented)
        rp_l, fp_l, rows = [], [], []
        n_chains = 0 if r % 7 == 6 else int(rng.integers(1, 4))
        for c in range(n_chains):
            k = int(rng.integers(2, 5))
            rp = np.sort(rng.choice(np.arange(0, max(n - 20, 1)), size=min(k, max(n - 20, 1)), replace=False))
            if c == 0:
                fp = s0 + rp + rng.integers(-3, 4, size=len(rp))
                cs = strand
            else:
                base = int(rng.integers(1000, len(ref) - n - 1000))
                fp = base + rp + rng.integers(-30, 31, size=len(rp))
                cs = strand if rng.random() < 0.5 else -strand
            lo = sum(len(x) for x in rp_l)
            rp_l.append(rp.astype(np.int64))
            fp_l.append(fp.astype(np.int64))
            rows.append((lo, lo + len(rp), cs))
        rpa = np.concatenate(rp_l) if rp_l else np.zeros(0, np.int64)
        fpa = np.concatenate(fp_l) if fp_l else np.zeros(0, np.int64)
        ln = np.full(len(rpa), 15, np.int64)
        st = np.concatenate([np.full(hi - lo, cs, np.int8) for lo, hi, cs in rows]) if rows else np.zeros(0, np.int8)
        anchors = AnchorSet.from_lists(rpa, fpa, ln, st)
        chains = [Chain(anchor_idx=np.arange(lo, hi), score=float(rng.integers(20, 400)), strand=cs,
                        read_start=int(rpa[lo:hi].min()), read_end=int((rpa[lo:hi] + 15).max()),
                        ref_start=int(fpa[lo:hi].min()), ref_end=int((fpa[lo:hi] + 15).max()),
                        is_primary=(c == 0))
                  for c, (lo, hi, cs) in enumerate(rows)]
        cfg = ExtensionConfig(algorithm="wfa" if algo else "banded_sw")
        eng = ExtensionEngine(cfg, device="cpu", backend="torch")
        exts = eng.extend_chains(seq, chains, anchors, ref_str) if chains else []
        if r % 11 == 3 and exts:
            exts = exts[:1]  # fewer extensions than chains: the rest keep chain spans, no CIGAR
        rid = f"read{r}/{L}"
        mapq = AlignmentPipeline._margin_mapq(stub, chains)
        records = AlignmentPipeline._records(stub, rid, len(seq), anchors, chains, exts, reference, mapq=mapq,
                                             route="fast")
        records = records or [AlignmentRecord.unmapped(rid, len(seq), pass_name="fast")]
        if r % 13 == 5:  # a record whose CIGAR does not cover the read, and one with an empty span
            records.append(AlignmentRecord(read_id=rid, read_len=len(seq), ref_id=0, ref_start=100, ref_end=160,
                                           strand=-1, mapq=7, cigar=[("=", 5)], is_mapped=True,
                                           is_primary=False))
            records.append(AlignmentRecord(read_id=rid, read_len=len(seq), ref_id=0, ref_start=100, ref_end=100,
                                           strand=1, mapq=7, cigar=[("=", len(seq))], is_mapped=True,
                                           is_primary=False))
        res = ReadAlignments(read_id=rid, read_len=len(seq), anchors=anchors, chains=list(chains), records=records)
        quals = None
        if r % 3 == 1:
            quals = [int(q) for q in rng.integers(-5, 120, size=len(seq) - (7 if r % 6 == 1 else 0))]
        src = seq if quals is None and r % 4 == 0 else SimpleNamespace(read_id=rid, seq=seq, quals=quals,
                                                                       modality=modalities[(r // 2) % 3])
        reads_in.append(src)
        results.append(res)
        calls.append(dict(read_id=rid, seq=seq, quals=quals, modality=None if isinstance(src, str) else src.modality,
                          anchors=np.stack([rpa, fpa, ln, st.astype(np.int64)], 1) if len(rpa) else np.zeros((0, 4),
                                                                                                        np.int64),
                          chains=[(lo, hi, cs, ch.score, ch.is_primary) for (lo, hi, cs), ch in zip(rows, chains)],
                          algo=algo, n_ext=len(exts), mapq=mapq,
                          ext=[dict(score=e.score, cigar=list(e.cigar), read_start=e.read_start, read_end=e.read_end,
                                    ref_start=e.ref_start, ref_end=e.ref_end,
                                    counts=(e.n_match, e.n_mismatch, e.n_insertion, e.n_deletion)) for e in exts],
                          records=[dict(vars(x), extension=None) for x in records]))
    out = {}
    refs = {0: SimpleNamespace(seq=ref_str)}
    for inc in (False, True):
        for names in (None, {0: "chr21"}):
            recs = alignment_io.alignments_to_records(results, reads_in, modality="pacbio_hifi",
                                                      include_secondary=inc)
            sq, ref_index = formats._sq_from_references(refs, names)
            segs = []
            for rec in recs:
                a = formats._make_segment(_Pysam, rec, ref_index)
                segs.append(dict(qname=a.query_name, flag=a.flag, ref=a.reference_id, pos=a.reference_start,
                                 mapq=a.mapping_quality, cigar=a.cigartuples, seq=a.query_sequence,
                                 qual=None if a.query_qualities is None else list(a.query_qualities),
                                 tags=list(a.tags), rnext=a.next_reference_id, pnext=a.next_reference_start,
                                 tlen=a.template_length))
            out[(inc, None if names is None else "chr21")] = dict(sq=sq, segments=segs)
    payload = dict(ref=ref, node_starts=bundle.node_starts, node_ids=bundle.node_ids, calls=calls, outputs=out,
                   header_rg=[formats._rg_from_records(alignment_io.alignments_to_records(
                       results, reads_in, modality="pacbio_hifi", include_secondary=True))])
    with open(os.path.join(HERE, "sam_golden.pkl"), "wb") as fh:
        pickle.dump(payload, fh, protocol=4)
    print(f"sam_golden.pkl: {len(calls)} reads, "
          f"{sum(len(c['records']) for c in calls)} records, "
          f"{len(out[(True, None)]['segments'])} segments with secondaries")


def make_pipeline(rng):
    """``FastAlignmentPipeline.align`` (pipeline.py L438-512) with its stock
    stage objects on the CPU: minimizer seeding (k=15, w=10), AffineChainer
    (chain_dp_numpy, f64), ExtensionEngine in both algorithms, margin MAPQ
    and records.  Stored per read: the seed stage's anchors (the input a
    drop-in chainer receives), the chains, the extensions and the records."""
    import pickle

    from graphmambaformer.alignment.pipeline import FastAlignmentPipeline
    from graphmambaformer.config import AccelConfig, PipelineConfig, SeedingConfig

    ref = synth.random_reference(400_000, rng)
    ref[200_000:200_050] = 5  # an N run
    ref_str = synth.decode_bases(ref)
    reads, ids = [], []
    for r in range(28):
        kind = r % 7
        if kind == 6:  # nothing to map
            read = synth.random_reference(int(rng.integers(300, 2000)), rng)
        else:
            prof = (synth.HIFI, synth.ONT, synth.ILLUMINA)[kind % 3]
            L = 150 if prof is synth.ILLUMINA else int(rng.integers(1500, 6000))
            s0 = int(rng.integers(0, len(ref) - L))
            tmpl = ref[s0: s0 + L]
            read = synth.apply_errors(tmpl if r % 2 else synth.reverse_complement(tmpl), prof, rng)
            if kind == 4:  # chimeric: a second locus joined on, for secondary chains
                s1 = int(rng.integers(0, len(ref) - 1500))
                read = np.concatenate([read, synth.apply_errors(ref[s1: s1 + 1500], synth.HIFI, rng)])
            if kind == 5:  # a repeated stretch, mapped at two places
                read = np.concatenate([read, read[: min(len(read), 800)]])
        reads.append(synth.decode_bases(read))
        ids.append(f"r{r}")
    runs = {}
    for algorithm in ("banded_sw", "wfa"):
        cfg = PipelineConfig(mode="fast", seeding=SeedingConfig(modes=("minimizer",)),
                             extension=ExtensionConfig(algorithm=algorithm),
                             accel=AccelConfig(device="cpu", num_workers=1, apply_global_switches=False))
        pipe = FastAlignmentPipeline(cfg, device="cpu")
        index = pipe.build_reference(ref_str)
        results, _ = pipe.align(reads, index, read_ids=ids)
        per = []
        for res in results:
            a = res.anchors
            per.append(dict(
                anchors=np.stack([a.read_pos, a.ref_pos, a.length, a.strand.astype(np.int64)], 1)
                if len(a) else np.zeros((0, 4), np.int64),
                chains=[dict(anchor_idx=np.asarray(c.anchor_idx, np.int64), score=float(c.score), strand=int(c.strand),
                             span=(int(c.read_start), int(c.read_end), int(c.ref_start), int(c.ref_end)),
                             is_primary=bool(c.is_primary)) for c in res.chains],
                records=[dict(ref_id=int(x.ref_id), ref_start=int(x.ref_start), ref_end=int(x.ref_end),
                              strand=int(x.strand), mapq=int(x.mapq), chain_score=float(x.chain_score),
                              alignment_score=float(x.alignment_score), cigar=[(op, int(n)) for op, n in x.cigar],
                              is_mapped=bool(x.is_mapped), is_primary=bool(x.is_primary),
                              is_supplementary=bool(x.is_supplementary), n_anchors=int(x.n_anchors),
                              n_chains=int(x.n_chains), node_id=int(x.node_id)) for x in res.records]))
        runs[algorithm] = dict(config=dict(chaining=vars(cfg.chaining).copy(), extension=vars(cfg.extension).copy()),
                               reads=per)
        n_rec = sum(len(x["records"]) for x in per)
        n_map = sum(1 for x in per for y in x["records"] if y["is_mapped"])
        print(f"pipeline_golden.pkl [{algorithm}]: {len(per)} reads, {n_rec} records, {n_map} mapped")
    with open(os.path.join(HERE, "pipeline_golden.pkl"), "wb") as fh:
        pickle.dump(dict(ref=ref, reads=reads, ids=ids, runs=runs), fh, protocol=4)


if __name__ == "__main__":
    which = sys.argv[1:] or ["sw", "chain", "extend", "hybrid"]
    if "sw" in which:
        make_sw(np.random.default_rng(101))
    if "chain" in which:
        make_chain(np.random.default_rng(202))
    if "extend" in which:
        make_extend(np.random.default_rng(303))
    if "hybrid" in which:
        make_hybrid(np.random.default_rng(404))
    if "hybrid_inputs" in which:
        make_hybrid_inputs(np.random.default_rng(909))
    if "seed" in which:
        make_seed(np.random.default_rng(505))
    if "wfa" in which:
        make_wfa(np.random.default_rng(606))
    if "xdrop" in which:
        make_xdrop(np.random.default_rng(707))
    if "sam" in which:
        make_sam(np.random.default_rng(808))
    if "pipeline" in which:
        make_pipeline(np.random.default_rng(1010))
