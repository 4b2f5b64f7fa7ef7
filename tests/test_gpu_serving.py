"""Serving loop: the batch pipeline (chaining, windows, device gather of
queries and targets from the resident reference, banded SW) reproduces the
stage objects field for field, and a request gets the same alignments when
it is served alone as when it is served among concurrent requests."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pool():
    from graphmambaformer_b200 import synth

    return synth.mixed_read_pool(n_reads=120, seed=14, ref_len=2_000_000, max_len=8000)


def _ext_equal(x, y):
    return (x.score == y.score and x.cigar == y.cigar and x.read_start == y.read_start and
            x.read_end == y.read_end and x.ref_start == y.ref_start and x.ref_end == y.ref_end and
            (x.n_match, x.n_mismatch, x.n_insertion, x.n_deletion) ==
            (y.n_match, y.n_mismatch, y.n_insertion, y.n_deletion))


def test_batch_pipeline_matches_stage_objects(pool):
    import torch

    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.chaining import AffineChainer, ChainingConfig
    from graphmambaformer_b200.config import ExtensionConfig
    from graphmambaformer_b200.extension import ExtensionEngine
    from graphmambaformer_b200.serving import BatchAligner
    from graphmambaformer_b200.types import AnchorSet

    idx = np.arange(60)
    reads, anchors = pool.take(idx)
    ccfg, ecfg = ChainingConfig(), ExtensionConfig()
    ref_d = torch.from_numpy(pool.ref).to("cuda:0")
    got = BatchAligner(ref_d, "cuda:0", ccfg, ecfg).align(reads, anchors)
    sets = []
    for r in range(len(reads)):
        rp, fp, ln, st = anchors.read(r)
        sets.append(AnchorSet.from_lists(rp, fp, ln, st, read_len=len(reads[r]), ref_len=len(pool.ref)))
    chains = AffineChainer(ccfg, device="cuda:0").chain_batch(sets)
    want = ExtensionEngine(ecfg, device="cuda:0").extend_batch(
        [synth.decode_bases(x) for x in reads], chains, sets, synth.decode_bases(pool.ref))
    assert sum(len(x) for x in want) > 0
    for r in range(len(reads)):
        assert len(got[r]) == len(want[r]), r
        assert all(_ext_equal(x, y) for x, y in zip(got[r], want[r])), r


@pytest.mark.parametrize("bound", [4096, 30])
def test_batch_pipeline_wfa_mode_matches_stage_objects(pool, bound):
    """algorithm="wfa": the serving pipeline gathers the WFA windows on the
    device and gives what AffineChainer + ExtensionEngine(wfa) give; with a
    bound of 30 many chains fall back to banded SW one chain per call."""
    import torch

    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.chaining import AffineChainer, ChainingConfig
    from graphmambaformer_b200.config import ExtensionConfig
    from graphmambaformer_b200.extension import ExtensionEngine
    from graphmambaformer_b200.serving import BatchAligner
    from graphmambaformer_b200.types import AnchorSet

    idx = np.arange(80)
    reads, anchors = pool.take(idx)
    ccfg, ecfg = ChainingConfig(), ExtensionConfig(algorithm="wfa", wfa_max_distance=bound)
    ref_d = torch.from_numpy(pool.ref).to("cuda:0")
    got = BatchAligner(ref_d, "cuda:0", ccfg, ecfg).align(reads, anchors)
    sets = []
    for r in range(len(reads)):
        rp, fp, ln, st = anchors.read(r)
        sets.append(AnchorSet.from_lists(rp, fp, ln, st, read_len=len(reads[r]), ref_len=len(pool.ref)))
    chains = AffineChainer(ccfg, device="cuda:0").chain_batch(sets)
    want = ExtensionEngine(ecfg, device="cuda:0").extend_batch(
        [synth.decode_bases(x) for x in reads], chains, sets, synth.decode_bases(pool.ref))
    assert sum(len(x) for x in want) > 0
    n_clipped = 0
    for r in range(len(reads)):
        assert len(got[r]) == len(want[r]), r
        assert all(_ext_equal(x, y) for x, y in zip(got[r], want[r])), r
        n_clipped += sum(1 for y in want[r] if y.cigar and y.cigar[0][0] == "S")
    if bound == 30:
        assert n_clipped > 0  # some chains went through the banded-SW fallback (local, soft-clipped)


def test_serving_same_alone_and_in_the_mix(pool):
    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.serving import AlignServer, serve_stream

    reqs = synth.poisson_requests(24, reads_per_s=4000, pool_size=len(pool), seed=8, max_reads=16)
    srv = AlignServer(pool.ref, "cuda:0", workers=2, max_batch_reads=40).start()
    try:
        alone = []
        for _, idx in reqs:  # one request at a time
            reads, anchors = pool.take(idx)
            alone.append(srv.submit(reads, anchors).result(timeout=300))
        futs = [srv.submit(*pool.take(idx)) for _, idx in reqs]  # all at once: mixed into shared batches
        mixed = [f.result(timeout=300) for f in futs]
        st = serve_stream(srv, pool, reqs)  # paced Poisson arrivals
    finally:
        srv.stop()
    for a, b in zip(alone, mixed):
        assert len(a) == len(b)
        for ra, rb in zip(a, b):
            assert len(ra) == len(rb) and all(_ext_equal(x, y) for x, y in zip(ra, rb))
    assert st["requests"] >= 3 * len(reqs) and st["p99_ms"] >= st["p50_ms"] > 0
    assert srv.batches < st["requests"]  # requests were batched together


def test_device_seeding_server_matches_client_anchors(pool):
    """A server holding the minimizer index seeds requests of bare reads on
    the device and returns exactly what the client-side anchors give."""
    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.seeding import DeviceMinimizerIndex
    from graphmambaformer_b200.serving import AlignServer

    reqs = synth.poisson_requests(12, reads_per_s=4000, pool_size=len(pool), seed=18, max_reads=12)
    idx = DeviceMinimizerIndex(pool.ref, k=15, w=10, max_occ=200, device="cuda:0")
    a_srv = AlignServer(pool.ref, "cuda:0", workers=2, max_batch_reads=40).start()
    b_srv = AlignServer(pool.ref, "cuda:0", workers=2, max_batch_reads=40, index=idx).start()
    try:
        fa = [a_srv.submit(*pool.take(ix)) for _, ix in reqs]
        fb = [b_srv.submit(pool.take(ix)[0]) for _, ix in reqs]  # reads only
        ra = [f.result(timeout=300) for f in fa]
        rb = [f.result(timeout=300) for f in fb]
    finally:
        a_srv.stop()
        b_srv.stop()
    assert sum(len(x) for r in ra for x in r) > 0
    for x, y in zip(ra, rb):
        assert len(x) == len(y)
        for cx, cy in zip(x, y):
            assert len(cx) == len(cy) and all(_ext_equal(p, q) for p, q in zip(cx, cy))


def test_device_seeding_with_concurrent_workers(pool):
    """Three workers seeding on the device at the same time, each on its own
    stream, give every request what one request at a time gives (seeding
    must keep all of its work on the worker's stream)."""
    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.seeding import DeviceMinimizerIndex
    from graphmambaformer_b200.serving import AlignServer

    reqs = synth.poisson_requests(48, reads_per_s=20000, pool_size=len(pool), seed=28, max_reads=24)
    idx = DeviceMinimizerIndex(pool.ref, k=15, w=10, max_occ=200, device="cuda:0")
    one = AlignServer(pool.ref, "cuda:0", workers=1, max_batch_reads=24, index=idx).start()
    many = AlignServer(pool.ref, "cuda:0", workers=3, max_batch_reads=24, index=idx).start()
    try:
        alone = [one.submit(pool.take(ix)[0]).result(timeout=300) for _, ix in reqs]
        for _ in range(2):  # all at once, twice: batches of different requests overlap on the GPU
            futs = [many.submit(pool.take(ix)[0]) for _, ix in reqs]
            mixed = [f.result(timeout=300) for f in futs]
            for a, b in zip(alone, mixed):
                assert len(a) == len(b)
                for ra, rb in zip(a, b):
                    assert len(ra) == len(rb) and all(_ext_equal(x, y) for x, y in zip(ra, rb))
    finally:
        one.stop()
        many.stop()
    assert many.batches > 3


@pytest.mark.parametrize("algorithm", ["banded_sw", "wfa"])
def test_batch_record_table_and_sam_match_object_path(pool, algorithm):
    """The serving batch's records built as arrays (record_table over the
    chain and extension columns) equal the fast pipeline's per-read records
    from the stage objects (read_alignments over AffineChainer +
    ExtensionEngine), and their SAM text (sam_batch + render) equals the
    object path's (sam_records + render), secondaries included or not."""
    import torch

    from graphmambaformer_b200 import synth
    from graphmambaformer_b200.chaining import AffineChainer, ChainingConfig
    from graphmambaformer_b200.config import ExtensionConfig
    from graphmambaformer_b200.extension import ExtensionEngine
    from graphmambaformer_b200.records import read_alignments, record_table, render_sam, sam_batch, sam_records
    from graphmambaformer_b200.serving import BatchAligner
    from graphmambaformer_b200.types import AnchorSet, words_to_cigar

    idx = np.arange(70)
    reads, anchors = pool.take(idx)
    ccfg, ecfg = ChainingConfig(), ExtensionConfig(algorithm=algorithm)
    ref_d = torch.from_numpy(pool.ref).to("cuda:0")
    ba = BatchAligner(ref_d, "cuda:0", ccfg, ecfg).align(reads, anchors)
    table = record_table(ba)
    sets = []
    for r in range(len(reads)):
        rp, fp, ln, st = anchors.read(r)
        sets.append(AnchorSet.from_lists(rp, fp, ln, st, read_len=len(reads[r]), ref_len=len(pool.ref)))
    chains = AffineChainer(ccfg, device="cuda:0").chain_batch(sets)
    exts = ExtensionEngine(ecfg, device="cuda:0").extend_batch(
        [synth.decode_bases(x) for x in reads], chains, sets, synth.decode_bases(pool.ref))
    names = [f"q{r}" for r in range(len(reads))]
    objs = [read_alignments(names[r], len(reads[r]), sets[r], chains[r], exts[r]) for r in range(len(reads))]
    recs = [rec for ra in objs for rec in ra.records]
    assert len(recs) == len(table)
    assert any(not x.is_mapped for x in recs) == bool((table.ref_id < 0).any())
    for i, rec in enumerate(recs):
        assert (table.ref_id[i] >= 0) == rec.is_mapped, i
        if rec.is_mapped:
            assert (table.ref_start[i], table.ref_end[i], table.strand[i], table.mapq[i], bool(table.is_primary[i])) \
                == (rec.ref_start, rec.ref_end, rec.strand, rec.mapq, rec.is_primary), i
            assert words_to_cigar(table.cigar[table.cigar_off[i]: table.cigar_off[i + 1]]) == \
                [tuple(x) for x in rec.cigar], i
    seq_off = np.zeros(len(reads) + 1, np.int64)
    np.cumsum([len(x) for x in reads], out=seq_off[1:])
    codes = np.concatenate(reads).astype(np.int8)
    texts = [synth.decode_bases(x) for x in reads]
    refs = {0: len(pool.ref)}
    for secondary in (False, True):
        want = render_sam(sam_records(objs, texts, "ont", secondary, refs))
        got = render_sam(sam_batch(table, names, codes, seq_off, None, "ont", secondary, refs))
        assert got == want and len(got) > 0
