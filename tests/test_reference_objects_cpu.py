"""The drop-in boundary with the reference's own objects, on the CPU.

The stage objects replace the reference's ``pipeline.chainer`` /
``pipeline.extender`` (graphmambaformer/pipeline.py L222-231), which call
them with the reference's ``AnchorSet``, ``Chain``, ``ChainingConfig``,
``ExtensionConfig`` and ``ChainingContext`` objects (the last holding the
reference's ``GraphDistanceOracle``).  These tests import the reference
from the checkout named by ``$GMF_REFERENCE`` (they are skipped without it)
and check every host-side step of the drop-in on those objects: anchor
batching, the chaining and scoring parameter blocks, the extension window
and band of each chain (against the reference's own ``_window``), and the
hybrid-mode weight and bonus rows (against the reference's own
``_weights`` / ``_graph_bonus``, with the reference's graph oracle object
inside the context).  The device calls that follow are covered by the GPU
suites on the same arrays.
"""

from __future__ import annotations

import os
import sys
from dataclasses import fields

import numpy as np
import pytest

REF = os.environ.get("GMF_REFERENCE")
pytestmark = pytest.mark.skipif(not REF or not os.path.isdir(os.path.join(REF or "", "graphmambaformer")),
                                reason="set $GMF_REFERENCE to a checkout of the reference")


@pytest.fixture(scope="module")
def ref():
    sys.dont_write_bytecode = True
    if REF not in sys.path:
        sys.path.append(REF)
    import graphmambaformer.alignment.chaining as chaining
    import graphmambaformer.alignment.extension as extension
    import graphmambaformer.alignment.types as types
    import graphmambaformer.config as config

    return dict(chaining=chaining, extension=extension, types=types, config=config)


def _reads(ref, n=12, seed=5):
    """Reference AnchorSets of simulated reads (both strands, node ids,
    neural scores on every other read)."""
    from graphmambaformer_b200 import synth

    batch = synth.chaining_reads_hifi(n_reads=n, seed=seed, ref_len=1_000_000, mean_len=3000)
    rng = np.random.default_rng(seed)
    sets = []
    for r in range(len(batch)):
        rp, fp, ln, st = batch.read(r)
        a = ref["types"].AnchorSet.from_lists(rp, fp, ln, st, node_id=rng.integers(-1, 40, len(rp)),
                                              read_len=int(batch.read_len[r]), ref_len=1_000_000)
        if r % 2:
            a.score = rng.random(len(a)).astype(np.float32)
        sets.append(a)
    return sets


def test_anchor_batching_accepts_reference_anchor_sets(ref):
    from graphmambaformer_b200.chaining import AnchorCSR
    from graphmambaformer_b200.types import AnchorSet

    sets = _reads(ref)
    got = AnchorCSR.from_sets(sets)
    ours = AnchorCSR.from_sets([AnchorSet.from_lists(a.read_pos, a.ref_pos, a.length, a.strand) for a in sets])
    for name in ("read_off", "read_pos", "ref_pos", "length", "strand"):
        assert np.array_equal(getattr(got, name), getattr(ours, name)), name


def test_parameter_blocks_from_reference_configs(ref):
    from graphmambaformer_b200.chaining import chain_params
    from graphmambaformer_b200.config import ChainingConfig, ExtensionConfig
    from graphmambaformer_b200.extension import params_from_config

    rc, re = ref["config"].ChainingConfig(max_lookback=50), ref["config"].ExtensionConfig()
    oc = ChainingConfig(**{f.name: getattr(rc, f.name) for f in fields(ChainingConfig) if hasattr(rc, f.name)})
    oe = ExtensionConfig(**{f.name: getattr(re, f.name) for f in fields(ExtensionConfig) if hasattr(re, f.name)})
    a, b = chain_params(rc), chain_params(oc)
    assert [getattr(a, n) for n, _ in a._fields_] == [getattr(b, n) for n, _ in b._fields_]
    a, b = params_from_config(re), params_from_config(oe)
    assert [getattr(a, n) for n, _ in a._fields_] == [getattr(b, n) for n, _ in b._fields_]


def test_extension_windows_of_reference_chains(ref):
    """Our ExtensionEngine._window on the reference's Chain and AnchorSet
    objects equals the reference's own _window."""
    from types import SimpleNamespace

    from graphmambaformer_b200.extension import ExtensionEngine

    cfg = ref["config"].ExtensionConfig()
    theirs = ref["extension"].ExtensionEngine(cfg, device="cpu", backend="torch")
    ours = SimpleNamespace(cfg=cfg)  # _window reads only the config (the engine itself wants a GPU)
    chainer = ref["chaining"].AffineChainer(ref["config"].ChainingConfig(max_lookback=50), backend="torch",
                                            workers=1)
    n = 0
    for a in _reads(ref, n=10, seed=9):
        a.score = np.full(len(a), np.nan, np.float32)
        for ch in chainer.chain(a, device="cpu"):
            got = ExtensionEngine._window(ours, ch, a, a.read_len, a.ref_len)
            assert got == theirs._window(ch, a, a.read_len, a.ref_len)
            n += 1
    assert n > 0


def test_hybrid_rows_with_reference_context_and_graph(ref):
    """Weights and bonus rows from the reference's ChainingContext holding
    the reference's GraphDistanceOracle equal the reference's own."""
    from graphmambaformer_b200.config import ChainingConfig
    from graphmambaformer_b200.hybrid import Segment, anchor_weights, bonus_rows

    ch = ref["chaining"]
    rng = np.random.default_rng(2)
    edges = np.array([[i, i + 1] for i in range(39)] + rng.integers(0, 40, size=(12, 2)).tolist()).T
    graph = ch.GraphDistanceOracle(edges, 40, max_hops=3)
    rcfg = ref["config"].ChainingConfig(max_lookback=24)
    ocfg = ChainingConfig(**{f.name: getattr(rcfg, f.name) for f in fields(ChainingConfig) if hasattr(rcfg, f.name)})
    chainer = ch.AffineChainer(rcfg, backend="torch", workers=1)
    checked = 0
    for k, a in enumerate(_reads(ref, n=8, seed=13)):
        for strand in (1, -1):
            sub, _ = a.for_strand(strand)
            sub, _ = sub.sorted_by_ref()
            if len(sub) == 0:
                continue
            keys = [(int(sub.read_pos[i]), int(sub.ref_pos[i]), int(sub.length[i]), int(sub.strand[i]))
                    for i in range(len(sub))]
            trans = {(keys[i], keys[i + 1]): float(rng.random()) for i in range(0, len(sub) - 1, 3)}
            ctx = ch.ChainingContext(oracle=graph, backbone=rng.random(40) < 0.5,
                                     trust_neural=[None, True][k % 2], learned_transitions=trans)
            seg = Segment.of(sub, np.arange(len(sub)))
            w_ref, b_ref = chainer._weights(sub, ctx), chainer._graph_bonus(sub, ctx)
            w, b = anchor_weights(ocfg, seg, ctx), bonus_rows(ocfg, seg, ctx)
            assert np.array_equal(w.view(np.int64), np.asarray(w_ref, np.float64).view(np.int64))
            assert (b is None) == (b_ref is None)
            if b is not None:
                assert np.array_equal(b.view(np.int64), b_ref.view(np.int64))
            checked += 1
    assert checked > 8
