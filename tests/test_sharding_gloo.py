"""Sharding of the alignment path across ranks, on CPU with gloo: two ranks
take disjoint longest-processing-time shares that cover every pair / read,
loads stay within the LPT bound, and the timing reduction returns the max
over ranks."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    import torch.distributed as dist

    from graphmambaformer_b200 import sharding, synth

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        ps = synth.extension_pairs_mixed(n_pairs=300, seed=3, ref_len=500_000, max_len=3000)
        sub, idx = sharding.shard_pairs(ps, rank, world)
        reads = synth.chaining_reads_hifi(n_reads=40, seed=2, ref_len=300_000, mean_len=3000)
        ridx = sharding.shard_reads(reads, rank, world)
        mx = sharding.max_over_ranks(float(rank + 1) * 1.5)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), idx=idx, ridx=ridx, mx=mx,
                 cells=sharding.pair_costs(sub).sum(), n=len(sub))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_without_overlap(tmp_path):
    import torch.multiprocessing as mp

    from graphmambaformer_b200 import sharding, synth

    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    ps = synth.extension_pairs_mixed(n_pairs=300, seed=3, ref_len=500_000, max_len=3000)
    costs = sharding.pair_costs(ps)
    allidx = np.concatenate([r["idx"] for r in res])
    assert sorted(allidx.tolist()) == list(range(len(ps)))  # disjoint and complete
    loads = [costs[r["idx"]].sum() for r in res]
    assert max(loads) <= costs.sum() / world + costs.max()
    assert all(abs(float(r["cells"]) - l) < 1e-6 for r, l in zip(res, loads))
    rall = np.concatenate([r["ridx"] for r in res])
    assert sorted(rall.tolist()) == list(range(40))
    assert all(float(r["mx"]) == 3.0 for r in res)  # max over ranks of 1.5, 3.0


def test_lpt_partition_bound_and_determinism():
    from graphmambaformer_b200 import sharding

    rng = np.random.default_rng(0)
    c = rng.lognormal(7, 1.2, size=1000)
    for w in (1, 2, 3, 8):
        parts = sharding.lpt_partition(c, w)
        assert sorted(np.concatenate(parts).tolist()) == list(range(len(c)))
        assert max(c[p].sum() for p in parts) <= c.sum() / w + c.max()
        again = sharding.lpt_partition(c, w)
        assert all(np.array_equal(a, b) for a, b in zip(parts, again))
    with pytest.raises(ValueError):
        sharding.lpt_partition(c, 0)
