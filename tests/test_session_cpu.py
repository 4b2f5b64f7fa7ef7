"""Host logic of the chain session: the runs a large host batch goes
through partition its reads in order, none empty, with about A / C anchors
each (a run can exceed that by at most one read)."""

from __future__ import annotations

import numpy as np
import pytest


@pytest.mark.parametrize("chunks", [None, 1, 2, 3, 4, 7, 1000])
def test_run_cuts_partition_the_reads(chunks):
    from graphmambaformer_b200.session import run_cuts

    rng = np.random.default_rng(0 if chunks is None else chunks)
    cases = [np.array([0]), np.array([0, 0]), np.array([0, 5]), np.array([0, 0, 0, 7, 7, 9])]
    for _ in range(50):
        counts = rng.integers(0, 3000, int(rng.integers(1, 400)))
        counts[rng.random(len(counts)) < 0.1] = 0
        cases.append(np.concatenate([[0], np.cumsum(counts)]))
    cases.append(np.concatenate([[0], np.cumsum(np.full(5000, 2722))]))  # the HiFi bench batch
    for off in cases:
        R, A = len(off) - 1, int(off[-1])
        cut = run_cuts(off, chunks)
        if R == 0:
            assert cut.tolist() == [0, 0]
            continue
        assert cut[0] == 0 and cut[-1] == R and np.all(np.diff(cut) > 0)
        C = len(cut) - 1
        want = chunks if chunks is not None else min(2, max(1, A // 2_000_000))
        assert C <= max(1, min(want, R))
        per_run = np.diff(off[cut])
        assert per_run.max() <= A / C + np.diff(off).max()
    assert len(run_cuts(cases[-1], None)) - 1 == 2
