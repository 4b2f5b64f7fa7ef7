"""C-ABI checks that need no GPU: the library loads, exports every function
the public header declares, and the ctypes structures match the C layout."""

from __future__ import annotations

import ctypes
import os
import re
import subprocess
import sys

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "gmf_align.h")


def declared_functions() -> list[str]:
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gmf_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    from graphmambaformer_b200 import _native

    lib = _native.lib()
    names = declared_functions()
    assert "gmf_banded_sw" in names and "gmf_chain_batch" in names
    for name in names:
        assert hasattr(lib, name), name
    # and the binding covers all of them with explicit signatures
    assert set(names) == set(_native.exported_symbols())


def test_status_strings_and_version():
    from graphmambaformer_b200 import _native

    assert _native.status_string(0) == "ok"
    assert "workspace" in _native.status_string(_native.GMF_ERR_WORKSPACE)
    assert _native.lib().gmf_version() >= 10000


def test_workspace_helpers_are_host_only():
    import numpy as np

    from graphmambaformer_b200 import _native

    q = np.array([150, 3000], np.int32)
    t = np.array([214, 3064], np.int32)
    hb = np.array([32, 100], np.int32)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    b = _native.lib().gmf_banded_sw_workspace_bytes(2, p(q), p(t), p(hb), 1)
    # traceback: one 4-bit code per pipeline step (>= one per DP cell), the
    # per-row maxima and the CIGAR-run scratch
    cells = sum(int(ql) * (2 * int(h) + 1) for ql, h in zip(q, hb))
    assert b >= 256 + cells // 2 + 4 * sum(2 * int(ql) + int(ql) + int(tl) + 1 for ql, tl in zip(q, t))
    no_tb = _native.lib().gmf_banded_sw_workspace_bytes(2, p(q), p(t), p(hb), 0)
    assert 256 + 8 * int(q.sum()) <= no_tb < b
    assert _native.lib().gmf_chain_workspace_bytes(10, 1000) > 1000 * 24


_LAYOUT_C = r"""
#include <stdio.h>
#include <stddef.h>
#include "gmf_align.h"
#define P(T) printf(#T " %zu\n", sizeof(T))
#define O(T, f) printf(#T "." #f " %zu\n", offsetof(T, f))
int main(void) {
  P(gmf_pairs); O(gmf_pairs, order); O(gmf_pairs, max_half_band); O(gmf_pairs, n_xdrop_groups);
  P(gmf_sw_params); P(gmf_sw_results); O(gmf_sw_results, cigar_capacity); O(gmf_sw_results, error_flags);
  P(gmf_chain_params); O(gmf_chain_params, min_chain_score);
  P(gmf_anchor_batch); O(gmf_anchor_batch, strand);
  P(gmf_sorted_anchors); P(gmf_chain_results); O(gmf_chain_results, members);
  P(gmf_wfa_pairs); O(gmf_wfa_pairs, query_total); O(gmf_wfa_pairs, max_len);
  P(gmf_wfa_results); O(gmf_wfa_results, cigar_capacity); O(gmf_wfa_results, error_flags);
  P(gmf_host_pairs); O(gmf_host_pairs, n_xdrop_groups);
  P(gmf_sam_records); O(gmf_sam_records, n_contigs); O(gmf_sam_records, tag_off);
  P(gmf_host_sw_results); O(gmf_host_sw_results, cigar_capacity); O(gmf_host_sw_results, error_flags);
  return 0;
}
"""


def test_ctypes_structs_match_c_layout(tmp_path):
    from graphmambaformer_b200 import _native as n

    src = tmp_path / "layout.c"
    exe = tmp_path / "layout"
    src.write_text(_LAYOUT_C)
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.rsplit(" ", 1) for line in subprocess.check_output([str(exe)]).decode().splitlines())
    want = {
        "gmf_pairs": ctypes.sizeof(n.GmfPairs),
        "gmf_pairs.order": n.GmfPairs.order.offset,
        "gmf_pairs.max_half_band": n.GmfPairs.max_half_band.offset,
        "gmf_pairs.n_xdrop_groups": n.GmfPairs.n_xdrop_groups.offset,
        "gmf_sw_params": ctypes.sizeof(n.GmfSwParams),
        "gmf_sw_results": ctypes.sizeof(n.GmfSwResults),
        "gmf_sw_results.cigar_capacity": n.GmfSwResults.cigar_capacity.offset,
        "gmf_sw_results.error_flags": n.GmfSwResults.error_flags.offset,
        "gmf_chain_params": ctypes.sizeof(n.GmfChainParams),
        "gmf_chain_params.min_chain_score": n.GmfChainParams.min_chain_score.offset,
        "gmf_anchor_batch": ctypes.sizeof(n.GmfAnchorBatch),
        "gmf_anchor_batch.strand": n.GmfAnchorBatch.strand.offset,
        "gmf_sorted_anchors": ctypes.sizeof(n.GmfSortedAnchors),
        "gmf_chain_results": ctypes.sizeof(n.GmfChainResults),
        "gmf_chain_results.members": n.GmfChainResults.members.offset,
        "gmf_wfa_pairs": ctypes.sizeof(n.GmfWfaPairs),
        "gmf_wfa_pairs.query_total": n.GmfWfaPairs.query_total.offset,
        "gmf_wfa_pairs.max_len": n.GmfWfaPairs.max_len.offset,
        "gmf_wfa_results": ctypes.sizeof(n.GmfWfaResults),
        "gmf_wfa_results.cigar_capacity": n.GmfWfaResults.cigar_capacity.offset,
        "gmf_wfa_results.error_flags": n.GmfWfaResults.error_flags.offset,
        "gmf_sam_records": ctypes.sizeof(n.GmfSamRecords),
        "gmf_sam_records.n_contigs": n.GmfSamRecords.n_contigs.offset,
        "gmf_sam_records.tag_off": n.GmfSamRecords.tag_off.offset,
        "gmf_host_pairs": ctypes.sizeof(n.GmfHostPairs),
        "gmf_host_pairs.n_xdrop_groups": n.GmfHostPairs.n_xdrop_groups.offset,
        "gmf_host_sw_results": ctypes.sizeof(n.GmfHostSwResults),
        "gmf_host_sw_results.cigar_capacity": n.GmfHostSwResults.cigar_capacity.offset,
        "gmf_host_sw_results.error_flags": n.GmfHostSwResults.error_flags.offset,
    }
    for k, v in want.items():
        assert int(got[k]) == v, (k, got[k], v)


def test_stages_refuse_to_run_without_a_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from graphmambaformer_b200.chaining import AffineChainer
    from graphmambaformer_b200.types import AnchorSet

    a = AnchorSet.from_lists([0, 20], [0, 20], [15, 15], [1, 1])
    with pytest.raises(RuntimeError, match="CUDA"):
        AffineChainer().chain(a)


def test_entry_points_reject_malformed_arguments_before_any_cuda_call():
    """Argument checks run on the host first, so these return the documented
    status without a GPU."""
    from graphmambaformer_b200 import _native
    from graphmambaformer_b200.autotune import SwTuning

    lib = _native.lib()
    bad_idx = _native.GmfMinimizerIndex(0, 10, 0, None, None, None)  # k = 0
    assert lib.gmf_seed_count(ctypes.byref(bad_idx), 1, None, None, 1, None, None) == _native.GMF_ERR_INVALID_ARGUMENT
    big_w = _native.GmfMinimizerIndex(15, 300, 0, None, None, None)
    assert lib.gmf_seed_fill(ctypes.byref(big_w), 1, None, None, 1, None, None, None, None, None, None) \
        == _native.GMF_ERR_INVALID_ARGUMENT
    assert lib.gmf_gather_segments(None, 0, -1, None, None, None, None, None, None) == _native.GMF_ERR_INVALID_ARGUMENT
    assert lib.gmf_gather_segments(None, 10, 3, None, None, None, None, None, None) == _native.GMF_ERR_INVALID_ARGUMENT
    assert lib.gmf_sw_set_tuning(ctypes.byref(SwTuning(130, 125).to_c())) == _native.GMF_ERR_INVALID_ARGUMENT
    assert lib.gmf_sw_set_tuning(None) == _native.GMF_ERR_INVALID_ARGUMENT
    batch = _native.GmfAnchorBatch(1, None, None, None, None, None)
    cp = _native.GmfChainParams(64, 5000, 1, 8, 20.0, 0.5, 0.6)
    res = _native.GmfChainResults(None, None, None, None, None, None, None)
    assert lib.gmf_chain_batch_noalloc(ctypes.byref(batch), ctypes.byref(cp), None, 0, 10 ** 9, ctypes.byref(res),
                                       None) == _native.GMF_ERR_LIMIT
    assert lib.gmf_banded_sw(None, None, None, None, 0, None) == _native.GMF_ERR_INVALID_ARGUMENT
    assert lib.gmf_chain_dp(-1, None, None, None, None, None, 64, 5000, None, 0, None, None, None) \
        == _native.GMF_ERR_INVALID_ARGUMENT
    # WFA: bounds and malformed pairs, all refused on the host
    bad_pairs = _native.GmfWfaPairs(2, None, None, None, None, None, 10, 10, 5)
    assert lib.gmf_wfa_distance(ctypes.byref(bad_pairs), 8, None, None, 0, None) == _native.GMF_ERR_INVALID_ARGUMENT
    empty = _native.GmfWfaPairs(0, None, None, None, None, None, 0, 0, 0)
    assert lib.gmf_wfa_distance(ctypes.byref(empty), _native.MAX_WFA_DISTANCE + 1, None, None, 0, None) \
        == _native.GMF_ERR_LIMIT
    assert lib.gmf_wfa_align(ctypes.byref(empty), None, -1, None, None, 0, None) == _native.GMF_ERR_LIMIT
    assert lib.gmf_wfa_distance(None, 8, None, None, 0, None) == _native.GMF_ERR_INVALID_ARGUMENT
    import numpy as np

    ql = np.array([10, 0, 5], np.int32)
    tl = np.array([12, 7, 5], np.int32)
    dist = np.array([3, 7, -1], np.int32)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    assert lib.gmf_wfa_history_entries(3, p(ql), p(tl), p(dist)) == 16
    assert lib.gmf_wfa_workspace_bytes(3, 12, 8, 16) >= lib.gmf_wfa_workspace_bytes(3, 12, 8, 0) + 64
    # contexts: malformed calls are refused before any CUDA call
    assert lib.gmf_ctx_create(0, 3, 0, None) == _native.GMF_ERR_INVALID_ARGUMENT
    h = ctypes.c_void_p()
    assert lib.gmf_ctx_create(0, 0, 0, ctypes.byref(h)) == _native.GMF_ERR_INVALID_ARGUMENT
    assert lib.gmf_ctx_create(0, 9, 0, ctypes.byref(h)) == _native.GMF_ERR_INVALID_ARGUMENT
    assert lib.gmf_ctx_destroy(None) == _native.GMF_ERR_INVALID_ARGUMENT
    assert lib.gmf_batch_submit(None, None, None, None, None) == _native.GMF_ERR_INVALID_ARGUMENT
    assert lib.gmf_batch_poll(None, 1) == _native.GMF_ERR_INVALID_ARGUMENT
    assert lib.gmf_batch_wait(None, 1) == _native.GMF_ERR_INVALID_ARGUMENT
    # SAM records: malformed batches refused on the host
    assert lib.gmf_sam_count(None, None, None) == _native.GMF_ERR_INVALID_ARGUMENT
    bad = _native.GmfSamRecords(3)  # no arrays
    assert lib.gmf_sam_count(ctypes.byref(bad), None, None) == _native.GMF_ERR_INVALID_ARGUMENT
    assert lib.gmf_sam_fill(ctypes.byref(bad), None, None, None) == _native.GMF_ERR_INVALID_ARGUMENT
