"""ctypes binding of the C ABI in ``include/gmf_align.h``.

The structures below mirror the header field for field.  Loading fails
loudly when the CUDA library has not been built: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, Structure, c_char_p, c_double, c_int, c_int32, c_int64, c_size_t, c_void_p

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libgmf_align.so")

GMF_OK = 0
GMF_ERR_INVALID_ARGUMENT = 1
GMF_ERR_CUDA = 2
GMF_ERR_WORKSPACE = 3
GMF_ERR_CAPACITY = 4
GMF_ERR_LIMIT = 5
GMF_ERR_TIMEOUT = 6
GMF_ERR_NOT_READY = 7
GMF_ERR_HOST = 8

GMF_SWF_WORKSPACE = 1
GMF_SWF_CAPACITY = 2
GMF_SWF_TIMEOUT = 4
GMF_SWF_INTERNAL = 8

MAX_HALF_BAND = 4096
MAX_READ_ANCHORS = 16384
MAX_LOOKBACK = 1024
CHAIN_NOALLOC_SCRATCH_BYTES = 32 << 20


class GmfPairs(Structure):
    _fields_ = [
        ("n_pairs", c_int32),
        ("query", c_void_p),
        ("query_off", c_void_p),
        ("target", c_void_p),
        ("target_off", c_void_p),
        ("half_band", c_void_p),
        ("band_offset", c_void_p),
        ("order", c_void_p),
        ("max_half_band", c_int32),
        ("xdrop_group_off", c_void_p),
        ("n_xdrop_groups", c_int32),
    ]


class GmfSwParams(Structure):
    _fields_ = [
        ("match_score", c_int32),
        ("mismatch_penalty", c_int32),
        ("gap_open", c_int32),
        ("gap_extend", c_int32),
        ("x_drop", c_int32),
    ]


class GmfSwResults(Structure):
    _fields_ = [
        ("score", c_void_p),
        ("query_end", c_void_p),
        ("target_end", c_void_p),
        ("query_start", c_void_p),
        ("target_start", c_void_p),
        ("op_counts", c_void_p),
        ("cigar", c_void_p),
        ("cigar_capacity", c_int64),
        ("cigar_start", c_void_p),
        ("cigar_len", c_void_p),
        ("cigar_used", c_void_p),
        ("error_flags", c_void_p),
    ]


class GmfSwTuning(Structure):
    _fields_ = [
        ("l8_max_w", c_int32),
        ("l16_max_w", c_int32),
        ("coop_min_strips", c_int32 * 3),
        ("warps_per_block", c_int32),
        ("side_streams", c_int32),
    ]


class GmfMinimizerIndex(Structure):
    _fields_ = [
        ("k", c_int32),
        ("w", c_int32),
        ("n_keys", c_int64),
        ("keys", c_void_p),
        ("offsets", c_void_p),
        ("positions", c_void_p),
    ]


class GmfChainParams(Structure):
    _fields_ = [
        ("max_lookback", c_int32),
        ("max_gap", c_int32),
        ("min_chain_anchors", c_int32),
        ("max_chains", c_int32),
        ("min_chain_score", c_double),
        ("secondary_overlap", c_double),
        ("secondary_score_ratio", c_double),
    ]


class GmfAnchorBatch(Structure):
    _fields_ = [
        ("n_reads", c_int32),
        ("read_off", c_void_p),
        ("read_pos", c_void_p),
        ("ref_pos", c_void_p),
        ("length", c_void_p),
        ("strand", c_void_p),
    ]


class GmfSortedAnchors(Structure):
    _fields_ = [
        ("perm", c_void_p),
        ("n_plus", c_void_p),
        ("n_minus", c_void_p),
        ("read_end", c_void_p),
        ("ref_end", c_void_p),
    ]


class GmfChainResults(Structure):
    _fields_ = [
        ("n_chains", c_void_p),
        ("score", c_void_p),
        ("strand", c_void_p),
        ("span", c_void_p),
        ("is_primary", c_void_p),
        ("n_members", c_void_p),
        ("members", c_void_p),
    ]


class GmfWfaPairs(Structure):
    _fields_ = [
        ("n_pairs", c_int32),
        ("query", c_void_p),
        ("query_off", c_void_p),
        ("target", c_void_p),
        ("target_off", c_void_p),
        ("order", c_void_p),
        ("query_total", c_int64),
        ("target_total", c_int64),
        ("max_len", c_int32),
    ]


class GmfWfaResults(Structure):
    _fields_ = [
        ("op_counts", c_void_p),
        ("cigar", c_void_p),
        ("cigar_capacity", c_int64),
        ("cigar_start", c_void_p),
        ("cigar_len", c_void_p),
        ("cigar_used", c_void_p),
        ("error_flags", c_void_p),
    ]


class GmfHostPairs(Structure):
    _fields_ = [
        ("n_pairs", c_int32),
        ("query", c_void_p),
        ("query_off", c_void_p),
        ("target", c_void_p),
        ("target_off", c_void_p),
        ("half_band", c_void_p),
        ("band_offset", c_void_p),
        ("xdrop_group_off", c_void_p),
        ("n_xdrop_groups", c_int32),
    ]


class GmfHostSwResults(Structure):
    _fields_ = [
        ("score", c_void_p),
        ("query_end", c_void_p),
        ("target_end", c_void_p),
        ("query_start", c_void_p),
        ("target_start", c_void_p),
        ("op_counts", c_void_p),
        ("cigar", c_void_p),
        ("cigar_capacity", c_int64),
        ("cigar_start", c_void_p),
        ("cigar_len", c_void_p),
        ("cigar_used", c_void_p),
        ("error_flags", c_void_p),
    ]


class GmfSamRecords(Structure):
    _fields_ = [
        ("n_records", c_int32),
        ("name", c_void_p),
        ("name_off", c_void_p),
        ("seq", c_void_p),
        ("seq_off", c_void_p),
        ("qual", c_void_p),
        ("contig", c_void_p),
        ("contig_names", c_void_p),
        ("contig_off", c_void_p),
        ("n_contigs", c_int32),
        ("ref_start", c_void_p),
        ("ref_end", c_void_p),
        ("strand", c_void_p),
        ("mapq", c_void_p),
        ("cigar", c_void_p),
        ("cigar_start", c_void_p),
        ("cigar_len", c_void_p),
        ("clip_left", c_void_p),
        ("clip_right", c_void_p),
        ("tags", c_void_p),
        ("tag_off", c_void_p),
        ("max_seq_len", c_int64),
    ]


MAX_WFA_DISTANCE = 1 << 16

# name -> (restype, argtypes)
_SIGNATURES = {
    "gmf_status_string": (c_char_p, [c_int]),
    "gmf_version": (c_int, []),
    "gmf_set_device": (c_int, [c_int]),
    "gmf_banded_sw_workspace_bytes": (c_size_t, [c_int32, c_void_p, c_void_p, c_void_p, c_int32]),
    "gmf_banded_sw": (c_int, [POINTER(GmfPairs), POINTER(GmfSwParams), POINTER(GmfSwResults),
                              c_void_p, c_size_t, c_void_p]),
    "gmf_banded_sw_plain": (c_int, [POINTER(GmfPairs), POINTER(GmfSwParams), POINTER(GmfSwResults),
                                    c_void_p, c_size_t, c_void_p]),
    "gmf_gather_segments": (c_int, [c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_void_p, c_void_p]),
    "gmf_chain_spread": (c_int, [POINTER(GmfAnchorBatch), POINTER(GmfChainResults), c_int32, c_void_p, c_void_p]),
    "gmf_seed_count": (c_int, [POINTER(GmfMinimizerIndex), c_int32, c_void_p, c_void_p, c_int32, c_void_p,
                               c_void_p]),
    "gmf_seed_fill": (c_int, [POINTER(GmfMinimizerIndex), c_int32, c_void_p, c_void_p, c_int32, c_void_p,
                              c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "gmf_sw_get_tuning": (c_int, [POINTER(GmfSwTuning)]),
    "gmf_sw_set_tuning": (c_int, [POINTER(GmfSwTuning)]),
    "gmf_sw_test_coop_wait": (c_int, [c_int32, c_int32]),
    "gmf_chain_dp": (c_int, [c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32,
                             c_int32, c_void_p, c_int32, c_void_p, c_void_p, c_void_p]),
    "gmf_chain_sort": (c_int, [POINTER(GmfAnchorBatch), POINTER(GmfSortedAnchors), c_void_p,
                               c_size_t, c_void_p]),
    "gmf_chain_workspace_bytes": (c_size_t, [c_int32, c_int64]),
    "gmf_chain_batch": (c_int, [POINTER(GmfAnchorBatch), POINTER(GmfChainParams), c_void_p,
                                c_int32, POINTER(GmfSortedAnchors), c_void_p, c_void_p,
                                POINTER(GmfChainResults), c_void_p, c_size_t, c_void_p]),
    "gmf_chain_batch_noalloc": (c_int, [POINTER(GmfAnchorBatch), POINTER(GmfChainParams), c_void_p,
                                        c_int32, c_int64, POINTER(GmfChainResults), c_void_p]),
    "gmf_chain_noalloc_error_flags": (c_int, [c_void_p, c_void_p]),
    "gmf_ctx_create": (c_int, [c_int, c_int32, c_size_t, POINTER(c_void_p)]),
    "gmf_ctx_destroy": (c_int, [c_void_p]),
    "gmf_batch_submit": (c_int, [c_void_p, POINTER(GmfHostPairs), POINTER(GmfSwParams), POINTER(GmfHostSwResults),
                                 POINTER(c_int64)]),
    "gmf_batch_poll": (c_int, [c_void_p, c_int64]),
    "gmf_batch_wait": (c_int, [c_void_p, c_int64]),
    "gmf_sam_count": (c_int, [POINTER(GmfSamRecords), c_void_p, c_void_p]),
    "gmf_sam_fill": (c_int, [POINTER(GmfSamRecords), c_void_p, c_void_p, c_void_p]),
    "gmf_wfa_workspace_bytes": (c_size_t, [c_int32, c_int32, c_int32, c_int64]),
    "gmf_wfa_history_entries": (c_int64, [c_int32, c_void_p, c_void_p, c_void_p]),
    "gmf_wfa_distance": (c_int, [POINTER(GmfWfaPairs), c_int32, c_void_p, c_void_p, c_size_t, c_void_p]),
    "gmf_wfa_align": (c_int, [POINTER(GmfWfaPairs), c_void_p, c_int32, POINTER(GmfWfaResults), c_void_p,
                              c_size_t, c_void_p]),
}

_lib = None


class GmfError(RuntimeError):
    """A gmf_* entry point returned a non-zero status."""

    def __init__(self, fn: str, status: int):
        self.status = status
        super().__init__(f"{fn} failed: {status_string(status)} (status {status})")


def exported_symbols() -> list[str]:
    return sorted(_SIGNATURES)


def lib() -> ctypes.CDLL:
    """The loaded library; raises if it was never built (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"gmf CUDA library missing at {LIB_PATH}; build it with "
                "`python -m graphmambaformer_b200.build` (there is no CPU fallback)")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def status_string(status: int) -> str:
    return lib().gmf_status_string(status).decode()


def check(fn: str, status: int) -> None:
    if status != GMF_OK:
        raise GmfError(fn, status)
