"""B200-native (sm_100a) alignment hot path of GraphMambaFormer.

Stage 2 (anchor chaining) and Stage 3 (banded affine-gap Smith-Waterman with
CIGAR traceback) re-built as hand-written CUDA kernels behind a C ABI
(``include/gmf_align.h``), with Python stage objects that keep the
reference's call signatures:

* :class:`AffineChainer` -- ``chain`` / ``chain_batch`` (anchors in, chains out)
* :class:`ExtensionEngine` -- ``extend_chains`` (pairs in, score, ends, CIGAR out)
* primitives :func:`chain_dp`, :func:`banded_sw`, :func:`banded_affine_sw_batch`,
  :func:`traceback_banded`;
* the ``algorithm="wfa"`` variant: :class:`WavefrontAligner`, :func:`wfa_distance`;
* device minimizer seeding (:class:`DeviceMinimizerIndex`), record assembly
  and SAM text (:mod:`.records`), the serving loop (:class:`AlignServer`) and
  the C ABI's asynchronous host-buffer contexts (:class:`AlignContext`).

There is no CPU fallback: without the built library and a CUDA GPU the calls
raise.
"""

from .config import ChainingConfig, ExtensionConfig
from .types import AnchorSet, Chain, ExtensionResult, merge_cigar, run_length_encode

__all__ = [
    "ChainingConfig", "ExtensionConfig", "AnchorSet", "Chain", "ExtensionResult", "merge_cigar",
    "run_length_encode", "AffineChainer", "ExtensionEngine", "chain_dp", "chain_dp_rows",
    "banded_sw", "banded_affine_sw_batch", "traceback_banded", "WavefrontAligner", "wfa_distance",
    "DeviceMinimizerIndex", "AlignServer", "AlignContext", "write_sam",
]

_LAZY = {
    "AffineChainer": "chaining", "chain_dp": "chaining", "chain_dp_rows": "chaining",
    "ExtensionEngine": "extension", "banded_sw": "extension", "banded_affine_sw_batch": "extension",
    "traceback_banded": "extension", "WavefrontAligner": "wfa", "wfa_distance": "wfa",
    "DeviceMinimizerIndex": "seeding", "AlignServer": "serving", "AlignContext": "context",
    "write_sam": "records",
}


def __getattr__(name):
    # stage objects import torch lazily so the package metadata stays cheap
    if name in _LAZY:
        import importlib

        return getattr(importlib.import_module(f".{_LAZY[name]}", __name__), name)
    raise AttributeError(name)
