"""B200-native (sm_100a) alignment hot path of GraphMambaFormer.

Stage 2 (anchor chaining) and Stage 3 (banded affine-gap Smith-Waterman with
CIGAR traceback) re-built as hand-written CUDA kernels behind a C ABI
(``include/gmf_align.h``), with Python stage objects that keep the
reference's call signatures:

* :class:`AffineChainer` -- ``chain`` / ``chain_batch`` (anchors in, chains out)
* :class:`ExtensionEngine` -- ``extend_chains`` (pairs in, score, ends, CIGAR out)
* primitives :func:`chain_dp`, :func:`banded_sw`, :func:`banded_affine_sw_batch`,
  :func:`traceback_banded`.

There is no CPU fallback: without the built library and a CUDA GPU the calls
raise.
"""

from .config import ChainingConfig, ExtensionConfig
from .types import AnchorSet, Chain, ExtensionResult, merge_cigar, run_length_encode

__all__ = [
    "ChainingConfig", "ExtensionConfig", "AnchorSet", "Chain", "ExtensionResult", "merge_cigar",
    "run_length_encode", "AffineChainer", "ExtensionEngine", "chain_dp", "chain_dp_rows",
    "banded_sw", "banded_affine_sw_batch", "traceback_banded",
]


def __getattr__(name):
    # stage objects import torch lazily so the package metadata stays cheap
    if name in ("AffineChainer", "chain_dp", "chain_dp_rows"):
        from . import chaining
        return getattr(chaining, name)
    if name in ("ExtensionEngine", "banded_sw", "banded_affine_sw_batch", "traceback_banded"):
        from . import extension
        return getattr(extension, name)
    raise AttributeError(name)
