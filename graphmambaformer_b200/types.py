"""Stage data contract: anchors in, chains out; pairs in, alignments out.

The classes keep the reference's field names and meaning
(graphmambaformer/alignment/types.py L26-432) so objects flow unchanged
between the reference pipeline and these stages; the engines only read the
attributes they need, so the reference's own ``AnchorSet`` / ``Chain``
instances are accepted as well.

Coordinates are 0-based, half-open, on the forward reference.  A reverse-
strand anchor stores its read position in reverse-complemented read
orientation and carries ``strand == -1``.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

CIGAR_OPS: tuple[str, ...] = ("=", "X", "I", "D", "S", "H", "M", "N")
#: op code of the packed CIGAR words returned by the CUDA library
WORD_OPS = "=XIDS"


@dataclass
class AnchorSet:
    """Columnar seed anchors of one read (types.py L26-206)."""

    read_pos: np.ndarray
    ref_pos: np.ndarray
    length: np.ndarray
    strand: np.ndarray
    node_id: np.ndarray
    source: np.ndarray
    score: np.ndarray
    read_len: int = 0
    ref_len: int = 0

    def __post_init__(self) -> None:
        n = len(self.read_pos)
        for name in ("ref_pos", "length", "strand", "node_id", "source", "score"):
            if len(getattr(self, name)) != n:
                raise ValueError(f"AnchorSet field {name!r} has inconsistent length")

    def __len__(self) -> int:
        return len(self.read_pos)

    @property
    def diagonal(self) -> np.ndarray:
        return self.ref_pos.astype(np.int64) - self.read_pos.astype(np.int64)

    @property
    def read_end(self) -> np.ndarray:
        return self.read_pos + self.length

    @property
    def ref_end(self) -> np.ndarray:
        return self.ref_pos + self.length

    @classmethod
    def empty(cls, read_len: int = 0, ref_len: int = 0) -> "AnchorSet":
        z = np.zeros(0, dtype=np.int64)
        return cls(z.copy(), z.copy(), z.copy(), np.zeros(0, np.int8), z.copy(),
                   np.zeros(0, np.int8), np.zeros(0, np.float32), read_len, ref_len)

    @classmethod
    def from_lists(cls, read_pos, ref_pos, length, strand, node_id=None, source=None,
                   read_len: int = 0, ref_len: int = 0) -> "AnchorSet":
        n = len(read_pos)
        return cls(
            np.asarray(read_pos, dtype=np.int64),
            np.asarray(ref_pos, dtype=np.int64),
            np.asarray(length, dtype=np.int64),
            np.asarray(strand, dtype=np.int8),
            np.asarray(node_id, dtype=np.int64) if node_id is not None else np.full(n, -1, np.int64),
            np.asarray(source, dtype=np.int8) if source is not None else np.zeros(n, np.int8),
            np.full(n, np.nan, dtype=np.float32),
            read_len,
            ref_len,
        )

    def take(self, idx) -> "AnchorSet":
        idx = np.asarray(idx, dtype=np.int64)
        return AnchorSet(self.read_pos[idx], self.ref_pos[idx], self.length[idx], self.strand[idx],
                         self.node_id[idx], self.source[idx], self.score[idx], self.read_len,
                         self.ref_len)

    def for_strand(self, strand: int) -> tuple["AnchorSet", np.ndarray]:
        idx = np.flatnonzero(self.strand == strand)
        return self.take(idx), idx

    def sorted_by_ref(self) -> tuple["AnchorSet", np.ndarray]:
        order = np.lexsort((self.read_end, self.ref_end))
        return self.take(order), order

    def concat(self, other: "AnchorSet") -> "AnchorSet":
        if len(other) == 0:
            return self
        if len(self) == 0:
            return other
        cat = np.concatenate
        return AnchorSet(cat([self.read_pos, other.read_pos]), cat([self.ref_pos, other.ref_pos]),
                         cat([self.length, other.length]), cat([self.strand, other.strand]),
                         cat([self.node_id, other.node_id]), cat([self.source, other.source]),
                         cat([self.score, other.score]), self.read_len or other.read_len,
                         self.ref_len or other.ref_len)


@dataclass
class Chain:
    """A collinear run of anchors (types.py L225-284)."""

    anchor_idx: np.ndarray
    score: float
    strand: int
    read_start: int
    read_end: int
    ref_start: int
    ref_end: int
    neural_score: float = float("nan")
    is_primary: bool = False

    def __len__(self) -> int:
        return len(self.anchor_idx)

    @property
    def read_span(self) -> int:
        return self.read_end - self.read_start

    @property
    def ref_span(self) -> int:
        return self.ref_end - self.ref_start

    def coverage(self, read_len: int) -> float:
        return self.read_span / max(read_len, 1)


@dataclass
class ExtensionResult:
    """Base-level alignment of one chain (types.py L287-322)."""

    score: float
    cigar: list
    read_start: int
    read_end: int
    ref_start: int
    ref_end: int
    n_match: int = 0
    n_mismatch: int = 0
    n_insertion: int = 0
    n_deletion: int = 0

    @property
    def cigar_string(self) -> str:
        return "".join(f"{n}{op}" for op, n in self.cigar)

    @property
    def identity(self) -> float:
        total = self.n_match + self.n_mismatch + self.n_insertion + self.n_deletion
        return self.n_match / total if total else 0.0

    @property
    def edit_distance(self) -> int:
        return self.n_mismatch + self.n_insertion + self.n_deletion


def run_length_encode(ops: Sequence[str]) -> list:
    if not ops:
        return []
    out = []
    cur, n = ops[0], 1
    for op in ops[1:]:
        if op == cur:
            n += 1
        else:
            out.append((cur, n))
            cur, n = op, 1
    out.append((cur, n))
    return out


def merge_cigar(cigar: Sequence) -> list:
    """Merge adjacent runs of one op and drop empty runs (types.py L422-432)."""
    out: list = []
    for op, n in cigar:
        if n <= 0:
            continue
        if out and out[-1][0] == op:
            out[-1] = (op, out[-1][1] + n)
        else:
            out.append((op, n))
    return out


def cigar_read_length(cigar: Sequence) -> int:
    return sum(n for op, n in cigar if op in ("=", "X", "M", "I", "S"))


def cigar_ref_length(cigar: Sequence) -> int:
    return sum(n for op, n in cigar if op in ("=", "X", "M", "D", "N"))


_OP_LETTERS = np.array(list(WORD_OPS) + ["?"] * (16 - len(WORD_OPS)))


def decode_words(words: np.ndarray) -> tuple:
    """Packed ``(run << 4) | op`` words -> (op letters, run lengths) as two
    Python lists, decoded in one vectorized pass."""
    w = np.asarray(words, dtype=np.uint32)
    return _OP_LETTERS[w & 15].tolist(), (w >> 4).astype(np.int64).tolist()


def words_to_cigar(words: np.ndarray) -> list:
    """Packed ``(run << 4) | op`` words -> ``[(op, run), ...]``."""
    ops, runs = decode_words(words)
    return list(zip(ops, runs))


def add_soft_clips(cigar: list, left: int, right: int) -> list:
    """``merge_cigar([("S", left)] + cigar + [("S", right)])``.  A CIGAR of
    merged runs that neither starts nor ends with S (what the device walk
    writes) only gains the clips; anything else goes through merge_cigar."""
    if cigar and cigar[0][0] != "S" and cigar[-1][0] != "S":
        out = [("S", left)] if left > 0 else []
        out.extend(cigar)
        if right > 0:
            out.append(("S", right))
        return out
    return merge_cigar([("S", left)] + list(cigar) + [("S", right)])
