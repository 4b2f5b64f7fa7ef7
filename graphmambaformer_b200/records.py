"""Record assembly and SAM output: the step after extension.

Drop-in for the reference's:

* ``AlignmentPipeline._records`` / ``_margin_mapq`` (``alignment/pipeline.py``
  L365-426) and the fast pipeline's record list per read (L486-511):
  :func:`margin_mapq`, :func:`assemble_records`, :func:`read_alignments`;
* ``AlignmentRecord`` / ``ReadAlignments`` (``alignment/types.py`` L325-390);
* ``alignments_to_records`` + ``write_alignments`` for ``.sam``
  (``data/alignment_io.py`` L55-188; ``data/formats.py`` L304-500):
  :func:`sam_records` and :func:`write_sam`.

Record assembly is a few fields per chain and stays on the host.  The SAM
text -- reverse complements, quality strings, CIGAR strings, numbers -- is
byte work proportional to the bases written, and is rendered by the gmf CUDA
library (``gmf_sam_count`` / ``gmf_sam_fill``) from device-resident records;
the host only writes the header and the bytes.  Records are single-end (the
reference's paired-end mate fields are not carried).

Records can also stay arrays from end to end: :func:`record_table` builds a
batch's records from the serving pipeline's chain and extension columns,
:func:`sam_batch` lays a :class:`RecordTable` and read columns out for the
kernels, and :func:`render_sam_array` returns the text in page-locked host
memory.  That path does no per-record Python work and gives the same layout
as the object path.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np
import torch

from . import _native
from .device import bind, require_cuda, stream_handle, to_device
from .types import AnchorSet, Chain, ExtensionResult

MAX_PHRED = 93

# SAM @RG PL codes per modality (formats.py L291-303)
MODALITY_PLATFORM = {
    "illumina": "ILLUMINA", "pacbio_hifi": "PACBIO", "ont": "ONT", "rna_seq": "ILLUMINA",
    "bisulfite": "ILLUMINA", "single_cell": "ILLUMINA", "linked_reads": "ILLUMINA",
}
MODALITIES = tuple(MODALITY_PLATFORM)
# accepted spellings (formats.py L70-80)
MODALITY_ALIASES = {
    "nanopore": "ont", "ont_r9": "ont", "ont_r10": "ont", "oxford_nanopore": "ont",
    "hifi": "pacbio_hifi", "pacbio": "pacbio_hifi", "pb": "pacbio_hifi", "ccs": "pacbio_hifi",
    "revio": "pacbio_hifi", "ngs": "illumina", "short_read": "illumina", "dnbseq": "illumina",
    "mgi": "illumina", "ultima": "illumina", "ion_torrent": "illumina", "rna": "rna_seq", "rnaseq": "rna_seq",
    "methylation": "bisulfite", "wgbs": "bisulfite", "sc": "single_cell", "scrna": "single_cell",
    "10x": "linked_reads", "chromium": "linked_reads",
}

OPS = "=XIDSMNH"  # CIGAR word op codes of the library


def validate_modality(modality: str) -> str:
    """Canonical modality name (formats.py L83-100)."""
    key = str(modality).strip().lower().replace("-", "_")
    if key in MODALITY_PLATFORM:
        return key
    if key in MODALITY_ALIASES:
        return MODALITY_ALIASES[key]
    raise ValueError(f"unknown modality {modality!r}. Valid: {sorted(MODALITIES)}. "
                     f"Aliases: {sorted(MODALITY_ALIASES)}")


@dataclass
class AlignmentRecord:
    """One alignment of one read, ready to become a SAM row (types.py L325-362)."""

    read_id: str
    read_len: int
    ref_id: int = -1
    ref_start: int = -1
    ref_end: int = -1
    strand: int = 1
    mapq: int = 0
    chain_score: float = 0.0
    alignment_score: float = 0.0
    cigar: list = field(default_factory=list)
    node_id: int = -1
    is_mapped: bool = False
    is_primary: bool = True
    is_supplementary: bool = False
    route: str = "full"
    pass_name: str = "hybrid"
    n_anchors: int = 0
    n_chains: int = 0
    stages: tuple = ()
    extension: Optional[ExtensionResult] = None

    @property
    def cigar_string(self) -> str:
        return "".join(f"{n}{op}" for op, n in self.cigar)

    @classmethod
    def unmapped(cls, read_id: str, read_len: int, **kwargs) -> "AlignmentRecord":
        return cls(read_id=read_id, read_len=read_len, is_mapped=False, **kwargs)


@dataclass
class ReadAlignments:
    """Every candidate of one read, the primary called out (types.py L365-390)."""

    read_id: str
    read_len: int
    anchors: Optional[AnchorSet] = None
    chains: list = field(default_factory=list)
    records: list = field(default_factory=list)

    def __iter__(self):
        return iter(self.records)

    @property
    def primary(self) -> Optional[AlignmentRecord]:
        for r in self.records:
            if r.is_primary:
                return r
        return self.records[0] if self.records else None


def margin_mapq(chains: Sequence[Chain], max_mapq: int = 60) -> int:
    """MAPQ from the primary/secondary chain-score margin (pipeline.py L416-426)."""
    if not chains:
        return 0
    ordered = sorted((c.score for c in chains), reverse=True)
    best = ordered[0]
    if best <= 0:
        return 0
    runner_up = ordered[1] if len(ordered) > 1 else 0.0
    margin = float(np.clip((best - runner_up) / best, 0.0, 1.0))
    return int(np.clip(round(margin * max_mapq), 0, max_mapq))


def node_of(ref_pos: np.ndarray, node_starts: Optional[np.ndarray], node_ids: Optional[np.ndarray]) -> np.ndarray:
    """Graph node of forward-reference offsets, -1 without nodes
    (seeding.py L918-928, ``SeedIndexBundle.node_of``)."""
    ref_pos = np.asarray(ref_pos, np.int64)
    if node_starts is None or len(node_starts) == 0:
        return np.full(len(ref_pos), -1, dtype=np.int64)
    slot = np.clip(np.searchsorted(node_starts, ref_pos, side="right") - 1, 0, len(node_starts) - 1)
    ids = node_ids if node_ids is not None else slot
    return np.asarray(ids, dtype=np.int64)[slot]


def assemble_records(read_id: str, read_len: int, anchors: AnchorSet, chains: Sequence[Chain],
                     extensions: Sequence, ref_id: int = 0, mapq: int = 0, route: str = "full",
                     pass_name: str = "fast", node_starts: Optional[np.ndarray] = None,
                     node_ids: Optional[np.ndarray] = None, neural_scoring: bool = False) -> list:
    """One read's chains (+ extensions) as output records (pipeline.py
    L365-414): the i-th extension belongs to the i-th chain; only the primary
    carries the read's MAPQ."""
    stages = ("seed", "chain") + (("extend",) if extensions else ())
    if neural_scoring:
        stages = stages + ("score",)
    out = []
    for rank, chain in enumerate(chains):
        ext = extensions[rank] if rank < len(extensions) else None
        ref_start = ext.ref_start if ext else chain.ref_start
        ref_end = ext.ref_end if ext else chain.ref_end
        node = node_of(np.asarray([ref_start], dtype=np.int64), node_starts, node_ids)
        out.append(AlignmentRecord(
            read_id=read_id, read_len=read_len, ref_id=ref_id, ref_start=int(ref_start), ref_end=int(ref_end),
            strand=int(chain.strand), mapq=int(mapq) if chain.is_primary else 0,
            chain_score=float(chain.score), alignment_score=float(ext.score) if ext else 0.0,
            cigar=list(ext.cigar) if ext else [], node_id=int(node[0]), is_mapped=True,
            is_primary=chain.is_primary, is_supplementary=not chain.is_primary, route=route,
            pass_name=pass_name, n_anchors=len(anchors), n_chains=len(chains), stages=stages, extension=ext))
    return out


def read_alignments(read_id: str, read_len: int, anchors: AnchorSet, chains: Sequence[Chain], extensions: Sequence,
                    ref_id: int = 0, max_mapq: int = 60, route: str = "fast", pass_name: str = "fast",
                    node_starts=None, node_ids=None) -> ReadAlignments:
    """The fast pipeline's result for one read (pipeline.py L486-511): margin
    MAPQ, records, and an unmapped record when there is no chain."""
    recs = assemble_records(read_id, read_len, anchors, chains, extensions, ref_id=ref_id,
                            mapq=margin_mapq(chains, max_mapq), route=route, pass_name=pass_name,
                            node_starts=node_starts, node_ids=node_ids)
    return ReadAlignments(read_id=read_id, read_len=read_len, anchors=anchors, chains=list(chains),
                          records=recs or [AlignmentRecord.unmapped(read_id, read_len, pass_name=pass_name)])


# --------------------------------------------------------------------------- #
# SAM
# --------------------------------------------------------------------------- #
@dataclass
class SamBatch:
    """Host arrays of the records to render (the layout of gmf_sam_records)."""

    names: np.ndarray
    name_off: np.ndarray
    seq: np.ndarray
    seq_off: np.ndarray
    qual: np.ndarray
    contig: np.ndarray
    contig_names: np.ndarray
    contig_off: np.ndarray
    ref_start: np.ndarray
    ref_end: np.ndarray
    strand: np.ndarray
    mapq: np.ndarray
    cigar: np.ndarray
    cigar_start: np.ndarray
    cigar_len: np.ndarray
    tags: np.ndarray
    tag_off: np.ndarray
    modalities: list  # in order of first appearance (@RG lines)

    def __len__(self) -> int:
        return len(self.contig)


def _csr_bytes(items: Sequence[bytes]) -> tuple:
    off = np.zeros(len(items) + 1, np.int64)
    np.cumsum([len(x) for x in items], out=off[1:])
    flat = np.frombuffer(b"".join(items), np.uint8) if off[-1] else np.zeros(1, np.uint8)
    return flat.copy(), off


def _read_index(reads: Sequence) -> tuple:
    by_id = {}
    for r in reads:
        rid = getattr(r, "read_id", None)
        if rid is not None and rid not in by_id:
            by_id[rid] = r
    return by_id, list(reads)


def sam_records(results: Sequence[ReadAlignments], reads: Sequence, modality: str = "pacbio_hifi",
                include_secondary: bool = False, references: Optional[dict] = None,
                contig_names: Optional[dict] = None) -> SamBatch:
    """Pair results with their reads (alignment_io.py L55-187: by read_id,
    else by position; plain strings or objects with ``seq`` / ``quals`` /
    ``modality``) and lay the records out for the device.  ``references``
    maps ref_id to its length (or an object with ``seq``); contigs are
    numbered in sorted ref_id order (formats.py L265-284)."""
    modality = validate_modality(modality)
    order = sorted(references) if references else []
    ref_index = {rid: i for i, rid in enumerate(order)}
    names_map = contig_names or {}
    contigs = [names_map.get(rid, f"ref{rid}").encode() for rid in order]
    by_id, ordered = _read_index(reads)
    names, seqs, quals, tags, mods = [], [], [], [], []
    contig, rs, re_, strand, mapq, cig, cstart, clen = [], [], [], [], [], [], [], []
    words_total = 0
    for row, al in enumerate(results):
        src = by_id.get(al.read_id)
        if src is None:
            src = ordered[row] if row < len(ordered) else ""
        if isinstance(src, str):
            seq, q, mod = src, None, modality
        else:
            seq = getattr(src, "seq", "")
            q = getattr(src, "quals", None)
            mod = getattr(src, "modality", None) or modality
        mod = validate_modality(mod)
        recs = al.records or []
        if not include_secondary:
            prim = next((r for r in recs if r.is_primary), None)
            recs = [prim] if prim is not None else recs[:1]
        if q is not None and len(q):  # padded with 0 / cut to the bases, clamped to [0, 93]
            qa = np.zeros(len(seq), np.int64)
            qv = np.asarray(q, np.int64)[: len(seq)]
            qa[: len(qv)] = qv
            qb = np.clip(qa, 0, MAX_PHRED).astype(np.uint8).tobytes()
        else:
            qb = bytes(len(seq))
        sb = seq.encode("ascii", errors="replace")
        for rec in recs:
            if rec is None:
                continue
            names.append(str(rec.read_id).encode())
            seqs.append(sb)
            quals.append(qb)
            tags.append(f"RG:Z:{mod}\tXM:Z:{mod}".encode())
            if mod not in mods:
                mods.append(mod)
            if rec.is_mapped:
                c = ref_index.get(int(rec.ref_id), -1)
                words = [(int(n) << 4) | OPS.index(op) for op, n in rec.cigar]
                contig.append(c)
                rs.append(int(rec.ref_start))
                re_.append(int(rec.ref_end))
                strand.append(int(rec.strand))
                mapq.append(min(max(int(rec.mapq), 0), 255))
            else:  # unmapped entry: no contig, no span, no CIGAR (alignment_io.py L80-85)
                words = []
                contig.append(-1)
                rs.append(0)
                re_.append(0)
                strand.append(1)
                mapq.append(0)
            cig.extend(words)
            cstart.append(words_total)
            clen.append(len(words))
            words_total += len(words)
    nm, nm_off = _csr_bytes(names)
    sq, sq_off = _csr_bytes(seqs)
    ql, _ = _csr_bytes(quals)
    tg, tg_off = _csr_bytes(tags)
    cn, cn_off = _csr_bytes(contigs)
    return SamBatch(nm, nm_off, sq, sq_off, ql, np.array(contig, np.int32), cn, cn_off,
                    np.array(rs, np.int64), np.array(re_, np.int64), np.array(strand, np.int8),
                    np.array(mapq, np.int32), np.array(cig if cig else [0], np.uint32),
                    np.array(cstart, np.int64), np.array(clen, np.int32), tg, tg_off, mods)


# --------------------------------------------------------------------------- #
# Records as arrays
# --------------------------------------------------------------------------- #
S_OP = OPS.index("S")
# base codes (A=1 C=2 G=3 T=4, N=5) -> ASCII, as synth.decode_bases maps them
_CODE_ASCII = np.frombuffer(b"$ACGTN", dtype=np.uint8)


@dataclass
class RecordTable:
    """Output records as arrays, one row per record, the rows of a read
    together and reads in order: the SAM fields of AlignmentRecord.  An
    unmapped record has ref_id -1 and an empty CIGAR."""

    read: np.ndarray        # int64: the record's read
    ref_id: np.ndarray      # int64, -1 unmapped
    ref_start: np.ndarray   # int64
    ref_end: np.ndarray     # int64
    strand: np.ndarray      # int8
    mapq: np.ndarray        # int32
    is_primary: np.ndarray  # bool
    cigar: np.ndarray       # uint32 words (run << 4 | op), soft clips included
    cigar_off: np.ndarray   # int64, len + 1

    def __len__(self) -> int:
        return len(self.read)


def margin_mapq_rows(scores: np.ndarray, n: np.ndarray, max_mapq: int = 60) -> np.ndarray:
    """:func:`margin_mapq` of many reads at once: row r holds read r's chain
    scores in its first ``n[r]`` entries.  The same f64 arithmetic
    (best - runner-up) / best, clipped to [0, 1], times ``max_mapq``, rounded
    half to even."""
    scores = np.asarray(scores, np.float64)
    R = len(n)
    out = np.zeros(R, np.int32)
    if R == 0 or scores.shape[1] == 0:
        return out
    valid = np.arange(scores.shape[1])[None, :] < np.asarray(n)[:, None]
    s = -np.sort(-np.where(valid, scores, -np.inf), axis=1)  # descending
    best = s[:, 0]
    runner = np.where(np.asarray(n) > 1, s[:, 1] if s.shape[1] > 1 else 0.0, 0.0)
    ok = (np.asarray(n) > 0) & (best > 0)
    with np.errstate(invalid="ignore", divide="ignore"):
        margin = np.clip((best - runner) / best, 0.0, 1.0)
    q = np.clip(np.rint(margin * max_mapq), 0, max_mapq)
    out[ok] = q[ok].astype(np.int32)
    return out


def _clip_words(words: np.ndarray, cstart: np.ndarray, clen: np.ndarray, left: np.ndarray,
                right: np.ndarray) -> tuple:
    """Each row's CIGAR words ``words[cstart: cstart + clen]`` with its soft
    clips added, as :func:`types.add_soft_clips` adds them to a CIGAR without
    S runs: S(left) before and S(right) after when positive, and an empty
    CIGAR becomes the single run S(left + right) (or stays empty)."""
    K = len(clen)
    clen = np.asarray(clen, np.int64)
    left, right = np.asarray(left, np.int64), np.asarray(right, np.int64)
    empty = clen <= 0
    hl = (~empty & (left > 0)).astype(np.int64)
    hr = (~empty & (right > 0)).astype(np.int64)
    hs = (empty & (left + right > 0)).astype(np.int64)
    body = np.where(empty, 0, clen)
    per = hl + body + hr + hs
    off = np.zeros(K + 1, np.int64)
    np.cumsum(per, out=off[1:])
    out = np.empty(int(off[-1]), np.uint32)
    tot = int(body.sum())
    if tot:
        rep = np.repeat(np.arange(K), body)
        bstart = np.zeros(K + 1, np.int64)
        np.cumsum(body, out=bstart[1:])
        within = np.arange(tot, dtype=np.int64) - bstart[rep]
        out[off[rep] + hl[rep] + within] = np.asarray(words, np.uint32)[np.asarray(cstart, np.int64)[rep] + within]
    k = np.flatnonzero(hl)
    out[off[k]] = (left[k] << 4 | S_OP).astype(np.uint32)
    k = np.flatnonzero(hr)
    out[off[k + 1] - 1] = (right[k] << 4 | S_OP).astype(np.uint32)
    k = np.flatnonzero(hs)
    out[off[k]] = ((left[k] + right[k]) << 4 | S_OP).astype(np.uint32)
    return out, off


def record_table(alignments, ref_id: int = 0, max_mapq: int = 60) -> RecordTable:
    """The fast pipeline's records (pipeline.py L486-511 with the record
    step L365-426) of a batch aligned by ``serving.BatchAligner``, built from
    its arrays: one record per chain in select order, reference span and
    CIGAR (soft clips added) from the chain's extension, the margin MAPQ on
    the primary only, and one unmapped record for a read without chains."""
    ba = alignments
    if ba.chains is None:
        raise ValueError("the batch carries no chain columns")
    # the reads [lo, hi) of the batch (a slice covers part of it)
    full = np.asarray(ba.chain_off, np.int64)
    c0, c1 = int(full[ba.lo]), int(full[ba.hi])
    coff = full[ba.lo: ba.hi + 1] - c0
    R = len(coff) - 1
    n = np.diff(coff)
    ch = {k: np.asarray(v)[c0:c1] for k, v in ba.chains.items()}
    C = c1 - c0
    # per read, the scores of its chains in a (R, max n) block
    width = int(n.max(initial=0))
    cols = np.arange(max(width, 1))[None, :]
    take = np.minimum(coff[:-1, None] + cols, max(C - 1, 0))
    block = np.asarray(ch["score"], np.float64)[take] if C else np.zeros((R, 1))
    mq = margin_mapq_rows(block, n, max_mapq)
    creads = np.repeat(np.arange(R, dtype=np.int64), n)
    prim = np.asarray(ch["prim"]).astype(bool)
    if ba.cols is not None:
        k = {name: np.asarray(v)[c0:c1] for name, v in ba.cols.items()}
        words, woff = _clip_words(ba.words, k["cstart"], k["clen"], k["clip_l"], k["clip_r"])
        rs, re_ = np.asarray(k["ts"], np.int64), np.asarray(k["te"], np.int64)
    else:  # per-chain ExtensionResults (the WFA path)
        exts = ba.objects[c0:c1]
        runs = [[(int(m) << 4) | OPS.index(op) for op, m in e.cigar] for e in exts]
        woff = np.zeros(C + 1, np.int64)
        np.cumsum([len(x) for x in runs], out=woff[1:])
        words = np.array([w for x in runs for w in x], np.uint32)
        rs = np.array([e.ref_start for e in exts], np.int64)
        re_ = np.array([e.ref_end for e in exts], np.int64)
    # reads without chains get one unmapped record, in read order
    none = np.flatnonzero(n == 0)
    N = C + len(none)
    row = np.empty(N, np.int64)
    row_of_chain = np.arange(C) + np.searchsorted(none, creads, side="left")
    # a chainless read's row follows every chain row of the reads before it
    row_of_none = np.searchsorted(creads, none, side="left") + np.arange(len(none))
    row[row_of_chain] = creads
    row[row_of_none] = none

    def fill(vals, default, dt):
        a = np.full(N, default, dt)
        a[row_of_chain] = vals
        return a

    per = np.zeros(N, np.int64)
    per[row_of_chain] = np.diff(woff)
    off = np.zeros(N + 1, np.int64)
    np.cumsum(per, out=off[1:])
    return RecordTable(read=row, ref_id=fill(ref_id, -1, np.int64), ref_start=fill(rs, -1, np.int64),
                       ref_end=fill(re_, -1, np.int64), strand=fill(np.asarray(ch["strand"], np.int8), 1, np.int8),
                       mapq=fill(np.where(prim, mq[creads], 0), 0, np.int32),
                       is_primary=fill(prim, True, bool), cigar=words, cigar_off=off)


def _name_csr(names) -> tuple:
    """Read names as (bytes, offsets): a (uint8 array, int64 offsets) pair
    passes through; a sequence of strings is joined once."""
    if isinstance(names, tuple):
        return np.asarray(names[0], np.uint8), np.asarray(names[1], np.int64)
    names = [str(x) for x in names]
    joined = "".join(names)
    raw = joined.encode("utf-8")
    if len(raw) == len(joined):
        lens = np.fromiter(map(len, names), np.int64, len(names))
    else:
        lens = np.fromiter((len(x.encode("utf-8")) for x in names), np.int64, len(names))
    off = np.zeros(len(names) + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    return np.frombuffer(raw, np.uint8), off


def _gather_csr(flat: np.ndarray, off: np.ndarray, rows: np.ndarray) -> tuple:
    """The rows ``rows`` of a CSR array, concatenated."""
    lens = off[rows + 1] - off[rows]
    out_off = np.zeros(len(rows) + 1, np.int64)
    np.cumsum(lens, out=out_off[1:])
    tot = int(out_off[-1])
    if tot == 0:
        return np.zeros(0, flat.dtype), out_off
    rep = np.repeat(np.arange(len(rows)), lens)
    src = off[rows][rep] + (np.arange(tot, dtype=np.int64) - out_off[:-1][rep])
    return flat[src], out_off


def sam_batch(table: RecordTable, names, seq: np.ndarray, seq_off: np.ndarray, qual: Optional[np.ndarray] = None,
              modality="pacbio_hifi", include_secondary: bool = False, references: Optional[dict] = None,
              contig_names: Optional[dict] = None) -> SamBatch:
    """:func:`sam_records` for records held as a :class:`RecordTable` and
    reads held as arrays: ``names`` (one string per read, or a (bytes,
    offsets) pair), ``seq`` / ``seq_off`` the reads' ASCII bases (or base
    codes, int8) as CSR, ``qual`` Phred values aligned with ``seq`` (None:
    no qualities), ``modality`` one name or one per read.  Without
    ``include_secondary`` a read keeps its first primary record, else its
    first record.  The layout equals :func:`sam_records`' for the same
    records, with no per-record Python work."""
    seq_off = np.asarray(seq_off, np.int64)
    R = len(seq_off) - 1
    rows = np.arange(len(table), dtype=np.int64)
    if not include_secondary and len(rows):
        # per read the first primary row, else its first row
        order = np.lexsort((rows, ~np.asarray(table.is_primary, bool), table.read))
        _, first = np.unique(table.read[order], return_index=True)
        rows = np.sort(order[first])
    rd = np.asarray(table.read, np.int64)[rows]
    if len(rd) and (rd.min() < 0 or rd.max() >= R):
        raise ValueError("a record's read index is outside the reads")
    # modalities: canonical names, first appearance order over the kept records
    if isinstance(modality, str):
        mod_names = [validate_modality(modality)]
        mod_of_read = np.zeros(R, np.int64)
    else:
        canon = [validate_modality(m) for m in modality]
        mod_names = list(dict.fromkeys(canon))
        idx = {m: i for i, m in enumerate(mod_names)}
        mod_of_read = np.array([idx[m] for m in canon], np.int64)
    rec_mod = mod_of_read[rd]
    seen = np.zeros(len(mod_names), np.int64)
    if len(rd):
        first_seen = np.full(len(mod_names), len(rd), np.int64)
        np.minimum.at(first_seen, rec_mod, np.arange(len(rd)))
        seen = first_seen
    used = [i for i in np.argsort(seen, kind="stable") if len(rd) and seen[i] < len(rd)]
    mods = [mod_names[i] for i in used]
    tag_items = [f"RG:Z:{m}\tXM:Z:{m}".encode() for m in mod_names]
    if len(mod_names) == 1:  # one tag string for every record
        t1 = np.frombuffer(tag_items[0], np.uint8)
        tg, tg_off = np.tile(t1, len(rd)), np.arange(len(rd) + 1, dtype=np.int64) * len(t1)
    else:
        tb, toff = _csr_bytes(tag_items)
        tg, tg_off = _gather_csr(tb, toff, rec_mod)
    identity = len(rd) == R and bool(np.all(rd == np.arange(R)))  # one record per read, in read order
    nm_flat, nm_off = _name_csr(names)
    nm, nmo = (nm_flat[: nm_off[-1]], nm_off) if identity else _gather_csr(nm_flat, nm_off, rd)
    sq = np.asarray(seq)
    if len(sq) < seq_off[-1] or (qual is not None and len(qual) < seq_off[-1]):
        raise ValueError("seq_off runs past the bases or the qualities")
    if sq.dtype == np.int8:
        sq = _CODE_ASCII[np.clip(sq, 0, 5)]
    if qual is None:
        ql = np.zeros(len(sq), np.uint8)
    else:
        ql = np.asarray(qual)
        if ql.dtype == np.uint8:  # clamped only when a value is above the Phred limit
            ql = ql if len(ql) == 0 or ql.max() <= MAX_PHRED else np.minimum(ql, MAX_PHRED)
        else:
            ql = np.clip(ql, 0, MAX_PHRED).astype(np.uint8)
    if identity:  # the read arrays as they are
        sq_r, sq_ro, ql_r = sq[: seq_off[-1]], seq_off, ql[: seq_off[-1]]
    else:
        sq_r, sq_ro = _gather_csr(sq, seq_off, rd)
        ql_r, _ = _gather_csr(ql, seq_off, rd)
    order_ids = sorted(references) if references else []
    names_map = contig_names or {}
    cn, cn_off = _csr_bytes([names_map.get(rid, f"ref{rid}").encode() for rid in order_ids])
    rid = np.asarray(table.ref_id, np.int64)[rows]
    mapped = rid >= 0
    ids = np.asarray(order_ids, np.int64)
    if len(ids):
        pos = np.clip(np.searchsorted(ids, rid), 0, len(ids) - 1)
        contig = np.where(mapped & (ids[pos] == rid), pos, -1).astype(np.int32)
    else:
        contig = np.full(len(rows), -1, np.int32)
    coff = np.asarray(table.cigar_off, np.int64)
    clen = np.where(mapped, coff[rows + 1] - coff[rows], 0)
    if len(rows) == len(table) and not np.any(clen != coff[rows + 1] - coff[rows]):
        # every row kept and no unmapped row holds words: the table's words as they are
        cw, cstart = np.asarray(table.cigar, np.uint32)[: coff[-1]], coff[:-1].copy()
    else:
        cw, cwo = _gather_csr(np.asarray(table.cigar, np.uint32), coff, rows[mapped])
        cstart = np.zeros(len(rows), np.int64)
        cstart[mapped] = cwo[:-1]
        cstart[~mapped] = np.searchsorted(np.flatnonzero(mapped), np.flatnonzero(~mapped))
        cstart[~mapped] = cwo[cstart[~mapped]]
    return SamBatch(nm if len(nm) else np.zeros(1, np.uint8), nmo, sq_r if len(sq_r) else np.zeros(1, np.uint8), sq_ro,
                    ql_r if len(ql_r) else np.zeros(1, np.uint8), contig, cn, cn_off,
                    np.where(mapped, np.asarray(table.ref_start, np.int64)[rows], 0),
                    np.where(mapped, np.asarray(table.ref_end, np.int64)[rows], 0),
                    np.where(mapped, np.asarray(table.strand, np.int8)[rows], 1).astype(np.int8),
                    np.where(mapped, np.clip(np.asarray(table.mapq, np.int64)[rows], 0, 255), 0).astype(np.int32),
                    cw if len(cw) else np.zeros(1, np.uint32), cstart, clen.astype(np.int32),
                    tg if len(tg) else np.zeros(1, np.uint8), tg_off, mods)


def sam_header(references: Optional[dict], contig_names: Optional[dict], modalities: Sequence[str]) -> str:
    """@HD, @SQ (sorted ref_id), @RG (one per modality), @PG lines
    (formats.py L323-340, unsorted output)."""
    lines = ["@HD\tVN:1.6\tSO:unsorted"]
    names = contig_names or {}
    for rid in sorted(references or {}):
        ref = references[rid]
        n = int(ref) if isinstance(ref, (int, np.integer)) else len(getattr(ref, "seq", ref))
        lines.append(f"@SQ\tSN:{names.get(rid, f'ref{rid}')}\tLN:{n}")
    for mod in modalities:
        lines.append(f"@RG\tID:{mod}\tPL:{MODALITY_PLATFORM.get(mod, 'UNKNOWN')}\tSM:sample\tLB:{mod}")
    lines.append("@PG\tID:graphmambaformer\tPN:graphmambaformer\tDS:reads/alignments emitted by the format I/O layer")
    return "\n".join(lines) + "\n"


def render_sam_array(batch: SamBatch, device=None, stream: Optional[torch.cuda.Stream] = None,
                     max_seq_len: Optional[int] = None) -> np.ndarray:
    """The records' SAM lines, rendered on the device (two launches and one
    scan), as a uint8 array in page-locked host memory (no further copy; a
    file's ``write`` takes it as it is).  Columns already page-locked go to
    the device directly.  ``max_seq_len`` overrides the longest-record hint
    that splits the fill pass (it changes speed only)."""
    dev = require_cuda(device)
    n = len(batch)
    if n == 0:
        return np.zeros(0, np.uint8)
    s = stream or torch.cuda.current_stream(dev)
    with torch.cuda.stream(s):
        up = lambda a: to_device(a, dev)  # noqa: E731
        d = dict(name=up(batch.names), name_off=up(batch.name_off), seq=up(batch.seq), seq_off=up(batch.seq_off),
                 qual=up(batch.qual), contig=up(batch.contig), contig_names=up(batch.contig_names),
                 contig_off=up(batch.contig_off), ref_start=up(batch.ref_start), ref_end=up(batch.ref_end),
                 strand=up(batch.strand), mapq=up(batch.mapq), cigar=up(batch.cigar),
                 cigar_start=up(batch.cigar_start), cigar_len=up(batch.cigar_len), tags=up(batch.tags),
                 tag_off=up(batch.tag_off))
        p = {k: v.data_ptr() for k, v in d.items()}
        longest = int(np.diff(batch.seq_off).max()) if max_seq_len is None else int(max_seq_len)
        rec = _native.GmfSamRecords(n, p["name"], p["name_off"], p["seq"], p["seq_off"], p["qual"], p["contig"],
                                    p["contig_names"], p["contig_off"], len(batch.contig_off) - 1, p["ref_start"],
                                    p["ref_end"], p["strand"], p["mapq"], p["cigar"], p["cigar_start"],
                                    p["cigar_len"], None, None, p["tags"], p["tag_off"], longest)
        sp = int(s.cuda_stream)
        bind(dev, sp)
        lens = torch.empty(n, dtype=torch.int64, device=dev)
        _native.check("gmf_sam_count", _native.lib().gmf_sam_count(ctypes.byref(rec),
                                                                   ctypes.c_void_p(lens.data_ptr()),
                                                                   ctypes.c_void_p(sp)))
        off = torch.zeros(n + 1, dtype=torch.int64, device=dev)
        torch.cumsum(lens, 0, out=off[1:])
        total = int(off[-1].item())
        text = torch.empty(max(total, 1), dtype=torch.uint8, device=dev)
        _native.check("gmf_sam_fill", _native.lib().gmf_sam_fill(ctypes.byref(rec), ctypes.c_void_p(off.data_ptr()),
                                                                 ctypes.c_void_p(text.data_ptr()),
                                                                 ctypes.c_void_p(sp)))
        host = torch.empty(max(total, 1), dtype=torch.uint8, pin_memory=True)
        host[:total].copy_(text[:total], non_blocking=True)
    s.synchronize()
    return host.numpy()[:total]


def render_sam(batch: SamBatch, device=None, stream: Optional[torch.cuda.Stream] = None,
               max_seq_len: Optional[int] = None) -> bytes:
    """:func:`render_sam_array` as bytes."""
    return render_sam_array(batch, device, stream, max_seq_len).tobytes()


def write_sam(results: Sequence[ReadAlignments], reads: Sequence, path: str, references: Optional[dict] = None,
              modality: str = "pacbio_hifi", include_secondary: bool = False,
              contig_names: Optional[dict] = None, device=None) -> str:
    """``write_alignments(results, reads, "x.sam", ...)`` (alignment_io.py
    L190-221): header, then one line per record, rendered on the device."""
    batch = sam_records(results, reads, modality, include_secondary, references, contig_names)
    return _write(path, batch, references, contig_names, device)


def write_sam_table(table: RecordTable, names, seq: np.ndarray, seq_off: np.ndarray, path: str,
                    qual: Optional[np.ndarray] = None, modality="pacbio_hifi", include_secondary: bool = False,
                    references: Optional[dict] = None, contig_names: Optional[dict] = None, device=None) -> str:
    """:func:`write_sam` for records and reads held as arrays (see
    :func:`sam_batch`)."""
    batch = sam_batch(table, names, seq, seq_off, qual, modality, include_secondary, references, contig_names)
    return _write(path, batch, references, contig_names, device)


def _write(path: str, batch: SamBatch, references, contig_names, device) -> str:
    text = render_sam_array(batch, device)
    with open(path, "wb") as fh:
        fh.write(sam_header(references, contig_names, batch.modalities).encode())
        fh.write(memoryview(text))
    return path
