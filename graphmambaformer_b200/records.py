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


def render_sam(batch: SamBatch, device=None, stream: Optional[torch.cuda.Stream] = None,
               max_seq_len: Optional[int] = None) -> bytes:
    """The records' SAM lines, rendered on the device (two launches and one
    scan), as bytes.  ``max_seq_len`` overrides the longest-record hint that
    splits the fill pass (it changes speed only)."""
    dev = require_cuda(device)
    n = len(batch)
    if n == 0:
        return b""
    up = lambda a: to_device(a, dev)  # noqa: E731
    d = dict(name=up(batch.names), name_off=up(batch.name_off), seq=up(batch.seq), seq_off=up(batch.seq_off),
             qual=up(batch.qual), contig=up(batch.contig), contig_names=up(batch.contig_names),
             contig_off=up(batch.contig_off), ref_start=up(batch.ref_start), ref_end=up(batch.ref_end),
             strand=up(batch.strand), mapq=up(batch.mapq), cigar=up(batch.cigar),
             cigar_start=up(batch.cigar_start), cigar_len=up(batch.cigar_len), tags=up(batch.tags),
             tag_off=up(batch.tag_off))
    p = {k: v.data_ptr() for k, v in d.items()}
    rec = _native.GmfSamRecords(n, p["name"], p["name_off"], p["seq"], p["seq_off"], p["qual"], p["contig"],
                                p["contig_names"], p["contig_off"], len(batch.contig_off) - 1, p["ref_start"],
                                p["ref_end"], p["strand"], p["mapq"], p["cigar"], p["cigar_start"], p["cigar_len"],
                                None, None, p["tags"], p["tag_off"], int(np.diff(batch.seq_off).max()) if max_seq_len is None else int(max_seq_len))
    sp = stream_handle(stream, dev)
    bind(dev, sp)
    lens = torch.empty(n, dtype=torch.int64, device=dev)
    _native.check("gmf_sam_count", _native.lib().gmf_sam_count(ctypes.byref(rec), ctypes.c_void_p(lens.data_ptr()),
                                                               ctypes.c_void_p(sp)))
    with torch.cuda.stream(stream or torch.cuda.current_stream(dev)):
        off = torch.zeros(n + 1, dtype=torch.int64, device=dev)
        torch.cumsum(lens, 0, out=off[1:])
        total = int(off[-1].item())
        text = torch.empty(max(total, 1), dtype=torch.uint8, device=dev)
    _native.check("gmf_sam_fill", _native.lib().gmf_sam_fill(ctypes.byref(rec), ctypes.c_void_p(off.data_ptr()),
                                                             ctypes.c_void_p(text.data_ptr()), ctypes.c_void_p(sp)))
    return text[:total].to("cpu").numpy().tobytes()


def write_sam(results: Sequence[ReadAlignments], reads: Sequence, path: str, references: Optional[dict] = None,
              modality: str = "pacbio_hifi", include_secondary: bool = False,
              contig_names: Optional[dict] = None, device=None) -> str:
    """``write_alignments(results, reads, "x.sam", ...)`` (alignment_io.py
    L190-221): header, then one line per record, rendered on the device."""
    batch = sam_records(results, reads, modality, include_secondary, references, contig_names)
    text = render_sam(batch, device)
    with open(path, "wb") as fh:
        fh.write(sam_header(references, contig_names, batch.modalities).encode())
        fh.write(text)
    return path
