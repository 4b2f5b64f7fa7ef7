"""SAM records restated in plain Python (test infrastructure only: the
checker of the device SAM formatter, never shipped or timed).

Follows graphmambaformer/data/alignment_io.py L55-106
(alignment_to_read_record) and data/formats.py L287-289 (_is_mapped) and
L343-397 (_make_segment), then renders the fields as SAM text the way the
SAM specification lays them out (what pysam writes for an AlignedSegment):
QNAME FLAG RNAME POS(1-based) MAPQ CIGAR RNEXT PNEXT TLEN SEQ QUAL TAGS.
Pinned by tests/golden/sam_golden.pkl, whose fields come from the reference's
own functions.
"""

from __future__ import annotations

_COMPLEMENT = {"A": "T", "C": "G", "G": "C", "T": "A", "N": "N"}
_OP2CODE = {"M": 0, "I": 1, "D": 2, "N": 3, "S": 4, "H": 5, "P": 6, "=": 7, "X": 8}
_CODE2OP = {v: k for k, v in _OP2CODE.items()}
_QUERY_OPS = {"M", "I", "S", "=", "X"}


def segment(rec: dict, seq: str, quals, modality: str, ref_index: dict) -> dict:
    """Fields of the SAM segment of one record.  ``rec``: read_id, is_mapped,
    ref_id, ref_start, ref_end, strand, mapq, cigar (list of (op, n))."""
    q = list(quals) if quals else [0] * len(seq)
    if len(q) < len(seq):
        q = q + [0] * (len(seq) - len(q))
    q = q[: len(seq)]
    if rec["is_mapped"]:
        ref_id, ref_start, ref_end, strand = rec["ref_id"], rec["ref_start"], rec["ref_end"], rec["strand"]
        cigar, mapq = list(rec["cigar"]), rec["mapq"]
    else:
        ref_id, ref_start, ref_end, strand, cigar, mapq = -1, 0, 0, 1, [], 0
    flag = 0
    mapped = (ref_id is not None and ref_id >= 0 and bool(seq) and ref_end > ref_start and bool(cigar)
              and ref_id in ref_index)
    if mapped and strand == -1:
        flag |= 0x10
        cigar = list(reversed(cigar))
        seq = "".join(_COMPLEMENT.get(b, "N") for b in reversed(seq))
        q = list(reversed(q))
    if mapped and sum(n for op, n in cigar if op in _QUERY_OPS) != len(seq):
        mapped = False
    out = dict(qname=rec["read_id"], rnext=-1, pnext=-1, tlen=0)
    if mapped:
        out.update(flag=flag, ref=ref_index[ref_id], pos=ref_start, mapq=int(mapq),
                   cigar=[(_OP2CODE.get(op, 0), n) for op, n in cigar])
    else:
        out.update(flag=flag | 0x4, ref=-1, pos=-1, mapq=0, cigar=None)
    out["seq"] = seq or "*"
    out["qual"] = [min(93, max(0, v)) for v in q[: len(seq)]] or None if seq else None
    out["tags"] = [("RG", str(modality)), ("XM", str(modality))] if modality else []
    return out


def render(seg: dict, contigs: list) -> str:
    """One SAM line (no newline) of a segment's fields."""
    cigar = "*" if not seg["cigar"] else "".join(f"{n}{_CODE2OP[c]}" for c, n in seg["cigar"])
    qual = "*" if seg["qual"] is None else "".join(chr(33 + v) for v in seg["qual"])
    cols = [seg["qname"], str(seg["flag"]), contigs[seg["ref"]] if seg["ref"] >= 0 else "*", str(seg["pos"] + 1),
            str(seg["mapq"]), cigar, "*" if seg["rnext"] < 0 else contigs[seg["rnext"]], str(seg["pnext"] + 1),
            str(seg["tlen"]), seg["seq"], qual]
    cols += [f"{k}:Z:{v}" for k, v in seg["tags"]]
    return "\t".join(cols)
