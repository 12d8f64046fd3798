"""SAM fields for comparisons (test infrastructure: used by tests/ and the
bench's post-timing validation, never by the product path).

ours_as_fields turns the library's tail records (msg_tail_batch /
msg_tail_pe_batch) into the fields of the reference harness's lines
(oracle/ref/ref_harness.cpp: QNAME FLAG TID POS MAPQ CIGAR L_SEQ SEQ QUAL
ISIZE, then aux AS, MD, XH, NH, XN, XP); ref_as_fields splits those lines,
float tags read back from their hex text, so both compare exactly."""
import numpy as np

_COMP = np.array([0, 8, 4, 12, 2, 10, 6, 14, 1, 9, 5, 13, 3, 11, 7, 15], dtype=np.uint8)


def ours_as_fields(recs, md, seq, qual, off, cigar, pairs=False):
    """The library's tail records as the fields of the reference harness's
    lines (floats as float values, compared exactly)."""
    rows = []
    for r in recs:
        i = int(r["read"])
        name = f"p{i // 2}" if pairs else f"r{i}"
        q = seq[off[i]:off[i + 1]]
        ql = qual[off[i]:off[i + 1]]
        if r["flag"] & 0x10:
            q, ql = _COMP[q[::-1]], ql[::-1]
        cg = cigar[r["cigar_off"]:r["cigar_off"] + r["n_cigar"]] if r["n_cigar"] else []
        cs = "".join(f"{int(c) >> 4}{'MIDNSHP=XB'[int(c) & 15]}" for c in cg) or "*"
        f = [name, str(int(r["flag"])), str(int(r["tid"])), str(int(r["pos"])), str(int(r["mapq"])), cs,
             str(len(q)), "".join(f"{int(x):x}" for x in q), "".join(f"{int(x):02x}" for x in ql),
             str(int(r["isize"]))]
        if not r["flag"] & 0x4:
            m = md[r["md_off"]:r["md_off"] + r["md_len"]].decode()
            f += [f"AS:i:{int(r['as'])}", f"MD:Z:{m}", ("XH", float(r["xh"])), f"NH:i:{int(r['nh'])}",
                  f"XN:i:{int(r['xn'])}", ("XP", float(r["xp"]))]
        rows.append(f)
    return rows


def ref_as_fields(lines):
    """The reference harness's SAM lines as fields."""
    rows = []
    for line in lines:
        f = line.split("\t")
        out = f[:10]
        for a in f[10:]:
            tag, typ, val = a.split(":", 2)
            out.append((tag, float.fromhex(val)) if typ == "f" else a)
        rows.append(out)
    return rows
