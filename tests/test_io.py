"""Reads in, SAM text out (host code of the library, no GPU):

* msg_fastq_parse against the reference's own FASTQ reader (SeqIO +
  PrimarySeq, compiled from its sources) on records with the inputs the
  reader meets: descriptions, lowercase and IUPAC bases, digits and other
  characters its table maps to 0, carriage returns, quality strings shorter or
  longer than the sequence, quality bytes below '!', names after blank
  lines, a final record without its last newline or its last lines; and
  streamed in pieces, the same reads as in one piece.
* msg_sam_format on the host tail's records: every SAM field against the
  record and read it comes from (htslib's own float formatting is not
  available here; %g is checked).
* BAM output (msg_bam_header, msg_bam_format, msg_bgzf_compress): the file
  decoded with gzip and a BAM reader written here carries the same fields.
"""
import os

import numpy as np
import pytest

from msgseqtk_b200 import index_build, lib, synth
from oracle.bind import REF_SO, Oracle, Reference

needs_ref = pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref not built")


def _ours_lines(res):
    lines = []
    names = res["text"].split(b"\n")
    for i in range(len(res["off"]) - 1):
        a, b = res["off"][i], res["off"][i + 1]
        name, desc = names[i].split(b"\t", 1)
        lines.append("\t".join([name.decode("latin-1"), desc.decode("latin-1"),
                                "".join(f"{int(x):x}" for x in res["seq"][a:b]),
                                "".join(f"{int(x):02x}" for x in res["qual"][a:b])]))
    return lines


def _fastq_text(seed):
    rng = np.random.default_rng(seed)
    chars = bytes(range(33, 127)).replace(b"@", b"").replace(b"\n", b"")
    recs = []
    for i in range(60):
        L = int(rng.integers(0, 40))
        seq = rng.choice(list(b"ACGTacgtNnRYKMSWBDHVU0123456.-XZ*"), L).astype(np.uint8).tobytes()
        ql = L + int(rng.integers(-3, 4)) if i % 7 == 0 else L
        qual = rng.choice(list(chars), max(ql, 0)).astype(np.uint8).tobytes()
        desc = [b"", b" len=%d" % L, b"\tx y\tz", b"   "][i % 4]
        eol = b"\r\n" if i % 11 == 5 else b"\n"
        recs.append(b"@r%d%s%s%s%s+%s%s%s" % (i, desc, eol, seq, eol, eol, qual, eol))
    recs.append(b"@\n  spaced name\nACGT\n+\nII\x1f!\n")  # name after a blank line; qualities below '!'
    recs.append(b"@last desc\nACGTN\n+\nIIIII")              # no final newline
    return b"".join(recs)


@needs_ref
def test_fastq_parse_matches_reference_reader():
    ref = Reference([synth.small_genomes(seed=1, n_genomes=1, length=2000)[0]])
    for seed in (3, 4):
        text = _fastq_text(seed)
        exp = ref.fastq_parse(text)
        got = lib.fastq_parse(text)
        assert got["consumed"] == len(text)
        assert _ours_lines(got) == exp
    # a final record cut short: the reader fills the missing lines with nothing
    for cut in (b"@a b\nACGT\n+\n", b"@a b\nACGT\n", b"@a b\n"):
        assert _ours_lines(lib.fastq_parse(cut)) == ref.fastq_parse(cut)
    # reading stops at a line that does not start with '@'
    t = b"@a\nAC\n+\nII\n\n@b\nGT\n+\nII\n"
    assert _ours_lines(lib.fastq_parse(t)) == ref.fastq_parse(t)


@needs_ref
def test_fastq_format_matches_reference_writer():
    """Reads parsed and written back (all, or a kept subset as msgseqtk-clean
    writes them) give the reference's SeqIO output byte for byte."""
    ref = Reference([synth.small_genomes(seed=1, n_genomes=1, length=2000)[0]])
    for seed in (6, 7):
        text = _fastq_text(seed)
        r = lib.fastq_parse(text)
        assert lib.fastq_format(r["seq"], r["off"], r["qual"], r["text"], r["name_off"]) == ref.fastq_rewrite(text)
        keep = (np.arange(len(r["off"]) - 1) % 3 != 1).astype(np.uint8)
        assert lib.fastq_format(r["seq"], r["off"], r["qual"], r["text"], r["name_off"], keep) == \
            ref.fastq_rewrite(text, keep)


@needs_ref
def test_clean_assignment_lines_match_reference(oracle_built):
    """FASTQ in (msg_fastq_parse), the lists' loglik (the oracle, pinned to the
    reference in test_clean.py) and msg_clean_format give the reference's
    assignment file lines byte for byte (-inf and nan included)."""
    g_ref = synth.small_genomes(seed=51, n_genomes=2, length=20_000)
    g_bg = synth.small_genomes(seed=52, n_genomes=2, length=20_000)
    ref, bg = Reference(g_ref), Reference(g_bg)
    o_ref, o_bg = Oracle(index_build.build_view(g_ref)), Oracle(index_build.build_view(g_bg))
    rng = np.random.default_rng(53)
    recs = []
    for k, gs in enumerate((g_ref, g_bg, g_ref)):
        rs = synth.sample_reads(gs, 20, seed=54 + k)
        for i in range(len(rs)):
            s = "".join("$ACMGRSVTWYHKDBN"[x] for x in rs.read(i))
            if k == 2 and i % 4 == 0:
                s = s[:30] + "N" + s[31:]  # N inside a kept MEM: loglik -inf
            recs.append(f"@read{k}_{i} desc {i}\n{s}\n+\n{'I' * len(s)}\n")
    text = "".join(recs).encode()
    exp = ref.clean_assign(bg, text)
    r = lib.fastq_parse(text)
    n = len(r["off"]) - 1
    reads = [r["seq"][r["off"][i]:r["off"][i + 1]] for i in range(n)]
    rl = np.array([o_ref.mems(x)[1] for x in reads])
    bl = np.array([o_bg.mems(x)[1] for x in reads])
    with np.errstate(invalid="ignore"):
        lod = -rl + bl
    got = lib.clean_format(r["text"], r["name_off"], rl, bl, lod)
    assert got == exp
    assert b"-inf" in got
    # special values as an ostream prints them
    t = b"a\td\nb\t\nc\t\n"
    line = lib.clean_format(t, np.array([0, 4, 7, 10]), [float("nan"), -float("inf"), 1e-300],
                            [123456789.0, 0.1, -0.0], [float("inf"), 2.5, 1e21])
    assert line == b"a\td\tnan\t1.23457e+08\tinf\nb\t\t-inf\t0.1\t2.5\nc\t\t1e-300\t-0\t1e+21\n"


def test_fastq_parse_streams_in_pieces():
    text = _fastq_text(5)
    whole = lib.fastq_parse(text)
    lines, pos = [], 0
    while pos < len(text):
        piece = text[pos:pos + 97]
        r = lib.fastq_parse(piece, at_eof=pos + 97 >= len(text))
        if r["consumed"] == 0:  # not one whole record in the piece: take a longer one
            piece = text[pos:pos + 2000]
            r = lib.fastq_parse(piece, at_eof=pos + 2000 >= len(text))
        lines += _ours_lines(r)
        pos += r["consumed"]
        assert r["consumed"] > 0
    assert lines == _ours_lines(whole)
    # a record whose name follows a line break is not taken before its last line
    t = b"@\n  n d\nACGT\n+\nIIII\n"
    assert lib.fastq_parse(t[:-6], at_eof=False)["consumed"] == 0
    assert _ours_lines(lib.fastq_parse(t[:-1], at_eof=False)) == []
    assert _ours_lines(lib.fastq_parse(t, at_eof=False)) == _ours_lines(lib.fastq_parse(t))
    # a read cap stops early and reports what was consumed
    r = lib.fastq_parse(text, max_reads=5)
    assert len(r["off"]) == 6 and 0 < r["consumed"] < len(text)


@needs_ref
def test_sam_format_fields(oracle_built):
    g = synth.small_genomes(seed=41, n_genomes=3, length=40_000)
    view = index_build.build_view(g)
    orc = Oracle(view)
    rs = synth.sample_reads(g, 60, seed=42)
    rng = np.random.default_rng(43)
    reads = [rs.read(i) for i in range(len(rs))] + [synth._BASES[rng.integers(0, 4, 150)] for _ in range(5)]
    quals = [rs.qual(i) for i in range(len(rs))] + [rng.integers(20, 41, 150).astype(np.uint8) for _ in range(5)]
    recs, cig, roff = [], [], [0]
    for i, r in enumerate(reads):
        for e in orc.align_read(r):
            recs.append((i, e["tid"], e["strand"], e["t_start"], e["t_end"], e["aln_from"], e["aln_to"],
                         e["aln_start"], e["aln_end"], int(e["aln_score"]), e["flags"], len(cig), len(e["cigar"]), 0))
            cig += e["cigar"]
        roff.append(len(recs))
    aln = np.array(recs, dtype=lib.ALN_DTYPE)
    cig = np.array(cig, dtype=np.uint32)
    seq = np.concatenate(reads).astype(np.uint8)
    qual = np.concatenate(quals).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(x) for x in reads])]).astype(np.int64)
    out, md = lib.tail(view, seq, off, qual, aln, cig, np.array(roff), lib.tail_params(max_report=0))
    names = b"".join(b"read%d\tsome description\n" % i for i in range(len(reads)))
    name_off = np.concatenate([[0], np.cumsum([len(b"read%d\tsome description\n" % i) for i in range(len(reads))])])
    chrom = [f"chr{t}" for t in range(len(g))]
    text = lib.sam_format(out, md, seq, off, qual, cig, names, name_off, chrom).decode()
    lines = text.rstrip("\n").split("\n")
    assert len(lines) == len(out)
    comp = np.array([0, 8, 4, 12, 2, 10, 6, 14, 1, 9, 5, 13, 3, 11, 7, 15])
    for line, r in zip(lines, out):
        f = line.split("\t")
        i = int(r["read"])
        assert f[0] == f"read{i}" and int(f[1]) == r["flag"]
        q, ql = reads[i], quals[i]
        if r["flag"] & 0x10:
            q, ql = comp[q[::-1]], ql[::-1]
        assert f[9] == "".join("=ACMGRSVTWYHKDBN"[int(x)] for x in q)
        assert f[10] == "".join(chr(int(x) + 33) for x in ql)
        assert f[6:9] == ["*", "1", str(int(r["isize"]))]
        if r["flag"] & 0x4:
            assert f[2:6] == ["*", "1", "0", "*"] and len(f) == 11
            continue
        assert f[2] == chrom[r["tid"]] and int(f[3]) == r["pos"] + 1 and int(f[4]) == r["mapq"]
        cs = "".join(f"{int(c) >> 4}{'MIDNSHP=XB'[int(c) & 15]}" for c in cig[r["cigar_off"]:r["cigar_off"] + r["n_cigar"]])
        assert f[5] == cs
        assert f[11:] == [f"AS:i:{int(r['as'])}", "MD:Z:" + md[r["md_off"]:r["md_off"] + r["md_len"]].decode(),
                          "XH:f:%g" % float(r["xh"]), f"NH:i:{int(r['nh'])}", f"XN:i:{int(r['xn'])}",
                          "XP:f:%g" % float(r["xp"])]


_EOF = bytes([31, 139, 8, 4, 0, 0, 0, 0, 0, 255, 6, 0, 66, 67, 2, 0, 27, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0])


def _bgzf_members(data: bytes):
    """(header bytes, deflated body, CRC32, ISIZE) of each BGZF member, with
    the member layout checked: gzip magic, FEXTRA, one 'BC' subfield whose
    BSIZE is the member's size - 1."""
    import struct
    out, p = [], 0
    while p < len(data):
        assert data[p:p + 4] == b"\x1f\x8b\x08\x04"
        xlen = struct.unpack_from("<H", data, p + 10)[0]
        assert xlen == 6 and data[p + 12:p + 16] == b"BC\x02\x00"
        bsize = struct.unpack_from("<H", data, p + 16)[0] + 1
        crc, isize = struct.unpack_from("<II", data, p + bsize - 8)
        out.append((data[p + 18:p + bsize - 8], crc, isize))
        p += bsize
    assert p == len(data)
    return out


def _bam_decode(raw: bytes):
    """The header (text, references) and records of an uncompressed BAM stream."""
    import struct
    assert raw[:4] == b"BAM\x01"
    lt = struct.unpack_from("<i", raw, 4)[0]
    text = raw[8:8 + lt]
    p = 8 + lt
    nref = struct.unpack_from("<i", raw, p)[0]
    p += 4
    refs = []
    for _ in range(nref):
        ln = struct.unpack_from("<i", raw, p)[0]
        name = raw[p + 4:p + 4 + ln]
        assert name.endswith(b"\0")
        refs.append((name[:-1].decode(), struct.unpack_from("<i", raw, p + 4 + ln)[0]))
        p += 8 + ln
    recs = []
    while p < len(raw):
        bs = struct.unpack_from("<i", raw, p)[0]
        r = raw[p + 4:p + 4 + bs]
        p += 4 + bs
        tid, pos, lrn, mapq, bin_, ncig, flag, lseq, ntid, npos, tlen = struct.unpack_from("<iiBBHHHiiii", r, 0)
        q = 32
        name = r[q:q + lrn]
        assert name.endswith(b"\0")
        q += lrn
        cig = list(struct.unpack_from("<%dI" % ncig, r, q))
        q += 4 * ncig
        packed = r[q:q + (lseq + 1) // 2]
        q += (lseq + 1) // 2
        seq = [(packed[i // 2] >> (4 if i % 2 == 0 else 0)) & 15 for i in range(lseq)]
        qual = list(r[q:q + lseq])
        q += lseq
        aux = []
        sizes = {"c": "<b", "C": "<B", "s": "<h", "S": "<H", "i": "<i", "I": "<I", "f": "<f"}
        while q < len(r):
            tag, typ = r[q:q + 2].decode(), chr(r[q + 2])
            q += 3
            if typ == "Z":
                e = r.index(b"\0", q)
                aux.append((tag, typ, r[q:e].decode()))
                q = e + 1
            else:
                v = struct.unpack_from(sizes[typ], r, q)[0]
                aux.append((tag, typ, v))
                q += struct.calcsize(sizes[typ])
        recs.append(dict(tid=tid, pos=pos, mapq=mapq, bin=bin_, flag=flag, tlen=tlen, ntid=ntid, npos=npos,
                         name=name[:-1].decode(), cigar=cig, seq=seq, qual=qual, aux=aux))
    return text, refs, recs


def _reg2bin(beg, end):
    """The SAM specification's reg2bin (section 5.3), on end - 1."""
    end -= 1
    for s, t in ((14, 4681), (17, 585), (20, 73), (23, 9), (26, 1)):
        if beg >> s == end >> s:
            return t + (beg >> s)
    return 0


@pytest.mark.parametrize("paired", [False, True])
def test_bam_output_carries_the_sam_fields(oracle_built, paired):
    """msg_bam_header + msg_bam_format + msg_bgzf_compress: a BGZF file whose
    members are well formed (gzip checks each member's CRC32 and size), whose
    header holds the text and references given, and whose records carry
    exactly the fields of msg_sam_format's lines and the tail's records (XH
    and XP as the same float32 values, integers in their smallest type)."""
    import gzip
    import zlib
    g = synth.small_genomes(seed=44, n_genomes=3, length=40_000)
    view = index_build.build_view(g)
    orc = Oracle(view)
    if paired:
        m1, m2 = synth.sample_pairs(g, 40, seed=45)
        reads = []
        quals = []
        for i in range(len(m1)):
            reads += [m1.read(i), m2.read(i)]
            quals += [m1.qual(i), m2.qual(i)]
    else:
        rs = synth.sample_reads(g, 80, seed=45)
        reads = [rs.read(i) for i in range(len(rs))]
        quals = [rs.qual(i) for i in range(len(rs))]
    rng = np.random.default_rng(46)
    reads += [synth._BASES[rng.integers(0, 4, 151)] for _ in range(4)]  # unmapped, odd length
    quals += [rng.integers(20, 41, 151).astype(np.uint8) for _ in range(4)]
    recs, cig, roff = [], [], [0]
    for i, r in enumerate(reads):
        for e in orc.align_read(r):
            recs.append((i, e["tid"], e["strand"], e["t_start"], e["t_end"], e["aln_from"], e["aln_to"],
                         e["aln_start"], e["aln_end"], int(e["aln_score"]), e["flags"], len(cig), len(e["cigar"]), 0))
            cig += e["cigar"]
        roff.append(len(recs))
    aln = np.array(recs, dtype=lib.ALN_DTYPE)
    cig = np.array(cig, dtype=np.uint32)
    seq = np.concatenate(reads).astype(np.uint8)
    qual = np.concatenate(quals).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(x) for x in reads])]).astype(np.int64)
    pairing = lib.pair_params(mean=400.0, sd=50.0, min_ins=-100.0, max_ins=900.0) if paired else None
    out, md = lib.tail(view, seq, off, qual, aln, cig, np.array(roff), lib.tail_params(max_report=0), pairing)
    lines = [b"read%d\tdesc\n" % i for i in range(len(reads))]
    names = b"".join(lines)
    name_off = np.concatenate([[0], np.cumsum([len(x) for x in lines])])
    chrom = [f"chr{t}" for t in range(len(g))]
    clen = [len(x) for x in g]
    text = b"@HD\tVN:1.6\tSO:unsorted\n" + b"".join(b"@SQ\tSN:%s\tLN:%d\n" % (c.encode(), n)
                                                   for c, n in zip(chrom, clen))
    head = lib.bam_header(text, chrom, clen)
    body = lib.bam_format(out, md, seq, off, qual, cig, names, name_off, len(g))
    f1 = lib.bgzf_compress(head, eof=False) + lib.bgzf_compress(body, n_threads=1)
    raw = gzip.decompress(f1)
    assert raw == head + body
    # several members (the records ten times over), compressed on one or
    # three threads alike, at every level
    big = body * 10
    z1 = lib.bgzf_compress(big, n_threads=1)
    assert z1 == lib.bgzf_compress(big, n_threads=3)
    members = _bgzf_members(z1)
    assert len(members) == -(-len(big) // 0xff00) + 1
    assert members[-1] == (b"\x03\x00", 0, 0)  # the end-of-file member
    for body_z, crc, isize in members[:-1]:
        plain = zlib.decompress(body_z, -15)
        assert len(plain) == isize <= 0xff00 and zlib.crc32(plain) == crc
    for level in (0, 1, 9):
        assert gzip.decompress(lib.bgzf_compress(big, level=level, n_threads=2)) == big
    assert lib.bgzf_compress(b"") == _EOF  # an empty input: the end-of-file member alone
    htext, refs, brecs = _bam_decode(raw)
    assert htext == text and refs == list(zip(chrom, clen))
    sam = lib.sam_format(out, md, seq, off, qual, cig, names, name_off, chrom).decode().rstrip("\n").split("\n")
    assert len(brecs) == len(out) == len(sam)
    for b, r, line in zip(brecs, out, sam):
        f = line.split("\t")
        assert b["name"] == f[0] and b["flag"] == int(f[1]) == r["flag"]
        assert (chrom[b["tid"]] if b["tid"] >= 0 else "*") == f[2]
        assert b["pos"] + 1 == int(f[3]) and b["mapq"] == int(f[4])
        assert ("".join(f"{c >> 4}{'MIDNSHP=XB'[c & 15]}" for c in b["cigar"]) or "*") == f[5]
        assert (b["ntid"], b["npos"], b["tlen"]) == (-1, 0, int(f[8])) and f[6:8] == ["*", "1"]
        assert "".join("=ACMGRSVTWYHKDBN"[x] for x in b["seq"]) == f[9]
        assert "".join(chr(x + 33) for x in b["qual"]) == f[10]
        rlen = sum(c >> 4 for c in b["cigar"] if c & 15 in (0, 2, 3, 7, 8))
        assert b["bin"] == _reg2bin(b["pos"], b["pos"] + rlen)
        if r["flag"] & 0x4:
            assert b["aux"] == []
            continue
        tags = [(t, v) for t, _, v in b["aux"]]
        assert tags == [("AS", int(r["as"])), ("MD", md[r["md_off"]:r["md_off"] + r["md_len"]].decode()),
                        ("XH", float(r["xh"])), ("NH", int(r["nh"])), ("XN", int(r["xn"])), ("XP", float(r["xp"]))]
        for t, typ, v in b["aux"]:
            if typ in "cCsSiI":  # the smallest integer type that holds the value
                fits = {"c": -128 <= v < 0, "C": 0 <= v <= 255, "s": -32768 <= v < -128, "S": 255 < v <= 65535,
                        "i": v < -32768, "I": v > 65535}
                assert fits[typ], (t, typ, v)
