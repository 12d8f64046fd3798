"""SAM records: alignment records fed through the reference's own tail
(filter, evaluate, calcMapQ, sort, exportBAM and msgseqtk-align's per-read
output) must give the same SAM fields as the reference's whole single-end
path, and the library's own host tail (msg_tail_batch) must give the same
fields as the reference's tail. On the CPU the records come from the oracle;
on the GPU (-m gpu) from the CUDA library through the C ABI."""
import os

import numpy as np
import pytest

from msgseqtk_b200 import lib, synth
from oracle.bind import REF_SO, Oracle, Reference
from oracle.sam_fields import ours_as_fields as _ours_as_fields, ref_as_fields as _ref_as_fields

needs_ref = pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref not built")


def _records_from_oracle(orc, reads, mode=0):
    recs, cig, roff = [], [], [0]
    for i, r in enumerate(reads):
        for e in orc.align_read(r, mode=mode):
            recs.append((i, e["tid"], e["strand"], e["t_start"], e["t_end"], e["aln_from"], e["aln_to"],
                         e["aln_start"], e["aln_end"],
                         int(e["aln_score"]) if np.isfinite(e["aln_score"]) else -(2 ** 31), e["flags"], len(cig),
                         len(e["cigar"]), 0))
            cig += e["cigar"]
        roff.append(len(recs))
    return (np.array(recs, dtype=lib.ALN_DTYPE), np.array(cig, dtype=np.uint32), np.array(roff, dtype=np.int64))


def _workload(seed):
    g = synth.small_genomes(seed=seed, n_genomes=3, length=60_000)
    a = synth.sample_reads(g, 300, seed=seed + 1)
    b = synth.sample_reads(g, 100, seed=seed + 2, sub_rate=0.05, indel_rate=0.01)
    reads = [a.read(i) for i in range(len(a))] + [b.read(i) for i in range(len(b))]
    quals = [a.qual(i) for i in range(len(a))] + [b.qual(i) for i in range(len(b))]
    rng = np.random.default_rng(seed)
    reads += [synth._BASES[rng.integers(0, 4, 150)] for _ in range(40)]
    quals += [rng.integers(20, 41, 150).astype(np.uint8) for _ in range(40)]
    seq = np.concatenate(reads).astype(np.uint8)
    qual = np.concatenate(quals).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(x) for x in reads])]).astype(np.int64)
    return g, reads, seq, qual, off


def _check_tail(view, ref, seq, qual, off, aln, cig, roff, rate, max_report):
    from msgseqtk_b200 import lib
    exp = _ref_as_fields(ref.sam_from_records(seq, qual, off, aln, cig, roff, min_score_rate=rate,
                                              max_report=max_report))
    for nt in (1, 3):
        recs, md = lib.tail(view, seq, off, qual, aln, cig, roff,
                            lib.tail_params(min_score_rate=rate, max_report=max_report, n_threads=nt))
        got = _ours_as_fields(recs, md, seq, qual, off, cig)
        assert len(got) == len(exp)
        for g, e in zip(got, exp):
            assert g == e, (g, e)


def _check_tail_pe(view, ref, seq, qual, off, aln, cig, roff, rate, max_report, pairing):
    from msgseqtk_b200 import lib
    exp = _ref_as_fields(ref.sam_pe_from_records(seq, qual, off, aln, cig, roff, min_score_rate=rate,
                                                 max_report=max_report, pairing=pairing))
    q = {"min_ins" if k == "min" else "max_ins" if k == "max" else k: v for k, v in pairing.items()}
    for nt in (1, 3):
        recs, md = lib.tail(view, seq, off, qual, aln, cig, roff,
                            lib.tail_params(min_score_rate=rate, max_report=max_report, n_threads=nt),
                            pairing=lib.pair_params(**q))
        got = _ours_as_fields(recs, md, seq, qual, off, cig, pairs=True)
        assert len(got) == len(exp)
        for g, e in zip(got, exp):
            assert g == e, (g, e)
    return exp


def _pair_workload(seed):
    """Pairs (mates at 2i, 2i+1): proper pairs, pairs with wide inserts,
    pairs with one random mate, random pairs."""
    g = synth.small_genomes(seed=seed, n_genomes=3, length=60_000)
    m1, m2 = synth.sample_pairs(g, 200, seed=seed + 1, ins_mean=400, ins_sd=50)
    w1, w2 = synth.sample_pairs(g, 40, seed=seed + 2, ins_mean=900, ins_sd=200, sub_rate=0.04, indel_rate=0.01)
    rng = np.random.default_rng(seed)
    mates, quals = [], []
    for a, b in ((m1, m2), (w1, w2)):
        for i in range(len(a)):
            mates += [a.read(i), b.read(i)]
            quals += [a.qual(i), b.qual(i)]
    for i in range(30):  # one mate random
        mates += [m1.read(i), synth._BASES[rng.integers(0, 4, 150)]]
        quals += [m1.qual(i), rng.integers(20, 41, 150).astype(np.uint8)]
    for i in range(20):
        mates += [synth._BASES[rng.integers(0, 4, 150)] for _ in range(2)]
        quals += [rng.integers(20, 41, 150).astype(np.uint8) for _ in range(2)]
    seq = np.concatenate(mates).astype(np.uint8)
    qual = np.concatenate(quals).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(x) for x in mates])]).astype(np.int64)
    return g, mates, seq, qual, off


PAIRINGS = [dict(), dict(mean=400.0, sd=50.0, min=-100.0, max=900.0),
            dict(mean=400.0, sd=50.0, min=-100.0, max=900.0, no_mixed=1, max_npair=2),
            dict(mean=0.0, sd=1.0, min=0.0, max=2000.0, no_overlap=1, no_contain=1)]


@needs_ref
def test_library_pe_tail_matches_reference_on_oracle_records(oracle_built):
    """msg_tail_pe_batch against the reference's paired-end tail
    (AlignmentPE pairing, filters, MAPQ, unpaired and unmapped fallbacks) on
    the same records, and those records through the reference's tail against
    its whole paired-end path."""
    from msgseqtk_b200 import index_build
    g, mates, seq, qual, off = _pair_workload(21)
    ref = Reference(g)
    view = index_build.build_view(g)
    aln, cig, roff = _records_from_oracle(Oracle(view), mates)
    kinds = set()
    for pairing in PAIRINGS:
        for rate, max_report in ((0.65, 1), (0.65, 0), (0.3, 2)):
            exp = _check_tail_pe(view, ref, seq, qual, off, aln, cig, roff, rate, max_report, pairing)
            kinds |= {int(e[1]) & 0x1cf for e in exp}
            if rate == 0.65:
                full = ref.sam_pe_batch(seq, qual, off, min_score_rate=rate, max_report=max_report, pairing=pairing)
                assert _ref_as_fields(full) == exp
    # proper pairs, unpaired mates and unmapped pairs all occur
    assert {0x43, 0x83} & kinds and {0x41, 0x81} & kinds and {77, 141} <= kinds


@needs_ref
def test_library_tail_matches_reference_tail_on_oracle_records(oracle_built):
    """msg_tail_batch (host C++ in the library) against the reference's own
    filter/evaluate/calcMapQ/sort/output on the same records: every field,
    float tags to the bit."""
    from msgseqtk_b200 import index_build
    g, reads, seq, qual, off = _workload(9)
    ref = Reference(g)
    view = index_build.build_view(g)
    orc = Oracle(view)
    aln, cig, roff = _records_from_oracle(orc, reads)
    for rate, max_report in ((0.65, 1), (0.65, 0), (0.3, 3), (-1.0, 0)):
        _check_tail(view, ref, seq, qual, off, aln, cig, roff, rate, max_report)
    # reads without qualities read 33 on every base (PrimarySeq::fixQual)
    q33 = np.full_like(qual, 33)
    a, ma = lib.tail(view, seq, off, None, aln, cig, roff)
    b, mb = lib.tail(view, seq, off, q33, aln, cig, roff)
    assert np.array_equal(a, b) and ma == mb
    # local (Smith-Waterman) records: soft clips and evaluate's clip penalty
    aln, cig, roff = _records_from_oracle(orc, reads, mode=1)
    assert any((c & 0xf) == 4 for c in cig)
    for rate, max_report in ((0.65, 1), (0.2, 0)):
        _check_tail(view, ref, seq, qual, off, aln, cig, roff, rate, max_report)


@needs_ref
def test_tail_on_oracle_records_matches_reference(oracle_built):
    from msgseqtk_b200 import index_build
    g, reads, seq, qual, off = _workload(5)
    ref = Reference(g)
    orc = Oracle(index_build.build_view(g))
    aln, cig, roff = _records_from_oracle(orc, reads)
    for max_report in (1, 0):
        exp = ref.sam_batch(seq, qual, off, max_report=max_report)
        got = ref.sam_from_records(seq, qual, off, aln, cig, roff, max_report=max_report)
        assert got == exp


@pytest.mark.gpu
@needs_ref
def test_gpu_records_give_reference_sam():
    from msgseqtk_b200 import index_build
    g, reads, seq, qual, off = _workload(7)
    ref = Reference(g)
    view = index_build.build_view(g)
    ctx = lib.Context(0)
    try:
        ctx.load_index(view)
        for params in (lib.default_params(min_score_rate=0.65), lib.default_params(),
                       lib.default_params(min_score_rate=0.65, band_mode=1, band_w=7)):
            res = ctx.map(seq, off, params)
            for max_report in (1, 0):
                exp = ref.sam_batch(seq, qual, off, max_report=max_report)
                got = ref.sam_from_records(seq, qual, off, res["aln"], res["cigar"], res["read_aln_off"],
                                           max_report=max_report)
                assert got == exp
                _check_tail(view, ref, seq, qual, off, res["aln"], res["cigar"], res["read_aln_off"], 0.65,
                            max_report)
    finally:
        ctx.close()


@pytest.mark.gpu
@needs_ref
def test_gpu_records_through_library_pe_tail_give_reference_pairs():
    """GPU records of interleaved mates through msg_tail_pe_batch equal the
    reference's whole paired-end path."""
    from msgseqtk_b200 import index_build
    g, mates, seq, qual, off = _pair_workload(23)
    ref = Reference(g)
    view = index_build.build_view(g)
    ctx = lib.Context(0)
    try:
        ctx.load_index(view)
        res = ctx.map(seq, off, lib.default_params(min_score_rate=0.65))
        for pairing in PAIRINGS[:2]:
            for max_report in (1, 0):
                full = _ref_as_fields(ref.sam_pe_batch(seq, qual, off, max_report=max_report, pairing=pairing))
                got = _check_tail_pe(view, ref, seq, qual, off, res["aln"], res["cigar"], res["read_aln_off"], 0.65,
                                     max_report, pairing)
                assert got == full
    finally:
        ctx.close()


@pytest.mark.gpu
@needs_ref
def test_small_config_sam_matches_reference():
    """The small configuration at its exact shape: 4 genomes of 500 kbp
    (i.i.d. uniform bases), 10,000 single-end 150 bp reads (1% substitutions,
    0.1% indels of 1-3 bp, Phred 20-40), default scores, GLOBAL mode, -k 1.
    The GPU records through the reference's own tail and through the
    library's tail give the SAM fields of the reference's whole single-end
    path, read for read."""
    from msgseqtk_b200 import index_build
    g = synth.small_genomes(seed=101, n_genomes=4, length=500_000)
    rs = synth.sample_reads(g, 10_000, seed=102)
    seq = rs.seqs.astype(np.uint8)
    off = rs.offs.astype(np.int64)
    qual = np.concatenate([rs.qual(i) for i in range(len(rs))]).astype(np.uint8)
    ref = Reference(g)
    view = index_build.build_view(g)
    ctx = lib.Context(0)
    try:
        ctx.load_index(view)
        res = ctx.map(seq, off, lib.default_params(min_score_rate=0.65))
        exp = ref.sam_batch(seq, qual, off, max_report=1)
        got = ref.sam_from_records(seq, qual, off, res["aln"], res["cigar"], res["read_aln_off"], max_report=1)
        assert got == exp
        _check_tail(view, ref, seq, qual, off, res["aln"], res["cigar"], res["read_aln_off"], 0.65, 1)
        assert len(res["aln"]) > 9_000
    finally:
        ctx.close()
