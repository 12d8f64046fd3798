"""Genomes holding N (runs of N and single N), which the reference indexes as
BWT symbol 15 (FMDIndex.cpp:118-133 rejects only IUPAC-extended codes):
the index view, the oracle and the CUDA path against the reference's own
code on the same genomes."""
import os

import numpy as np
import pytest

from msgseqtk_b200 import index_build, lib, synth
from oracle.bind import REF_SO, Oracle, Reference

needs_ref = pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref not built")


def n_genomes():
    g = [x.copy() for x in synth.small_genomes(seed=51, n_genomes=3, length=40_000)]
    g[0][5000:5200] = 15            # a run of N inside a chromosome
    g[0][:30] = 15                  # ... and at its start
    rng = np.random.default_rng(52)
    g[1][rng.integers(0, len(g[1]), 40)] = 15  # single N
    g[2][-700:] = 15                # a run at the end
    g[2][20000:21000] = 15
    return g


def n_reads(g):
    """Reads with errors from every genome (some over N runs or next to them),
    reads holding N, and reads that end inside an N run."""
    rs = synth.sample_reads(g, 600, seed=53, sub_rate=0.02, indel_rate=0.005)
    extra = [g[0][4900:5050].copy(), g[0][5150:5300].copy(), g[2][19880:20030].copy(), g[0][:150].copy(),
             g[2][-160:-10].copy(), g[1][1000:1150].copy()]
    extra[5][[10, 70, 71]] = 15
    seqs = [rs.read(i) for i in range(len(rs))] + extra
    seq = np.concatenate(seqs).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(x) for x in seqs])]).astype(np.int64)
    return seq, off, seqs


@needs_ref
def test_n_index_view_and_oracle_match_reference(oracle_built):
    g = n_genomes()
    ref = Reference(g)
    view = index_build.build_view(g)
    assert view.B[15] > 0
    assert np.array_equal(view.bwt, ref.bwt())
    B, _ = ref.counts()
    assert np.array_equal(view.B, B[:16])
    rows, vals = ref.sa_samples()
    assert np.array_equal(view.sample_rows, rows) and np.array_equal(view.sample_vals, vals)
    orc = Oracle(view)
    rng = np.random.default_rng(54)
    for i in rng.integers(0, view.n, 300):
        for b in (0, 1, 2, 4, 8, 15):
            assert orc.rank(b, int(i)) == ref.rank(b, int(i))
    _, _, seqs = n_reads(g)
    for r in seqs[::3] + seqs[-6:]:
        assert np.array_equal(orc.smems(r), ref.smems(r))
        got, exp = orc.align_read(r), ref.align_read(r)
        assert [(e["tid"], e["strand"], e["aln_start"], int(e["aln_score"]), e["cigar"]) for e in got] == \
            [(e["tid"], e["strand"], e["aln_start"], int(e["aln_score"]), e["cigar"]) for e in exp]


@needs_ref
def test_n_db_files_decode(tmp_path):
    g = n_genomes()
    ref = Reference(g)
    paths = [tmp_path / "n.mtg", tmp_path / "n.mgs", tmp_path / "n.fmd"]
    ref.save(*paths)
    db = lib.Database(*paths, n_threads=3)
    a = db.arrays()
    assert np.array_equal(a["bwt"], ref.bwt())
    assert np.array_equal(a["chr_seq"], np.concatenate(g))
    db.close()


@pytest.mark.gpu
def test_iupac_extended_bwt_is_rejected():
    """The reference refuses IUPAC-extended codes in the BWT; so does the
    loader (MSG_EINVAL), before any kernel reads them."""
    g = synth.small_genomes(seed=55, n_genomes=1, length=3000)
    view = index_build.build_view(g)
    i = int(np.nonzero(view.bwt == 1)[0][5])
    view.bwt = view.bwt.copy()
    view.bwt[i] = 5  # A/C ambiguity code
    view.B = view.B.copy()
    view.B[1] -= 1
    view.B[5] += 1
    c = lib.Context(0)
    try:
        with pytest.raises(lib.MsgError) as e:
            c.load_index(view)
        assert e.value.code == lib.MSG_EINVAL
    finally:
        c.close()


@pytest.mark.gpu
@needs_ref
def test_gpu_maps_n_genomes_like_reference(oracle_built):
    """occ (every symbol, N included), bi-interval extension, the recovered
    suffix array, SMEMs and alignments on genomes with N, against the
    reference's own code."""
    g = n_genomes()
    ref = Reference(g)
    view = index_build.build_view(g)
    orc = Oracle(view)
    c = lib.Context(0)
    try:
        c.load_index(view)
        n = view.n
        rng = np.random.default_rng(56)
        b = rng.choice(np.array([0, 1, 2, 4, 8, 15], dtype=np.uint8), size=3000)
        i = rng.integers(-1, n + 1, size=3000)
        got = c.occ(b, i)
        exp = [ref.rank(int(x), int(y)) if 0 <= y < n else -1 for x, y in zip(b, i)]
        assert np.array_equal(got, np.array(exp))
        rows = rng.integers(0, n, 2000)
        assert np.array_equal(c.sa(rows), np.array([ref.access_sa(int(r)) for r in rows]))
        sa_host = index_build.suffix_array(index_build.bd_text(g)).numpy()
        assert np.array_equal(c.sa(np.arange(n)), sa_host)
        # extensions from random intervals by every symbol, N included
        Cc = np.concatenate([[0], np.cumsum(view.B)])
        P, Q, S, Bs, E = [], [], [], [], []
        for k in range(600):
            base = int(rng.choice([1, 2, 4, 8]))
            p, q, s = int(Cc[base]), int(Cc[{1: 8, 2: 4, 4: 2, 8: 1}[base]]), int(Cc[base + 1] - Cc[base])
            nb = int(rng.choice([0, 1, 2, 4, 8, 15]))
            P.append(p); Q.append(q); S.append(s); Bs.append(nb)
            E.append(orc.back_ext(p, q, s, nb))
        ret, p2, q2, s2 = c.bi_ext(0, Bs, P, Q, S)
        for k, e in enumerate(E):
            assert (ret[k], p2[k], q2[k], s2[k]) == e, k
        seq, off, seqs = n_reads(g)
        res = c.map(seq, off, dump=True)
        for k, r in enumerate(seqs):
            sm = res["smem"][res["smem_off"][k]:res["smem_off"][k + 1]]
            assert np.array_equal(sm, ref.smems(r)), k
            got = res["aln"][res["read_aln_off"][k]:res["read_aln_off"][k + 1]]
            exp = ref.align_read(r)
            assert len(got) == len(exp), k
            for x, e in zip(got, exp):
                assert [int(x["tid"]), int(x["strand"]), int(x["t_start"]), int(x["t_end"]), int(x["aln_start"]),
                        int(x["aln_end"]), int(x["aln_score"])] == \
                    [e["tid"], e["strand"], e["t_start"], e["t_end"], e["aln_start"], e["aln_end"],
                     int(e["aln_score"])], k
                w = [int(v) for v in res["cigar"][x["cigar_off"]:x["cigar_off"] + x["n_cigar"]]]
                assert w == e["cigar"], k
    finally:
        c.close()
