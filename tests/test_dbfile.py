"""Reading msgseqtk-build's database files (msg_db_read): the reference writes
a DB with its own save functions; the decoded BWT, base counts, SA samples
and MetaGenome tables must equal the reference's in-memory index."""
import os

import numpy as np
import pytest

from msgseqtk_b200 import lib, synth
from oracle.bind import REF_SO, Reference

needs_ref = pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref not built")


def _write(tmp_path, genomes):
    ref = Reference(genomes)
    paths = [tmp_path / "db.mtg", tmp_path / "db.mgs", tmp_path / "db.fmd"]
    ref.save(*paths)
    return ref, paths


@needs_ref
@pytest.mark.parametrize("kind", ["small", "repeats"])
def test_db_files_decode_to_reference_index(tmp_path, kind):
    if kind == "small":
        g = synth.small_genomes(seed=3, n_genomes=3, length=40_000)
    else:
        g = synth.repeat_genomes(seed=4, n_genomes=3, length=30_000)
    ref, paths = _write(tmp_path, g)
    db = lib.Database(*paths, n_threads=4)
    a = db.arrays()
    assert np.array_equal(a["bwt"], ref.bwt())
    B, _ = ref.counts()
    assert np.array_equal(a["B"], B[:16])
    rows, vals = ref.sa_samples()
    assert np.array_equal(a["sample_rows"], rows)
    assert np.array_equal(a["sample_vals"], vals)
    starts, ends, lens = ref.chroms()
    assert np.array_equal(a["bd_start"], starts) and np.array_equal(a["bd_end"], ends)
    assert np.array_equal(a["chr_len"], np.array([len(x) for x in g]))
    assert np.array_equal(a["chr_seq"], np.concatenate(g))
    db.close()


@needs_ref
def test_db_read_rejects_bad_files(tmp_path):
    g = synth.small_genomes(seed=5, n_genomes=1, length=5_000)
    _, paths = _write(tmp_path, g)
    bad = tmp_path / "bad.fmd"
    data = open(paths[2], "rb").read()
    open(bad, "wb").write(data[: len(data) // 2])  # truncated
    with pytest.raises(lib.MsgError) as e:
        lib.Database(paths[0], paths[1], bad)
    assert e.value.code == lib.MSG_EINVAL
    with pytest.raises(lib.MsgError):
        lib.Database(paths[0], paths[1], tmp_path / "missing.fmd")


@pytest.mark.gpu
@needs_ref
def test_index_from_db_files_maps_like_view(tmp_path):
    from msgseqtk_b200 import index_build
    g = synth.repeat_genomes(seed=4, n_genomes=3, length=30_000)
    _, paths = _write(tmp_path, g)
    db = lib.Database(*paths)
    rs = synth.sample_reads(g, 400, seed=9)
    c = lib.Context(0)
    try:
        c.load_database(db)
        a = c.map(rs.seqs, rs.offs)
        c.load_index(index_build.build_view(g))
        b = c.map(rs.seqs, rs.offs)
        for k in ("aln", "cigar", "read_aln_off"):
            assert np.array_equal(a[k], b[k]), k
        assert len(a["aln"]) > 0
    finally:
        c.close()
        db.close()
