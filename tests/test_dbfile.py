"""Reading msgseqtk-build's database files (msg_db_read): the reference writes
a DB with its own save functions; the decoded BWT, base counts, SA samples
and MetaGenome tables must equal the reference's in-memory index. Merged DBs
(msgseqtk-mergedb: BWT merge of two DBs, then buildSA) are read and mapped
the same way."""
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
@pytest.mark.parametrize("kind,n_threads", [("small", 4), ("repeats", 4), ("small", 1), ("repeats", 3),
                                            ("small", 7)])
def test_db_files_decode_to_reference_index(tmp_path, kind, n_threads):
    """Odd thread counts put the decode's chunk boundaries at uneven node
    splits; one thread decodes from row 0 with no boundary set-up."""
    if kind == "small":
        g = synth.small_genomes(seed=3, n_genomes=3, length=40_000)
    else:
        g = synth.repeat_genomes(seed=4, n_genomes=3, length=30_000)
    ref, paths = _write(tmp_path, g)
    db = lib.Database(*paths, n_threads=n_threads)
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


# .fmd layout up to the wavelet tree's occurrence table: program header
# (8-byte name, three int32 version fields), B[256] and C[256] as int64, then
# the tree's n, sigma, height, wid, min, max, sample_rate and the table size
# (FMDIndex::save, WaveletTreeRRR::save).
_OCC_AT = 20 + 2 * 256 * 8 + 8 * 8


@needs_ref
@pytest.mark.parametrize("entry,delta", [(8, 1000_000), (8, -1), (4, 3), (2, -2)])
def test_db_read_rejects_inconsistent_occurrence_table(tmp_path, entry, delta):
    """A corrupted occurrence-table entry of the BWT's wavelet tree moves a
    node's rows: the decode then leaves the node, reaches a symbol without an
    entry in the table, or the suffix-array walk meets counts that do not
    fit -- the file is rejected, never read out of bounds."""
    g = synth.small_genomes(seed=5, n_genomes=2, length=6_000)
    _, paths = _write(tmp_path, g)
    data = bytearray(open(paths[2], "rb").read())
    nocc = int(np.frombuffer(bytes(data[_OCC_AT - 8:_OCC_AT]), np.uint64)[0])
    occ = np.frombuffer(bytes(data[_OCC_AT:_OCC_AT + 8 * nocc]), np.uint64).copy()
    # the tree is built over nt16 codes 0..15 (FMDIndex.cpp:47): 17 entries,
    # cumulative, the last one the BWT's length
    assert nocc == 17 and occ[-1] == 2 * 2 * (6_000 + 1)
    occ[entry] = np.uint64(int(occ[entry]) + delta)
    data[_OCC_AT:_OCC_AT + 8 * nocc] = occ.tobytes()
    bad = tmp_path / "bad.fmd"
    open(bad, "wb").write(bytes(data))
    for n_threads in (1, 3):
        with pytest.raises(lib.MsgError) as e:
            lib.Database(paths[0], paths[1], bad, n_threads=n_threads)
        assert e.value.code == lib.MSG_EINVAL


def _same_arrays(a, b):
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


@needs_ref
def test_decoded_image_is_reused_and_rebuilt(tmp_path):
    """msg_db_read_cached: the first read decodes and writes the image, the
    next reads it back (same arrays as a plain decode, for any thread
    count); an image whose source files changed, whose body was altered or
    cut short, or of another format is ignored and written anew."""
    g = synth.repeat_genomes(seed=6, n_genomes=3, length=20_000)
    _, paths = _write(tmp_path, g)
    img = tmp_path / "db.fmd.b200"
    plain = lib.Database(*paths, n_threads=2)
    want = plain.arrays()
    plain.close()
    first = lib.Database(*paths, n_threads=3, image=img)
    assert first.from_image == 0 and img.exists()
    _same_arrays(first.arrays(), want)
    first.close()
    for nt in (1, 5):
        again = lib.Database(*paths, n_threads=nt, image=img)
        assert again.from_image == 1
        _same_arrays(again.arrays(), want)
        again.close()

    good = img.read_bytes()
    for damaged in (good[:-1], good[:len(good) // 2], good[:9] + bytes([good[9] ^ 1]) + good[10:],
                    good[:-200] + bytes([good[-200] ^ 0x40]) + good[-199:]):
        img.write_bytes(damaged)
        db = lib.Database(*paths, n_threads=2, image=img)
        assert db.from_image == 0
        _same_arrays(db.arrays(), want)
        db.close()
        assert img.read_bytes() == good

    # other source files at the same paths: a new key, the new database
    g2 = synth.small_genomes(seed=7, n_genomes=2, length=15_000)
    _, paths2 = _write(tmp_path, g2)
    assert paths2 == paths
    db = lib.Database(*paths, n_threads=2, image=img)
    assert db.from_image == 0
    a = db.arrays()
    assert np.array_equal(a["chr_seq"], np.concatenate(g2))
    db.close()
    db = lib.Database(*paths, n_threads=2, image=img)
    assert db.from_image == 1
    _same_arrays(db.arrays(), a)
    db.close()

    # an image path that cannot be written: decoded all the same
    db = lib.Database(*paths, n_threads=2, image=tmp_path / "missing_dir" / "x.b200")
    assert db.from_image == -1
    _same_arrays(db.arrays(), a)
    db.close()
    # unreadable source files are an error, as for msg_db_read
    with pytest.raises(lib.MsgError) as e:
        lib.Database(paths[0], paths[1], tmp_path / "missing.fmd", image=img)
    assert e.value.code == lib.MSG_EINVAL
    L = lib.load_library()
    assert L.msg_db_read_cached(None, None, None, None, 1, None, None) == lib.MSG_EINVAL


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("kind", ["small", "repeats", "merged"])
def test_device_decode_equals_host_decode(tmp_path, kind):
    """msg_db_read_device (BWT unranked, walked and listed by device
    kernels) gives msg_db_read's database: BWT, counts, sampled rows and
    values -- the last sample recomputed where the file lacks it -- and the
    MetaGenome tables."""
    if kind == "merged":
        _, _, paths = _merged(tmp_path)
    else:
        g = (synth.small_genomes(seed=3, n_genomes=3, length=40_000) if kind == "small"
             else synth.repeat_genomes(seed=4, n_genomes=3, length=30_000))
        _, paths = _write(tmp_path, g)
    host = lib.Database(*paths, n_threads=3)
    dev = lib.Database(*paths, device=0)
    _same_arrays(dev.arrays(), host.arrays())
    host.close()
    dev.close()


@pytest.mark.gpu
@needs_ref
def test_device_decode_rejects_what_host_rejects(tmp_path):
    g = synth.small_genomes(seed=5, n_genomes=2, length=6_000)
    _, paths = _write(tmp_path, g)
    data = open(paths[2], "rb").read()
    nocc = int(np.frombuffer(data[_OCC_AT - 8:_OCC_AT], np.uint64)[0])
    for entry, delta in [(8, 1000_000), (8, -1), (4, 3), (2, -2)]:
        occ = np.frombuffer(data[_OCC_AT:_OCC_AT + 8 * nocc], np.uint64).copy()
        occ[entry] = np.uint64(int(occ[entry]) + delta)
        bad = tmp_path / "bad.fmd"
        bad.write_bytes(data[:_OCC_AT] + occ.tobytes() + data[_OCC_AT + 8 * nocc:])
        with pytest.raises(lib.MsgError) as e:
            lib.Database(paths[0], paths[1], bad, device=0)
        assert e.value.code == lib.MSG_EINVAL, (entry, delta)
    (tmp_path / "cut.fmd").write_bytes(data[: len(data) // 2])
    with pytest.raises(lib.MsgError) as e:
        lib.Database(paths[0], paths[1], tmp_path / "cut.fmd", device=0)
    assert e.value.code == lib.MSG_EINVAL
    # a good file still decodes after the rejected ones
    dev = lib.Database(*paths, device=0)
    _same_arrays(dev.arrays(), lib.Database(*paths, n_threads=1).arrays())
    dev.close()


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


def _merged(tmp_path):
    ga = synth.small_genomes(seed=31, n_genomes=2, length=25_000)
    gb = synth.repeat_genomes(seed=32, n_genomes=2, length=20_000)
    ref = Reference.merged(ga, gb)
    paths = [tmp_path / "m.mtg", tmp_path / "m.mgs", tmp_path / "m.fmd"]
    ref.save(*paths)
    return ga + gb, ref, paths


@needs_ref
def test_merged_db_decodes_and_maps_like_reference(tmp_path, oracle_built):
    """A merged DB read from its files equals the reference's merged index,
    and the oracle on it aligns reads exactly as the reference does."""
    from oracle.bind import Oracle
    g, ref, paths = _merged(tmp_path)
    db = lib.Database(*paths, n_threads=4)
    a = db.arrays()
    assert np.array_equal(a["bwt"], ref.bwt())
    rows, vals = ref.sa_samples()
    assert np.array_equal(a["sample_rows"], rows) and np.array_equal(a["sample_vals"], vals)
    assert np.array_equal(a["chr_seq"], np.concatenate(g))
    view = db.view()
    orc = Oracle(view)
    rs = synth.sample_reads(g, 80, seed=33, sub_rate=0.02, indel_rate=0.005)
    for i in range(len(rs)):
        r = rs.read(i)
        assert np.array_equal(orc.smems(r), ref.smems(r))
        exp = ref.align_read(r)
        got = orc.align_read(r)
        assert [(e["tid"], e["strand"], e["aln_start"], int(e["aln_score"]), e["cigar"]) for e in got] == \
            [(e["tid"], e["strand"], e["aln_start"], int(e["aln_score"]), e["cigar"]) for e in exp]
    db.close()


@pytest.mark.gpu
@needs_ref
def test_gpu_maps_merged_db_like_oracle(tmp_path, oracle_built):
    from oracle.bind import Oracle
    g, ref, paths = _merged(tmp_path)
    db = lib.Database(*paths)
    orc = Oracle(db.view())
    rs = synth.sample_reads(g, 300, seed=34, sub_rate=0.02, indel_rate=0.005)
    c = lib.Context(0)
    try:
        c.load_database(db)
        res = c.map(rs.seqs, rs.offs)
        for i in range(len(rs)):
            got = res["aln"][res["read_aln_off"][i]:res["read_aln_off"][i + 1]]
            exp = orc.align_read(rs.read(i))
            assert [(int(x["tid"]), int(x["strand"]), int(x["aln_start"]), int(x["aln_score"])) for x in got] == \
                [(e["tid"], e["strand"], e["aln_start"], int(e["aln_score"])) for e in exp]
    finally:
        c.close()
        db.close()
