"""msgseqtk-clean's path: SMEM_LIST::findMEMS per read against a reference
and a background index, the lists' loglik and the log-odds decision.

On the CPU the oracle is checked against the reference's outputs committed in
tests/golden/clean.npz (made by tests/golden/make_golden.py from the reference
compiled from its sources). On the GPU (-m gpu) the CUDA library is checked,
through the C ABI, against the same fixture and against the oracle on
workloads the fixture does not hold (long reads, more reads). Every number is
compared bit for bit: -inf log-likelihoods (N in a read) and NaN log-odds
included.
"""
import os

import numpy as np
import pytest

from msgseqtk_b200 import index_build, lib, synth
from oracle.bind import REF_SO, Oracle, Reference

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "clean.npz")


def _split(flat, off):
    return [flat[off[k]:off[k + 1]] for k in range(len(off) - 1)]


def _bits(x):
    return np.ascontiguousarray(x, dtype=np.float64).view(np.int64)


@pytest.fixture(scope="module")
def fx():
    d = np.load(GOLDEN)
    g_ref = _split(d["ref_genome"], d["ref_genome_off"])
    g_bg = _split(d["bg_genome"], d["bg_genome_off"])
    return d, index_build.build_view(g_ref), index_build.build_view(g_bg), g_ref, g_bg


def _clean_from_lls(ll_ref, ll_bg, ll_ref2, ll_bg2, min_lod):
    """msgseqtk-clean.cpp:430-433 (pairs: :467-470) in double arithmetic."""
    r = np.array([a + b for a, b in zip(ll_ref, ll_ref2)]) if ll_ref2 is not None else np.array(ll_ref)
    g = np.array([a + b for a, b in zip(ll_bg, ll_bg2)]) if ll_bg2 is not None else np.array(ll_bg)
    with np.errstate(invalid="ignore"):  # -inf + inf: NaN, as in the reference
        lod = -r + g
    return r, g, lod, lod > min_lod


def test_oracle_mems_and_clean_match_reference_fixture(fx, oracle_built):
    d, v_ref, v_bg, _, _ = fx
    o_ref, o_bg = Oracle(v_ref), Oracle(v_bg)
    reads, mates = _split(d["reads"], d["read_off"]), _split(d["mates"], d["mate_off"])
    for k, (ml, me) in enumerate(d["params"]):
        ml = int(ml)
        lls = {}
        for name, orc in (("ref", o_ref), ("bg", o_bg)):
            lls[name] = [orc.mems(r, ml, me)[1] for r in reads]
            lls[name + "2"] = [orc.mems(r, ml, me)[1] for r in mates]
        for i, r in enumerate(reads):
            rows, ll = o_ref.mems(r, ml, me)
            off = d[f"p{k}_mem_off"]
            assert np.array_equal(rows, d[f"p{k}_mem"][off[i]:off[i + 1]]), (k, i)
            assert _bits([ll]) == _bits(d[f"p{k}_mem_ll"][i:i + 1]), (k, i)
        for j, lod in enumerate(d["lods"]):
            for tag, pe in (("se", False), ("pe", True)):
                r, g, lo, keep = _clean_from_lls(lls["ref"], lls["bg"], lls["ref2"] if pe else None,
                                                 lls["bg2"] if pe else None, lod)
                ex = d[f"p{k}_l{j}_{tag}"]
                assert np.array_equal(_bits(np.stack([r, g, lo])), _bits(ex)), (k, j, tag)
                assert np.array_equal(keep, d[f"p{k}_l{j}_{tag}_keep"]), (k, j, tag)


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref not built")
def test_oracle_mems_match_reference_on_repeats(oracle_built):
    """Repeat-rich genomes (large intervals, long matches) and errorful reads."""
    g = synth.repeat_genomes(seed=31, n_genomes=2, length=15000)
    ref, orc = Reference(g), Oracle(index_build.build_view(g))
    rs = synth.sample_reads(g, 150, seed=32, sub_rate=0.04, indel_rate=0.01)
    for i in range(len(rs)):
        for ml, me in ((17, 0.01), (4, 1e6), (1, float("inf"))):
            a, la = ref.mems(rs.read(i), ml, me)
            b, lb = orc.mems(rs.read(i), ml, me)
            assert np.array_equal(a, b) and _bits([la]) == _bits([lb])


# ---------------------------------------------------------------- GPU ----

def _contexts(v_ref, v_bg):
    a, b = lib.Context(0), lib.Context(0)
    a.load_index(v_ref)
    b.load_index(v_bg)
    return a, b


@pytest.mark.gpu
def test_gpu_mems_match_reference_fixture(fx):
    d, v_ref, v_bg, _, _ = fx
    a, b = _contexts(v_ref, v_bg)
    try:
        for k, (ml, me) in enumerate(d["params"]):
            p = lib.mem_params(min_len=int(ml), max_evalue=float(me))
            ll, cnt, rows = a.mems(d["reads"], d["read_off"], p)
            assert np.array_equal(rows, d[f"p{k}_mem"]), k
            assert np.array_equal(np.diff(d[f"p{k}_mem_off"]), cnt), k
            assert np.array_equal(_bits(ll), _bits(d[f"p{k}_mem_ll"])), k
            ll2, cnt2, none = a.mems(d["reads"], d["read_off"], p, rows=False)
            assert none is None and np.array_equal(_bits(ll2), _bits(ll)) and np.array_equal(cnt2, cnt)
            st = a.stats()
            assert st["n_smem"] == len(rows) and st["n_ext"] > 0 and st["n_launch"] >= 1
    finally:
        a.close()
        b.close()


@pytest.mark.gpu
def test_gpu_clean_matches_reference_fixture(fx):
    d, v_ref, v_bg, _, _ = fx
    a, b = _contexts(v_ref, v_bg)
    try:
        for k, (ml, me) in enumerate(d["params"]):
            p = lib.mem_params(min_len=int(ml), max_evalue=float(me))
            for j, lod in enumerate(d["lods"]):
                for tag, pe in (("se", False), ("pe", True)):
                    res = a.clean(b, d["reads"], d["read_off"], d["mates"] if pe else None,
                                  d["mate_off"] if pe else None, params=p, min_lod=float(lod))
                    assert np.array_equal(_bits(np.stack(res[:3])), _bits(d[f"p{k}_l{j}_{tag}"])), (k, j, tag)
                    assert np.array_equal(res[3], d[f"p{k}_l{j}_{tag}_keep"]), (k, j, tag)
    finally:
        a.close()
        b.close()


@pytest.mark.gpu
def test_gpu_clean_device_reads_and_long_reads_match_oracle(fx):
    """Reads of 1-6 kbp and a larger batch, against the oracle; the
    device-pointer entry point gives the host one's results."""
    import torch
    d, v_ref, v_bg, g_ref, g_bg = fx
    rng = np.random.default_rng(77)
    reads = []
    for gs in (g_ref, g_bg):
        rs = synth.sample_reads(gs, 400, seed=int(rng.integers(1 << 30)), sub_rate=0.01, indel_rate=0.002)
        reads += [rs.read(i) for i in range(len(rs))]
    for _ in range(40):  # long reads cut from the genomes with 2% substitutions
        gs = g_ref if rng.random() < 0.5 else g_bg
        c = gs[int(rng.integers(len(gs)))]
        L = int(rng.integers(1000, 6000))
        s = int(rng.integers(0, len(c) - L))
        r = c[s:s + L].copy()
        m = rng.random(L) < 0.02
        r[m] = synth._BASES[rng.integers(0, 4, int(m.sum()))]
        reads.append(r)
    off = np.cumsum([0] + [len(r) for r in reads]).astype(np.int64)
    seq = np.concatenate(reads).astype(np.uint8)
    o_ref, o_bg = Oracle(v_ref), Oracle(v_bg)
    exp_ref = np.array([o_ref.mems(r)[1] for r in reads])
    exp_bg = np.array([o_bg.mems(r)[1] for r in reads])
    a, b = _contexts(v_ref, v_bg)
    try:
        r, g, lod, keep = a.clean(b, seq, off)
        assert np.array_equal(_bits(r), _bits(exp_ref)) and np.array_equal(_bits(g), _bits(exp_bg))
        with np.errstate(invalid="ignore"):
            assert np.array_equal(keep, (-exp_ref + exp_bg) > 0)
        d_seq = torch.from_numpy(seq).cuda()
        d_off = torch.from_numpy(off).cuda()
        r2, g2, lod2, keep2 = a.clean_device(b, d_seq.data_ptr(), d_off.data_ptr(), len(off) - 1)
        torch.cuda.synchronize()
        assert np.array_equal(_bits(np.stack([r, g, lod])), _bits(np.stack([r2, g2, lod2])))
        assert np.array_equal(keep, keep2)
        # the same context keeps mapping correctly after MEM calls
        ll, cnt, rows = a.mems(seq, off)
        assert np.array_equal(_bits(ll), _bits(exp_ref))
    finally:
        a.close()
        b.close()


@pytest.mark.gpu
def test_gpu_clean_rejects_bad_arguments(fx):
    d, v_ref, v_bg, _, _ = fx
    a, b = _contexts(v_ref, v_bg)
    empty = lib.Context(0)
    try:
        with pytest.raises(lib.MsgError) as e:
            a.clean(a, d["reads"], d["read_off"])
        assert e.value.code == lib.MSG_EINVAL
        with pytest.raises(lib.MsgError) as e:
            a.clean(empty, d["reads"], d["read_off"])
        assert e.value.code == lib.MSG_ESTATE
        with pytest.raises(lib.MsgError) as e:
            a.clean(b, d["reads"], d["read_off"], d["mates"], d["mate_off"][:10])
        assert e.value.code == lib.MSG_EINVAL
        with pytest.raises(lib.MsgError) as e:
            a.mems(d["reads"], d["read_off"], lib.mem_params(max_evalue=-1.0))
        assert e.value.code == lib.MSG_EINVAL
        ll, cnt, rows = a.mems(np.zeros(0, np.uint8), np.zeros(1, np.int64))
        assert len(ll) == 0 and len(rows) == 0
        with pytest.raises(lib.MsgError) as e:  # ASCII instead of nt16 codes
            a.clean(b, np.frombuffer(b"ACGTACGT", np.uint8), np.array([0, 8], np.int64))
        assert e.value.code == lib.MSG_EINVAL
    finally:
        for c in (a, b, empty):
            c.close()
