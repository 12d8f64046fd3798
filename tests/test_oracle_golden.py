"""The CPU restatement (oracle) against the reference's own outputs committed
as fixtures (generated by tests/golden/make_golden.py from the reference
compiled from its sources)."""
import numpy as np
import pytest

from oracle.bind import Oracle


@pytest.mark.parametrize("name", ["uniform", "repeats"])
def test_oracle_matches_reference_fixtures(cases, oracle_built, name):
    c = cases[name]
    orc = Oracle(c.view)
    for k in range(c.n_params):
        ps = c.params(k)
        ex = c.expected(k)
        for i in range(len(c.read_off) - 1):
            r = c.read(i)
            sm = orc.smems(r, ps["min_len"], ps["max_evalue"])
            assert np.array_equal(sm, ex["smem"][ex["smem_off"][i]:ex["smem_off"][i + 1]]), (name, k, i)
            sd = orc.seeds(r, ps["min_len"], ps["max_evalue"], ps["max_nseed"])
            assert np.array_equal(sd, ex["seed"][ex["seed_off"][i]:ex["seed_off"][i + 1]]), (name, k, i)
            al = orc.align_read(r, ps["min_len"], ps["max_evalue"], ps["max_nseed"], ps["mode"])
            rows = ex["aln"][ex["aln_off"][i]:ex["aln_off"][i + 1]]
            assert len(al) == len(rows)
            for a, row, j in zip(al, rows, range(ex["aln_off"][i], ex["aln_off"][i + 1])):
                got = [a["tid"], a["strand"], a["t_start"], a["t_end"], a["aln_from"], a["aln_to"], a["aln_start"],
                       a["aln_end"], int(a["aln_score"])]
                assert got == list(row[:9]), (name, k, i)
                assert a["cigar"] == [int(x) for x in ex["cigar"][row[9]:row[9] + row[10]]]
                assert a["md"] == ex["md"][j]


def test_oracle_rank_and_extension_properties(cases, oracle_built):
    """occ/rank is a count over the BWT; backExt/fwdExt keep |fwd| == |rev|."""
    c = cases["uniform"]
    orc = Oracle(c.view)
    bwt = c.view.bwt
    rng = np.random.default_rng(5)
    for _ in range(300):
        b = int(rng.choice([0, 1, 2, 4, 8]))
        i = int(rng.integers(0, len(bwt)))
        assert orc.rank(b, i) == int(np.count_nonzero(bwt[:i + 1] == b))
    assert orc.rank(1, len(bwt)) == -1
