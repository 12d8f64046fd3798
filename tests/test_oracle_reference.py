"""The oracle against the reference compiled from its own sources, on inputs
generated here rather than the committed fixtures: repeat-rich genomes,
reads with 3% substitutions and 1% indels, random reads, reads shorter than
the seed length, reads with N and reads at both ends of a chromosome, under
the default parameters, local mode, and a short seed length with no e-value
limit and a tight maxNSeed cut. SMEM lists, seeds and every alignment field
(window, coordinates, score, CIGAR, MD) must be equal."""
import os

import numpy as np
import pytest

from msgseqtk_b200 import index_build, synth
from oracle.bind import REF_SO, Oracle, Reference

needs_ref = pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref not built")

FIELDS = ("tid", "strand", "t_start", "t_end", "aln_from", "aln_to", "aln_start", "aln_end", "cigar", "md")


def _reads(g, seed):
    rng = np.random.default_rng(seed)
    a = synth.sample_reads(g, 60, seed=seed + 1, sub_rate=0.03, indel_rate=0.01)
    reads = [a.read(i) for i in range(len(a))]
    reads += [synth._BASES[rng.integers(0, 4, 150)] for _ in range(8)]  # random
    reads += [synth._BASES[rng.integers(0, 4, k)] for k in (1, 9, 16)]  # shorter than the seed length
    for i in range(6):  # N bases in true reads
        r = a.read(i).copy()
        r[rng.integers(0, len(r), 3)] = 15
        reads.append(r)
    for s in g[:2]:  # reads at both ends of a chromosome (windows reach past them)
        reads += [s[:120].copy(), s[-110:].copy()]
    return reads


@needs_ref
@pytest.mark.parametrize("ps", [dict(), dict(mode=1), dict(min_len=12, max_evalue=float("inf"), max_nseed=25)],
                         ids=["default", "local", "short-seeds"])
def test_oracle_equals_reference_on_fresh_reads(oracle_built, ps):
    g = synth.repeat_genomes(seed=61, n_genomes=3, length=25_000)
    view = index_build.build_view(g)
    ref = Reference(g, view=view)
    orc = Oracle(view)
    seed_ps = {k: v for k, v in ps.items() if k != "mode"}
    n_aln = 0
    for i, r in enumerate(_reads(g, 62)):
        assert np.array_equal(orc.smems(r, **{k: v for k, v in seed_ps.items() if k != "max_nseed"}),
                              ref.smems(r, **{k: v for k, v in seed_ps.items() if k != "max_nseed"})), i
        assert np.array_equal(orc.seeds(r, **seed_ps), ref.seeds(r, **seed_ps)), i
        got, exp = orc.align_read(r, **ps), ref.align_read(r, **ps)
        assert len(got) == len(exp), i
        for x, y in zip(got, exp):
            assert [x[k] for k in FIELDS] == [y[k] for k in FIELDS], i
            sx, sy = float(x["aln_score"]), float(y["aln_score"])
            assert sx == sy or (np.isinf(sx) and np.isinf(sy) and sx == sy), i
        n_aln += len(got)
    assert n_aln > 60
