"""The mapping task one stage at a time through the C ABI
(msg_seed_batch -> msg_locate_batch -> msg_chain_batch -> msg_align_batch):
every stage equals the fused msg_map_batch, the chain stage equals the
reference's own SeedChain::getChains on the same seeds, and caller arrays
that would make a kernel read outside the index, a read or a seed list are
rejected."""
import math
import os

import numpy as np
import pytest

from msgseqtk_b200 import index_build, lib, synth
from oracle.bind import REF_SO, Reference

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not os.path.exists(REF_SO), reason="oracle/_ref not built")


def workload():
    g = synth.repeat_genomes(seed=91, n_genomes=2, length=30_000) + synth.small_genomes(seed=92, n_genomes=2,
                                                                                       length=40_000)
    rs = synth.sample_reads(g, 400, seed=93, sub_rate=0.03, indel_rate=0.01)
    rng = np.random.default_rng(94)
    rand = synth._BASES[rng.integers(0, 4, 150 * 20)]
    seq = np.concatenate([rs.seqs, rand]).astype(np.uint8)
    off = np.concatenate([rs.offs, rs.offs[-1] + 150 * np.arange(1, 21)]).astype(np.int64)
    return g, seq, off


@needs_ref
def test_stages_equal_fused_mapping():
    g, seq, off = workload()
    view = index_build.build_view(g)
    ref = Reference(g)
    c = lib.Context(0)
    try:
        c.load_index(view)
        # every SMEM selected (no maxNSeed cut), so the caller's selection is the whole list
        params = lib.default_params(max_nseed=1 << 40)
        full = c.map(seq, off, params, dump=True)
        smem, soff = c.seed_batch(seq, off, params)
        assert np.array_equal(smem, full["smem"]) and np.array_equal(soff, full["smem_off"])
        seeds, sdo = c.locate_batch(seq, off, smem, soff)
        assert np.array_equal(seeds, full["seed"]) and np.array_equal(sdo, full["seed_off"])
        cs, cso, rco = c.chain_batch(seq, off, seeds, sdo)
        n_chains = 0
        for r in range(len(off) - 1):
            L = int(off[r + 1] - off[r])
            mine = [cs[cso[k]:cso[k + 1]].tolist() for k in range(rco[r], rco[r + 1])]
            exp = ref.chains(seeds[sdo[r]:sdo[r + 1]], math.ceil(L * 0.2), math.ceil(L * 0.1))
            assert mine == [e.tolist() for e in exp], r
            n_chains += len(mine)
        assert n_chains == len(full["aln"]) > 0
        for prm in (params, lib.default_params(max_nseed=1 << 40, mode=1),
                    lib.default_params(max_nseed=1 << 40, min_score_rate=0.65, band_mode=1, band_w=15)):
            exp = c.map(seq, off, prm)
            got = c.align_batch(seq, off, seeds, sdo, cs, cso, rco, prm)
            for k in ("aln", "cigar", "read_aln_off"):
                assert np.array_equal(got[k], exp[k]), k
        # default maxNSeed: the fused call's own selection, fed back through the stages
        dflt = lib.default_params()
        full = c.map(seq, off, dflt, dump=True)
        cs, cso, rco = c.chain_batch(seq, off, full["seed"], full["seed_off"])
        got = c.align_batch(seq, off, full["seed"], full["seed_off"], cs, cso, rco, dflt)
        for k in ("aln", "cigar", "read_aln_off"):
            assert np.array_equal(got[k], full[k]), k
    finally:
        c.close()


def test_stage_inputs_are_checked():
    g, seq, off = workload()
    view = index_build.build_view(g)
    c = lib.Context(0)
    try:
        c.load_index(view)
        smem, soff = c.seed_batch(seq, off)
        bad = smem.copy()
        bad[0, 2] = view.n  # suffix-array rows past the index
        with pytest.raises(lib.MsgError) as e:
            c.locate_batch(seq, off, bad, soff)
        assert e.value.code == lib.MSG_EINVAL
        bad = smem.copy()
        bad[0, 1] = 10_000  # past the read
        with pytest.raises(lib.MsgError) as e:
            c.locate_batch(seq, off, bad, soff)
        assert e.value.code == lib.MSG_EINVAL
        seeds, sdo = c.locate_batch(seq, off, smem, soff)
        cs, cso, rco = c.chain_batch(seq, off, seeds, sdo)
        bad_cs = cs.copy()
        bad_cs[0] = 1 << 20  # not a seed of the read
        with pytest.raises(lib.MsgError) as e:
            c.align_batch(seq, off, seeds, sdo, bad_cs, cso, rco)
        assert e.value.code == lib.MSG_EINVAL
        bad_seeds = seeds.copy()
        bad_seeds[0, 4] = len(g)  # no such chromosome
        with pytest.raises(lib.MsgError) as e:
            c.chain_batch(seq, off, bad_seeds, sdo)
        assert e.value.code == lib.MSG_EINVAL
        # the context keeps working
        got = c.align_batch(seq, off, seeds, sdo, cs, cso, rco)
        assert len(got["aln"]) == len(cso) - 1
    finally:
        c.close()
