"""Contexts sharing one loaded index (msg_ctx_share_index), as the
reference's OpenMP mapping tasks share one FMDIndex and MetaGenome: a
sharer's records equal the owner's; batches mapped side by side, one host
thread per context, equal the same batches mapped one after another; the
index stays usable by sharers after its owner is destroyed, and a sharer
that loads its own index leaves the others alone."""
import threading

import numpy as np
import pytest

from msgseqtk_b200 import index_build, lib, synth

pytestmark = pytest.mark.gpu


def same(got, exp):
    assert np.array_equal(got["read_aln_off"], exp["read_aln_off"])
    assert np.array_equal(got["aln"], exp["aln"])
    assert np.array_equal(got["cigar"], exp["cigar"])


def test_shared_index_contexts_map_alike():
    g = synth.small_genomes(seed=91, n_genomes=3, length=80_000)
    view = index_build.build_view(g)
    owner = lib.Context(0)
    sharers = []
    try:
        # nothing to share yet, and a context cannot share with itself
        probe = lib.Context(0)
        sharers.append(probe)
        with pytest.raises(lib.MsgError) as e:
            probe.share_index(owner)
        assert e.value.code == lib.MSG_ESTATE
        owner.load_index(view)
        with pytest.raises(lib.MsgError) as e:
            owner.share_index(owner)
        assert e.value.code == lib.MSG_EINVAL

        rs = synth.sample_reads(g, 2000, seed=92, sub_rate=0.02, indel_rate=0.005)
        params = lib.default_params(min_score_rate=0.65)
        cuts = [0, 500, 1000, 1500, 2000]
        batches = [(rs.seqs[rs.offs[a]:rs.offs[b]], np.ascontiguousarray(rs.offs[a:b + 1] - rs.offs[a]))
                   for a, b in zip(cuts[:-1], cuts[1:])]
        expect = [owner.map(s, o, params) for s, o in batches]
        assert sum(len(x["aln"]) for x in expect) > 1000

        sharers += [lib.Context(0) for _ in range(2)]
        for c in sharers:
            c.share_index(owner)
            assert c.index_bytes() == owner.index_bytes()
        same(sharers[0].map(*batches[1], params), expect[1])

        # side by side: one host thread per context, each mapping its own
        # batch three times while the others run
        ctxs = [owner] + sharers
        results, errors = {}, []

        def work(k):
            try:
                for rep in range(3):
                    results[(k, rep)] = ctxs[k].map(*batches[k], params)
            except Exception as exc:  # reported below
                errors.append(exc)

        threads = [threading.Thread(target=work, args=(k,)) for k in range(len(ctxs))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        assert not errors, errors
        for (k, rep), got in results.items():
            same(got, expect[k])
        assert len(results) == 3 * len(ctxs)

        # the owner goes away: the sharers still hold the index memory
        owner.close()
        same(sharers[2].map(*batches[3], params), expect[3])
        # a sharer that loads its own index leaves the other sharers' alone
        sharers[1].load_index(view)
        same(sharers[1].map(*batches[0], params), expect[0])
        same(sharers[2].map(*batches[0], params), expect[0])
    finally:
        for c in sharers:
            c.close()
        owner.close()
