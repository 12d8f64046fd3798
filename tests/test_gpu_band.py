"""Banded flank DP and the learned band, through the C ABI.

Whatever band a chain gets, the records must equal those of the whole
reference cell set (and the oracle's, after Alignment::filter when
min_score_rate is set). The classifier's gradients must match the CPU
oracle, and the trained classifier must compute fewer DP cells than the
whole cell set on fresh reads."""
import numpy as np
import pytest

from msgseqtk_b200 import index_build, lib, synth
from oracle import band_mlp as bm
from oracle.bind import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def _mixed_reads(g, seed, n_true, n_noisy, n_random):
    """True reads (1% errors), noisy reads (5% substitutions, 1% indels) and
    random reads: the last two give chains with large flank rectangles."""
    a = synth.sample_reads(g, n_true, seed=seed)
    b = synth.sample_reads(g, n_noisy, seed=seed + 1, sub_rate=0.05, indel_rate=0.01)
    rng = np.random.default_rng(seed + 2)
    reads = [a.read(i) for i in range(len(a))] + [b.read(i) for i in range(len(b))]
    reads += [synth._BASES[rng.integers(0, 4, 150)] for _ in range(n_random)]
    order = rng.permutation(len(reads))
    reads = [reads[k] for k in order]
    seq = np.concatenate(reads).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(x) for x in reads])]).astype(np.int64)
    return reads, seq, off


@pytest.fixture(scope="module")
def world(ctx):
    g = synth.scale_genomes(seed=51, n_genomes=8, median=2e5)
    view = index_build.build_view(g)
    ctx.load_index(view)
    return g, view


PSETS = [dict(min_len=17, max_evalue=0.01), dict(min_len=12, max_evalue=float("inf"))]


def _same(a, b):
    assert np.array_equal(a["read_aln_off"], b["read_aln_off"])
    assert np.array_equal(a["aln"], b["aln"])
    assert np.array_equal(a["cigar"], b["cigar"])


def _oracle_filtered(orc, reads, res, rate, ps):
    roff, aln, cig = res["read_aln_off"], res["aln"], res["cigar"]
    for i, r in enumerate(reads):
        exp = [e for e in orc.align_read(r, **ps) if not (rate >= 0 and e["aln_score"] < len(r) * rate)]
        got = aln[roff[i]:roff[i + 1]]
        assert len(got) == len(exp), (i, len(got), len(exp))
        for gg, e in zip(got, exp):
            assert [int(gg[k]) for k in ("tid", "strand", "t_start", "t_end", "aln_from", "aln_to", "aln_start",
                                         "aln_end", "aln_score")] == \
                [e["tid"], e["strand"], e["t_start"], e["t_end"], e["aln_from"], e["aln_to"], e["aln_start"],
                 e["aln_end"], int(e["aln_score"]) if np.isfinite(e["aln_score"]) else -(2 ** 31)], i
            assert [int(x) for x in cig[gg["cigar_off"]:gg["cigar_off"] + gg["n_cigar"]]] == e["cigar"], i


def test_fixed_band_equals_whole_cell_set(ctx, world, oracle_built):
    g, view = world
    orc = Oracle(view)
    reads, seq, off = _mixed_reads(g, 61, 600, 300, 150)
    seen = dict(exact=0, drop=0, fallback=0)
    for ps in PSETS:
        for rate in (-1.0, 0.65):
            plain = ctx.map(seq, off, lib.default_params(min_score_rate=rate, **ps))
            st0 = ctx.stats()
            _oracle_filtered(orc, reads, plain, rate, ps)
            for w in (7, 15, 31):
                res = ctx.map(seq, off, lib.default_params(min_score_rate=rate, band_mode=1, band_w=w, **ps))
                _same(res, plain)
                st = ctx.stats()
                assert st["n_filtered"] == st0["n_filtered"]
                seen["exact"] += st["n_band_exact"]
                seen["drop"] += st["n_band_drop"]
                seen["fallback"] += st["n_band_fallback"]
                if rate < 0:
                    assert st["n_band_drop"] == 0
    # every certificate outcome was exercised
    assert seen["exact"] > 0 and seen["drop"] > 0 and seen["fallback"] > 0, seen


def test_band_ignored_in_local_mode(ctx, world):
    g, _ = world
    _, seq, off = _mixed_reads(g, 71, 200, 100, 50)
    plain = ctx.map(seq, off, lib.default_params(mode=1, min_len=12))
    res = ctx.map(seq, off, lib.default_params(mode=1, min_len=12, band_mode=1, band_w=7))
    _same(res, plain)
    assert ctx.stats()["n_band_exact"] == 0


def test_gradient_matches_oracle(ctx, world):
    g, _ = world
    _, seq, off = _mixed_reads(g, 81, 300, 150, 80)
    feat, lab = ctx.band_collect(seq, off, lib.default_params(min_score_rate=0.65, min_len=12))
    assert set(np.unique(lab)) <= {-1, 0, 1, 2, 3}
    feat, lab = feat[lab >= 0], lab[lab >= 0]
    assert len(lab) > 50
    rng = np.random.default_rng(3)
    params = bm.random_params(rng, feat)
    grad, loss = ctx.band_grad(params, feat, lab)
    eloss, egrad = bm.loss_and_grad(params, feat, lab)
    assert abs(loss - eloss) <= 1e-4 * max(1.0, abs(eloss))
    scale = np.abs(egrad).max()
    assert np.allclose(grad, egrad, rtol=2e-3, atol=2e-5 * scale), np.abs(grad - egrad).max() / scale


def test_learned_band_is_exact_and_saves_cells(ctx, world, oracle_built):
    g, view = world
    ps = dict(min_len=12, max_evalue=float("inf"), min_score_rate=0.65)
    _, tseq, toff = _mixed_reads(g, 91, 2000, 1000, 500)
    feat, lab = ctx.band_collect(tseq, toff, lib.default_params(**ps))
    feat, lab = feat[lab >= 0], lab[lab >= 0]
    params, loss = ctx.band_train(feat, lab, epochs=30, batch=512, lr=3e-3, seed=7)
    assert loss[-1] < loss[0]
    # the device classifier and the oracle's agree on most fresh chains
    reads, seq, off = _mixed_reads(g, 101, 800, 400, 200)
    f2, l2 = ctx.band_collect(seq, off, lib.default_params(**ps))
    f2, l2 = f2[l2 >= 0], l2[l2 >= 0]
    acc = float(np.mean(bm.classify(params, f2) == l2))
    assert acc > 0.5, acc
    plain = ctx.map(seq, off, lib.default_params(**ps))
    cells_plain = ctx.stats()["dp_cells_done"]
    res = ctx.map(seq, off, lib.default_params(band_mode=2, **ps))
    st = ctx.stats()
    _same(res, plain)
    _oracle_filtered(Oracle(view), reads, res, ps["min_score_rate"], dict(min_len=12, max_evalue=float("inf")))
    assert st["n_band_exact"] + st["n_band_drop"] > 0
    assert st["dp_cells_done"] < cells_plain, (st["dp_cells_done"], cells_plain)


def test_band_model_errors(world):
    c = lib.Context(0)
    try:
        g, view = world
        c.load_index(view)
        with pytest.raises(lib.MsgError) as e:
            c.map(g[0][:150], np.array([0, 150]), lib.default_params(band_mode=2))
        assert e.value.code == lib.MSG_ESTATE
        with pytest.raises(lib.MsgError) as e:
            c.band_model_set(np.zeros(10, np.float32))
        assert e.value.code == lib.MSG_EINVAL
        p = bm.random_params(np.random.default_rng(1))
        p[bm.FEAT] = 0.0  # a zero feature scale
        with pytest.raises(lib.MsgError) as e:
            c.band_model_set(p)
        assert e.value.code == lib.MSG_EINVAL
        with pytest.raises(lib.MsgError) as e:
            c.map(g[0][:150], np.array([0, 150]), lib.default_params(band_mode=1, band_w=-3))
        assert e.value.code == lib.MSG_EINVAL
    finally:
        c.close()
