"""Parity of the CUDA path (through the C ABI) with the reference: committed
fixtures from the reference's own code, and the CPU restatement (oracle) on
freshly generated inputs. Integer/byte results must be bit-exact."""
import numpy as np
import pytest

from msgseqtk_b200 import index_build, lib, synth
from oracle.bind import Oracle

pytestmark = pytest.mark.gpu

COMP = [0, 8, 4, 12, 2, 10, 6, 14, 1, 9, 5, 13, 3, 11, 7, 15]


@pytest.fixture(scope="module")
def ctx():
    c = lib.Context(0)
    yield c
    c.close()


def aln_records(res, i):
    aln, cig, roff = res["aln"], res["cigar"], res["read_aln_off"]
    out = []
    for g in aln[roff[i]:roff[i + 1]]:
        fields = [int(g["tid"]), int(g["strand"]), int(g["t_start"]), int(g["t_end"]), int(g["aln_from"]),
                  int(g["aln_to"]), int(g["aln_start"]), int(g["aln_end"]), int(g["aln_score"])]
        words = [int(x) for x in cig[g["cigar_off"]:g["cigar_off"] + g["n_cigar"]]]
        out.append((fields, words, int(g["flags"])))
    return out


def md_of(words, read, strand, chrom, aln_from, aln_start):
    q = read if strand == 1 else synth.revcom(read)
    return lib.md_tag(words, q, lambda j: chrom[j] if j < len(chrom) else 0, aln_from, aln_start)


def compare_with_oracle(res, orc, reads_fn, n_reads, genomes, **ps):
    for i in range(n_reads):
        r = reads_fn(i)
        exp = orc.align_read(r, **ps)
        got = aln_records(res, i)
        assert len(got) == len(exp), (i, len(got), len(exp))
        for (fields, words, flags), e in zip(got, exp):
            ef = [e["tid"], e["strand"], e["t_start"], e["t_end"], e["aln_from"], e["aln_to"], e["aln_start"],
                  e["aln_end"], int(e["aln_score"]) if np.isfinite(e["aln_score"]) else -(2 ** 31)]
            assert fields == ef, (i, fields, ef)
            assert words == e["cigar"], (i, words, e["cigar"])
            assert flags == e["flags"], (i, flags, e["flags"])
            md = md_of(words, r, fields[1], genomes[fields[0]], fields[4], fields[6])
            assert md == e["md"], (i, md, e["md"])


@pytest.mark.parametrize("name", ["uniform", "repeats"])
def test_occ_ext_sa_match_oracle(ctx, cases, oracle_built, name):
    c = cases[name]
    ctx.load_index(c.view)
    orc = Oracle(c.view)
    n = c.view.n
    rng = np.random.default_rng(11)
    b = rng.choice(np.array([0, 1, 2, 4, 8], dtype=np.uint8), size=4000)
    i = rng.integers(-1, n + 2, size=4000)
    got = ctx.occ(b, i)
    exp = [orc.rank(int(x), int(y)) if 0 <= y < n else -1 for x, y in zip(b, i)]
    assert np.array_equal(got, np.array(exp))
    # bi-intervals reached by extending read substrings, then one more step
    Cc = np.concatenate([[0], np.cumsum(c.view.B)])
    for direction in (0, 1):
        P, Q, S, Bs, E = [], [], [], [], []
        for k in range(400):
            r = c.read(k % (len(c.read_off) - 1))
            pos = int(rng.integers(1, len(r) - 1))
            base = int(r[pos])
            p, q, s = int(Cc[base]), int(Cc[COMP[base]]), int(Cc[base + 1] - Cc[base])
            steps = int(rng.integers(0, 25))
            for t in range(steps + 1):
                j = pos - 1 - t if direction == 0 else pos + 1 + t
                nb = int(r[j]) if 0 <= j < len(r) else 0
                if t == steps or s <= 0:
                    if rng.random() < 0.2:
                        nb = int(rng.choice([0, 1, 2, 4, 8, 15]))
                    P.append(p); Q.append(q); S.append(s); Bs.append(nb)
                    E.append((orc.back_ext if direction == 0 else orc.fwd_ext)(p, q, s, nb))
                    break
                _, p, q, s = (orc.back_ext if direction == 0 else orc.fwd_ext)(p, q, s, nb)
        ret, p2, q2, s2 = ctx.bi_ext(direction, Bs, P, Q, S)
        for k, e in enumerate(E):
            assert (ret[k], p2[k], q2[k], s2[k]) == e, (direction, k, e)
    # the full suffix array recovered on the device equals a host suffix sort
    sa_ref = index_build.suffix_array(index_build.bd_text(c.genomes)).numpy()
    assert np.array_equal(ctx.sa(np.arange(n)), sa_ref)


@pytest.mark.parametrize("name", ["uniform", "repeats"])
def test_mapping_matches_reference_fixtures(ctx, cases, name):
    c = cases[name]
    ctx.load_index(c.view)
    n = len(c.read_off) - 1
    for k in range(c.n_params):
        ps = c.params(k)
        ex = c.expected(k)
        params = lib.default_params(min_len=ps["min_len"], max_evalue=ps["max_evalue"], max_nseed=ps["max_nseed"],
                                    mode=ps["mode"])
        res = ctx.map(c.reads, c.read_off, params, dump=True)
        assert np.array_equal(res["smem_off"], ex["smem_off"])
        assert np.array_equal(res["smem"], ex["smem"])
        assert np.array_equal(res["seed_off"], ex["seed_off"])
        assert np.array_equal(res["seed"], ex["seed"])
        assert np.array_equal(res["read_aln_off"], ex["aln_off"])
        for i in range(n):
            got = aln_records(res, i)
            rows = ex["aln"][ex["aln_off"][i]:ex["aln_off"][i + 1]]
            for (fields, words, flags), row, j in zip(got, rows, range(ex["aln_off"][i], ex["aln_off"][i + 1])):
                assert fields == [int(x) for x in row[:9]], (name, k, i)
                assert words == [int(x) for x in ex["cigar"][row[9]:row[9] + row[10]]], (name, k, i)
                md = md_of(words, c.read(i), fields[1], c.genomes[fields[0]], fields[4], fields[6])
                assert md == ex["md"][j], (name, k, i)


def test_mapping_matches_oracle_small_workload(ctx, oracle_built):
    """4 genomes x 200 kbp, 2000 single-end 150 bp reads with the small
    workload's error model, plus paired-end mates with 5% random pairs."""
    g = synth.small_genomes(seed=21, n_genomes=4, length=200_000)
    view = index_build.build_view(g)
    ctx.load_index(view)
    orc = Oracle(view)
    rs = synth.sample_reads(g, 2000, seed=22)
    res = ctx.map(rs.seqs, rs.offs)
    compare_with_oracle(res, orc, rs.read, len(rs), g)
    m1, m2 = synth.sample_pairs(g, 500, seed=23)
    pe = synth.interleave(m1, m2)
    res = ctx.map(pe.seqs, pe.offs)
    compare_with_oracle(res, orc, pe.read, len(pe), g)


def test_edge_cases_match_oracle(ctx, oracle_built):
    """Empty and ragged reads, N bases, reads shorter than the seed length,
    reads at chromosome ends (window reaching the terminator), random reads,
    local mode, infinite e-value and a tight maxNSeed."""
    g = synth.repeat_genomes(seed=31, n_genomes=3, length=12_000)
    view = index_build.build_view(g)
    ctx.load_index(view)
    orc = Oracle(view)
    rng = np.random.default_rng(32)
    reads = [np.zeros(0, np.uint8), g[0][:150].copy(), g[1][-150:].copy(), synth.revcom(g[2][:120]),
             synth.revcom(g[0][-90:]), g[1][500:510].copy(), synth._BASES[rng.integers(0, 4, 150)]]
    r = g[2][1000:1150].copy(); r[[10, 75, 140]] = 15; reads.append(r)
    r = g[0][3000:3200].copy(); r[100] = 15; reads.append(r)
    reads += [g[k][s:s + int(L)].copy() for k, s, L in zip(rng.integers(0, 3, 40), rng.integers(0, 11_000, 40),
                                                            rng.integers(1, 400, 40)) if s + L <= len(g[k])]
    seq = np.concatenate(reads).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(x) for x in reads])]).astype(np.int64)
    for ps in (dict(min_len=17, max_evalue=0.01, max_nseed=500, mode=0),
               dict(min_len=5, max_evalue=float("inf"), max_nseed=40, mode=0),
               dict(min_len=9, max_evalue=0.5, max_nseed=500, mode=1)):
        res = ctx.map(seq, off, lib.default_params(**ps))
        compare_with_oracle(res, orc, lambda i: reads[i], len(reads), g, **ps)
    res = ctx.map(np.zeros(0, np.uint8), np.zeros(1, np.int64))
    assert len(res["aln"]) == 0


def test_tandem_repeats_long_candidate_lists_match_oracle(ctx, oracle_built):
    """A genome of 200 diverged copies of one 600 bp unit: a walk's interval
    shrinks a few copies per base, so candidate lists outgrow the one-thread
    SMEM kernel's cap (those reads are abandoned and mapped again on the warp
    kernel), and with a small maxNSeed many reads need the host sort of
    their SMEMs (done for the whole batch in one round trip). Records equal
    the oracle's either way, and both paths are taken."""
    rng = np.random.default_rng(91)
    unit = synth._BASES[rng.integers(0, 4, 600)]
    parts = []
    for _ in range(200):
        u = unit.copy()
        mut = rng.random(600) < 0.015
        u[mut] = synth._BASES[rng.integers(0, 4, int(mut.sum()))]
        parts.append(u)
    g = [np.concatenate(parts), synth._BASES[rng.integers(0, 4, 50_000)]]
    view = index_build.build_view(g)
    ctx.load_index(view)
    orc = Oracle(view)
    rs = synth.sample_reads(g, 600, seed=92)
    for ps in (dict(min_len=13, max_evalue=0.01, max_nseed=500, mode=0),
               dict(min_len=13, max_evalue=0.01, max_nseed=30, mode=0)):
        res = ctx.map(rs.seqs, rs.offs, lib.default_params(**ps))
        st = ctx.stats()
        compare_with_oracle(res, orc, rs.read, len(rs), g, **ps)
        assert st["n_smem_rerun"] > 0
        if ps["max_nseed"] == 30:
            assert st["host_sorted"] > 0


def test_unsupported_inputs_fail_loudly(ctx):
    g = synth.small_genomes(seed=41, n_genomes=1, length=5000)
    view = index_build.build_view(g)
    ctx.load_index(view)
    with pytest.raises(lib.MsgError) as e:
        ctx.map(g[0][:150], np.array([0, 150]), lib.default_params(match=1.5))
    assert e.value.code == lib.MSG_EUNSUPPORTED


def test_uneven_lengths_match_oracle(ctx, oracle_built):
    """One batch mixing read lengths as the uneven-length workload does (75-150,
    250-300 and 1-2 kbp; 5% errors, 70% substitutions / 30% indels): short
    reads take the thread SMEM kernel, the others the warp kernel."""
    g = synth.small_genomes(seed=61, n_genomes=3, length=100_000)
    view = index_build.build_view(g)
    ctx.load_index(view)
    orc = Oracle(view)
    rng = np.random.default_rng(62)
    lens = list(rng.integers(75, 151, 40)) + list(rng.integers(250, 301, 20)) + list(rng.integers(1000, 2001, 8))
    reads = []
    for k, L in enumerate(lens):
        rs = synth.sample_reads(g, 1, L=int(L), seed=1000 + k, sub_rate=0.035, indel_rate=0.015)
        reads.append(rs.read(0).copy())
    order = rng.permutation(len(reads))
    reads = [reads[k] for k in order]
    seq = np.concatenate(reads).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum([len(x) for x in reads])]).astype(np.int64)
    res = ctx.map(seq, off)
    compare_with_oracle(res, orc, lambda i: reads[i], len(reads), g)
    res = ctx.map(seq, off, lib.default_params(min_score_rate=0.65, band_mode=1, band_w=15))
    n_kept = 0
    for i, r in enumerate(reads):
        exp = [e for e in orc.align_read(r) if not (e["aln_score"] < len(r) * 0.65)]
        got = aln_records(res, i)
        assert len(got) == len(exp), i
        n_kept += len(got)
        for (fields, words, flags), e in zip(got, exp):
            assert fields[:8] == [e["tid"], e["strand"], e["t_start"], e["t_end"], e["aln_from"], e["aln_to"],
                                  e["aln_start"], e["aln_end"]], i
            assert words == e["cigar"], i
    assert n_kept > 0


def test_scratch_limit_gives_same_records(oracle_built):
    """With the DP's rectangle storage capped far below the batch's need, the
    chains are aligned range by range; the records are unchanged."""
    g = synth.small_genomes(seed=71, n_genomes=3, length=80_000)
    view = index_build.build_view(g)
    c = lib.Context(0)
    try:
        c.load_index(view)
        rs = synth.sample_reads(g, 600, seed=72, sub_rate=0.035, indel_rate=0.015)
        rng = np.random.default_rng(73)
        rand = synth._BASES[rng.integers(0, 4, 150 * 60)]
        seq = np.concatenate([rs.seqs, rand]).astype(np.uint8)
        off = np.concatenate([rs.offs, rs.offs[-1] + 150 * np.arange(1, 61)]).astype(np.int64)
        for params in (lib.default_params(min_len=12), lib.default_params(min_score_rate=0.65, band_mode=1, band_w=7)):
            full = c.map(seq, off, params)
            c.set_scratch_limit(1 << 16)
            part = c.map(seq, off, params)
            c.set_scratch_limit(16 << 30)
            for k in ("aln", "cigar", "read_aln_off"):
                assert np.array_equal(full[k], part[k]), k
    finally:
        c.close()


@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5, 6, 7])
def test_smem_variants_match_reference_fixtures(cases, variant):
    """The SMEM kernel variants -- two reads per thread (1, 2), a pass's
    candidates extended four (3) or two (4) at a time, one read per thread
    with smaller register budgets (5, 6), one read per thread with the
    fast-forward over unique matches (7) -- emit every read's
    SMEMs exactly as the reference does (committed fixtures, all parameter
    sets), and map to the same records."""
    c = lib.Context(0)
    try:
        for name in ("uniform", "repeats"):
            cs = cases[name]
            c.load_index(cs.view)
            for k in range(cs.n_params):
                ps = cs.params(k)
                ex = cs.expected(k)
                params = lib.default_params(min_len=ps["min_len"], max_evalue=ps["max_evalue"],
                                            max_nseed=ps["max_nseed"], mode=ps["mode"])
                c.set_smem_shape(0)
                one = c.map(cs.reads, cs.read_off, params, dump=True)
                c.set_smem_shape(variant)
                two = c.map(cs.reads, cs.read_off, params, dump=True)
                assert np.array_equal(two["smem_off"], ex["smem_off"]) and np.array_equal(two["smem"], ex["smem"])
                for key in ("seed", "seed_off", "aln", "cigar", "read_aln_off"):
                    assert np.array_equal(one[key], two[key]), (name, k, key)
        with pytest.raises(lib.MsgError):
            c.set_smem_shape(8)
    finally:
        c.close()


DP_SHAPES = [(16, 256, 65536), (8, 0, 1 << 40), (32, 0, 1 << 40), (16, 1 << 40, 1 << 40), (16, 0, 0),
             (8, 64, 4096), (32, 256, 20000)]


def test_dp_shape_gives_same_records(oracle_built):
    """The DP's work split (row-by-row threads, register stripes of 8/16/32
    rows, warps) and lane width (16-bit two-stripe fill where the score
    bound allows it, or 32-bit everywhere) never change a record: every
    split maps the same reads -- with errors, random, and long (1 kbp) ones
    whose chains are large -- to the same records, plain, banded (fixed
    widths, certified or recomputed), local, and under a scoring scheme whose
    bound leaves only the shorter chains in 16 bits; the default split also
    equals the oracle."""
    g = synth.small_genomes(seed=75, n_genomes=3, length=120_000)
    view = index_build.build_view(g)
    orc = Oracle(view)
    c = lib.Context(0)
    try:
        c.load_index(view)
        rs = synth.sample_reads(g, 500, seed=76, sub_rate=0.03, indel_rate=0.01)
        rl = synth.sample_reads(g, 12, L=1000, seed=77, sub_rate=0.03, indel_rate=0.01)
        rng = np.random.default_rng(78)
        rand = synth._BASES[rng.integers(0, 4, 150 * 40)]
        seq = np.concatenate([rs.seqs, rl.seqs, rand]).astype(np.uint8)
        off = np.concatenate([rs.offs, rs.offs[-1] + rl.offs[1:],
                              rs.offs[-1] + rl.offs[-1] + 150 * np.arange(1, 41)]).astype(np.int64)
        reads = [seq[off[i]:off[i + 1]] for i in range(len(off) - 1)]
        plist = [lib.default_params(min_len=13), lib.default_params(min_len=13, mode=1),
                 lib.default_params(min_len=13, min_score_rate=0.65, band_mode=1, band_w=7),
                 lib.default_params(min_len=13, min_score_rate=0.5, band_mode=1, band_w=31),
                 lib.default_params(min_len=13, band_mode=1, band_w=15),
                 lib.default_params(min_len=13, mismatch=4, gap_open=10, gap_ext=10)]
        for pi, params in enumerate(plist):
            c.set_dp_shape(*DP_SHAPES[0])
            c.set_dp_lanes(16)
            base = c.map(seq, off, params)
            st0 = c.stats()
            if pi < 2 or pi == 5:
                compare_with_oracle(base, orc, lambda i: reads[i], len(reads), g, min_len=13, mode=params.mode,
                                    score=tuple(int(v) for v in (params.match, params.mismatch, params.gap_open,
                                                                   params.gap_ext)))
            for lanes, blocks in ((16, 3), (32, 3), (16, 4)):
                c.set_dp_lanes(lanes)
                c.set_dp_occupancy(blocks)
                for shape in DP_SHAPES[1:] if (lanes, blocks) == (16, 3) else DP_SHAPES[:4]:
                    c.set_dp_shape(*shape)
                    got = c.map(seq, off, params)
                    for k in ("aln", "cigar", "read_aln_off"):
                        assert np.array_equal(base[k], got[k]), (pi, lanes, shape, k)
                    st = c.stats()
                    assert st["dp_cells"] == st0["dp_cells"], (pi, shape)
                    assert (st["n_band_exact"], st["n_band_drop"], st["n_band_fallback"]) == \
                        (st0["n_band_exact"], st0["n_band_drop"], st0["n_band_fallback"]), (pi, shape)
            c.set_dp_lanes(16)
            c.set_dp_occupancy(3)
            assert len(base["aln"]) > 0
        with pytest.raises(lib.MsgError):
            c.set_dp_lanes(8)
        with pytest.raises(lib.MsgError):
            c.set_dp_shape(12, 256, 65536)
        # the autotuner picks one of its candidates and changes no record
        params = plist[2]
        c.set_dp_shape(*DP_SHAPES[0])
        before = c.map(seq, off, params)
        tune = c.autotune(seq, off, params)
        assert tune["stripe_rows"] in (8, 16, 32) and tune["n_tried"] == 18 and tune["smem_variant"] in range(8)
        assert tune["dp_lanes"] in (16, 32) and tune["dp_stripe_blocks"] in (3, 4)
        assert tune["warp_area"] in (4096, 16384, 65536, 262144) and tune["small_area"] in (0, 64, 256, 1024)
        after = c.map(seq, off, params)
        for k in ("aln", "cigar", "read_aln_off"):
            assert np.array_equal(before[k], after[k]), k
    finally:
        c.close()


def test_map_batches_equals_map_batch(oracle_built):
    """msg_map_batches (copies overlapped with the neighbouring batches'
    mapping) gives each batch exactly msg_map_batch's records: batches of
    different sizes, an empty one, offsets that do not start at 0, pinned and
    pageable host buffers."""
    import torch
    g = synth.small_genomes(seed=81, n_genomes=3, length=80_000)
    view = index_build.build_view(g)
    c = lib.Context(0)
    try:
        c.load_index(view)
        rs = synth.sample_reads(g, 1500, seed=82, sub_rate=0.02, indel_rate=0.005)
        params = lib.default_params(min_score_rate=0.65)
        cuts = [0, 700, 700, 1100, 1101, 1500]
        batches, expect = [], []
        for a, b in zip(cuts[:-1], cuts[1:]):
            batches.append((rs.seqs, np.ascontiguousarray(rs.offs[a:b + 1])))  # offsets into the whole array
            o = rs.offs[a:b + 1] - rs.offs[a]
            expect.append(c.map(rs.seqs[rs.offs[a]:rs.offs[b]], o, params))

        def pinned(n, dt):
            dt = np.dtype(dt)
            return torch.empty(n * dt.itemsize, dtype=torch.uint8).pin_memory().numpy().view(dt)

        for pin in (True, False):
            outs = []
            for (s, o) in batches:
                n = len(o) - 1
                mk = pinned if pin else (lambda k, dt: np.zeros(k, dtype=dt))
                outs.append((mk(4 * n + 16, lib.ALN_DTYPE), mk(64 * n + 64, np.uint32), mk(n + 1, np.int64)))
            counts = c.map_batches(batches, outs, params)
            for (na, nc), (al, cg, ro), ex in zip(counts, outs, expect):
                assert np.array_equal(al[:na], ex["aln"])
                assert np.array_equal(cg[:nc], ex["cigar"])
                assert np.array_equal(ro, ex["read_aln_off"])
        # a batch whose records do not fit: MSG_EINVAL, the others still mapped
        outs = [(np.zeros(4 * (len(o) - 1) + 16, lib.ALN_DTYPE), np.zeros(64 * len(o), np.uint32),
                 np.zeros(len(o), np.int64)) for _, o in batches]
        outs[0] = (np.zeros(1, lib.ALN_DTYPE), outs[0][1], outs[0][2])
        with pytest.raises(lib.MsgError) as e:
            c.map_batches(batches, outs, params)
        assert e.value.code == lib.MSG_EINVAL
        al, cg, ro = outs[2]
        assert np.array_equal(ro, expect[2]["read_aln_off"])
    finally:
        c.close()


def test_read_bytes_must_be_nt16_codes(oracle_built):
    """Bytes above 15 (e.g. ASCII letters) are rejected with MSG_EINVAL before
    any kernel uses them; the context keeps working."""
    g = synth.small_genomes(seed=91, n_genomes=1, length=20_000)
    view = index_build.build_view(g)
    c = lib.Context(0)
    try:
        c.load_index(view)
        good = g[0][1000:1150].copy()
        bad = np.frombuffer(b"ACGT" * 30, dtype=np.uint8).copy()
        seq = np.concatenate([good, bad])
        off = np.array([0, 150, 270], dtype=np.int64)
        with pytest.raises(lib.MsgError) as e:
            c.map(seq, off)
        assert e.value.code == lib.MSG_EINVAL
        res = c.map(good, np.array([0, 150], dtype=np.int64))
        assert len(res["aln"]) >= 1
    finally:
        c.close()
