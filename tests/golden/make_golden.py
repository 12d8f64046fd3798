"""Generate the committed parity fixtures from the reference's own code path
(oracle/_ref/libmsgref.so, compiled from MSGseqTK's sources by
oracle/ref/Makefile). Run in the build container, where the reference tree
exists:  python tests/golden/make_golden.py

Each fixture holds the synthetic genome (seeded), the reads, and what the
reference computes for them: the FMD-index view (BWT, counts, SA samples,
chromosome table), SMEM lists, seed lists after removeRedundant, and the
per-chain alignments (window, score, coordinates, CIGAR, MD). The "clean"
fixture holds msgseqtk-clean's path: two genome sets (reference and
background), reads from both plus random and odd-symbol reads, the
reference's findMEMS lists and loglik, and its clean decisions for single
reads and pairs.

    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py clean      # only the named ones
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from msgseqtk_b200 import synth  # noqa: E402
from oracle.bind import Reference, build_reference  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

CASES = {
    # name: (genome builder, reads builder, param sets)
    "uniform": (lambda: synth.small_genomes(seed=101, n_genomes=3, length=20000),
                lambda g: synth.sample_reads(g, 120, seed=102),
                [dict(min_len=17, max_evalue=0.01, max_nseed=500, mode=0)]),
    "repeats": (lambda: synth.repeat_genomes(seed=103, n_genomes=2, length=15000),
                lambda g: synth.sample_reads(g, 120, seed=104, sub_rate=0.03, indel_rate=0.01),
                [dict(min_len=17, max_evalue=0.01, max_nseed=500, mode=0),
                 dict(min_len=6, max_evalue=float("inf"), max_nseed=60, mode=0),
                 dict(min_len=12, max_evalue=1.0, max_nseed=500, mode=1)]),
}


CLEAN_PARAMS = [(17, 0.01), (1, float("inf")), (9, 1e3)]  # (min_len, max_evalue)
CLEAN_LOD = [0.0, 25.0]


def clean_reads(g_ref, g_bg, seed):
    """Reads from both genome sets, random reads, and reads holding the
    symbols the reference's encoder can produce besides A/C/G/T (0 for
    unknown characters, N, IUPAC codes), an empty read and a 1-base read."""
    rng = np.random.default_rng(seed)
    a = synth.sample_reads(g_ref, 60, seed=seed + 1)
    b = synth.sample_reads(g_bg, 60, seed=seed + 2, sub_rate=0.03, indel_rate=0.01)
    reads = [a.read(i) for i in range(len(a))] + [b.read(i) for i in range(len(b))]
    reads += [synth._BASES[rng.integers(0, 4, int(rng.integers(20, 200)))] for _ in range(20)]
    for i in range(20):
        r = reads[i].copy()
        pos = rng.integers(0, len(r), 4)
        r[pos] = rng.choice(np.array([0, 15, 5, 3, 14], dtype=np.uint8), 4)
        reads.append(r)
    reads += [np.zeros(0, np.uint8), np.array([4], np.uint8), np.array([0, 0, 1, 2, 0], np.uint8)]
    reads += [synth._BASES[rng.integers(0, 4, 1500)]]
    off = np.cumsum([0] + [len(r) for r in reads]).astype(np.int64)
    return np.concatenate(reads).astype(np.uint8), off


def make_clean():
    g_ref = synth.small_genomes(seed=111, n_genomes=3, length=20000)
    g_bg = synth.small_genomes(seed=112, n_genomes=2, length=25000)
    ref, bg = Reference(g_ref), Reference(g_bg)
    seq, off = clean_reads(g_ref, g_bg, 113)
    seq2, off2 = clean_reads(g_bg, g_ref, 114)  # second mates (same count)
    data = dict(ref_genome=np.concatenate(g_ref).astype(np.uint8),
                ref_genome_off=np.cumsum([0] + [len(x) for x in g_ref]).astype(np.int64),
                bg_genome=np.concatenate(g_bg).astype(np.uint8),
                bg_genome_off=np.cumsum([0] + [len(x) for x in g_bg]).astype(np.int64),
                reads=seq, read_off=off, mates=seq2, mate_off=off2,
                params=np.array(CLEAN_PARAMS, dtype=np.float64), lods=np.array(CLEAN_LOD))
    n = len(off) - 1
    for k, (ml, me) in enumerate(CLEAN_PARAMS):
        rows, roff, ll = [], [0], []
        for i in range(n):
            m, l = ref.mems(seq[off[i]:off[i + 1]], ml, me)
            rows.append(m); roff.append(roff[-1] + len(m)); ll.append(l)
        data[f"p{k}_mem"] = np.concatenate(rows)
        data[f"p{k}_mem_off"] = np.array(roff, dtype=np.int64)
        data[f"p{k}_mem_ll"] = np.array(ll, dtype=np.float64)
        for j, lod in enumerate(CLEAN_LOD):
            se = ref.clean_batch(bg, seq, off, min_len=ml, max_evalue=me, min_lod=lod, n_threads=4)
            pe = ref.clean_batch(bg, seq, off, seq2, off2, min_len=ml, max_evalue=me, min_lod=lod, n_threads=4)
            for tag, res in (("se", se), ("pe", pe)):
                data[f"p{k}_l{j}_{tag}"] = np.stack(res[:3])
                data[f"p{k}_l{j}_{tag}_keep"] = res[3]
    np.savez_compressed(os.path.join(OUT, "clean.npz"), **data)
    print("clean", {k: v.shape for k, v in data.items() if hasattr(v, "shape")})


def main():
    build_reference()
    names = sys.argv[1:] or list(CASES) + ["clean"]
    if "clean" in names:
        make_clean()
    for name, (gb, rb, psets) in CASES.items():
        if name not in names:
            continue
        g = gb()
        ref = Reference(g)
        rs = rb(g)
        B, _ = ref.counts()
        rows, vals = ref.sa_samples()
        bs, be, cl = ref.chroms()
        data = dict(genome_off=np.cumsum([0] + [len(x) for x in g]).astype(np.int64),
                    genome=np.concatenate(g).astype(np.uint8), reads=rs.seqs, read_off=rs.offs,
                    bwt=ref.bwt(), B=B[:16].copy(), sample_rows=rows, sample_vals=vals, bd_start=bs, bd_end=be,
                    chr_len_ref=cl)
        for k, ps in enumerate(psets):
            smem, smem_off, seed, seed_off = [], [0], [], [0]
            aln, aln_off, cig, md = [], [0], [], []
            for i in range(len(rs)):
                r = rs.read(i)
                a = ref.smems(r, ps["min_len"], ps["max_evalue"])
                smem.append(a); smem_off.append(smem_off[-1] + len(a))
                s = ref.seeds(r, ps["min_len"], ps["max_evalue"], ps["max_nseed"])
                seed.append(s); seed_off.append(seed_off[-1] + len(s))
                al = ref.align_read(r, ps["min_len"], ps["max_evalue"], ps["max_nseed"], ps["mode"])
                for x in al:
                    aln.append([x["tid"], x["strand"], x["t_start"], x["t_end"], x["aln_from"], x["aln_to"],
                                x["aln_start"], x["aln_end"], int(x["aln_score"]), len(cig), len(x["cigar"])])
                    cig.extend(x["cigar"])
                    md.append(x["md"])
                aln_off.append(len(aln))
            data[f"p{k}_params"] = np.array([ps["min_len"], ps["max_evalue"], ps["max_nseed"], ps["mode"]], dtype=np.float64)
            data[f"p{k}_smem"] = np.concatenate(smem) if smem else np.zeros((0, 6), np.int64)
            data[f"p{k}_smem_off"] = np.array(smem_off, dtype=np.int64)
            data[f"p{k}_seed"] = np.concatenate(seed) if seed else np.zeros((0, 6), np.int64)
            data[f"p{k}_seed_off"] = np.array(seed_off, dtype=np.int64)
            data[f"p{k}_aln"] = np.array(aln, dtype=np.int64).reshape(-1, 11)
            data[f"p{k}_aln_off"] = np.array(aln_off, dtype=np.int64)
            data[f"p{k}_cigar"] = np.array(cig, dtype=np.uint32)
            data[f"p{k}_md"] = np.frombuffer("\n".join(md).encode(), dtype=np.uint8)
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **data)
        print(name, {k: v.shape for k, v in data.items() if hasattr(v, "shape")})


if __name__ == "__main__":
    main()
