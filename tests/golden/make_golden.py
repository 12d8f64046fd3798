"""Generate the committed parity fixtures from the reference's own code path
(oracle/_ref/libmsgref.so, compiled from MSGseqTK's sources by
oracle/ref/Makefile). Run in the build container, where the reference tree
exists:  python tests/golden/make_golden.py

Each fixture holds the synthetic genome (seeded), the reads, and what the
reference computes for them: the FMD-index view (BWT, counts, SA samples,
chromosome table), SMEM lists, seed lists after removeRedundant, and the
per-chain alignments (window, score, coordinates, CIGAR, MD).
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


def main():
    build_reference()
    for name, (gb, rb, psets) in CASES.items():
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
