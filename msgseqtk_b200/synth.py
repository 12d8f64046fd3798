"""Seeded synthetic metagenomes and reads with the shapes of the mapping
workloads this library is measured on.

Sequences are nt16 codes as MSGseqTK stores them (A=1, C=2, G=4, T=8, N=15;
DNAalphabet.h:37-51). Everything is drawn from numpy's PCG64 generator seeded
by the caller, so a (config, seed) pair always yields the same bytes on any
machine.

Workloads:
  * small: 4 genomes x 500 kbp, i.i.d. uniform ACGT; 10,000 single-end 150 bp
    reads, 1% substitutions, 0.1% indels of length 1-3, Phred 20-40.
  * scale: 200 genomes with log-normal lengths (median 3 Mbp, sigma 0.5,
    ~600 Mbp total), per-genome GC uniform in 30-70%; paired 2x150 bp reads,
    fragment ~ Normal(400, 50), same error model, plus 5% random pairs.
  * repeats: two metagenomes of ~750 Mbp each (repeat_metagenome: 10% of
    the sequence in repeat families), indexed together; reads as for scale.
"""
from __future__ import annotations

import numpy as np

A, C, G, T, N = 1, 2, 4, 8, 15
_COMP = np.array([0, 8, 4, 12, 2, 10, 6, 14, 1, 9, 5, 13, 3, 11, 7, 15], dtype=np.uint8)
_BASES = np.array([A, C, G, T], dtype=np.uint8)
_ASCII = np.frombuffer(b"$ACMGRSVTWYHKDBN", dtype=np.uint8)


def revcom(seq: np.ndarray) -> np.ndarray:
    """Reverse complement of an nt16 array (dna::revcom, DNAseq.h:134-153)."""
    return _COMP[seq[::-1]]


def to_ascii(seq: np.ndarray) -> str:
    return _ASCII[seq].tobytes().decode()


def random_genome(rng: np.random.Generator, length: int, gc: float = 0.5) -> np.ndarray:
    """i.i.d. bases with P(G)=P(C)=gc/2 and P(A)=P(T)=(1-gc)/2."""
    u = rng.random(length)
    half_at = (1.0 - gc) / 2.0
    out = np.empty(length, dtype=np.uint8)
    out[u < half_at] = A
    m = (u >= half_at) & (u < 0.5)
    out[m] = T
    m = (u >= 0.5) & (u < 0.5 + gc / 2.0)
    out[m] = C
    out[u >= 0.5 + gc / 2.0] = G
    return out


def small_genomes(seed: int = 1, n_genomes: int = 4, length: int = 500_000):
    rng = np.random.Generator(np.random.PCG64(seed))
    return [_BASES[rng.integers(0, 4, size=length)] for _ in range(n_genomes)]


def scale_genomes(seed: int = 2, n_genomes: int = 200, median: float = 3e6, sigma: float = 0.5):
    rng = np.random.Generator(np.random.PCG64(seed))
    lens = np.maximum(1000, np.round(median * np.exp(sigma * rng.standard_normal(n_genomes)))).astype(np.int64)
    gcs = rng.uniform(0.3, 0.7, size=n_genomes)
    return [random_genome(rng, int(l), float(g)) for l, g in zip(lens, gcs)]


def repeat_metagenome(seed: int, total_bp: float = 750e6, median: float = 3e6, sigma: float = 0.5,
                      repeat_frac: float = 0.10, unit_range=(500, 5001), copies_range=(10, 201),
                      divergence_range=(0.02, 0.05)):
    """A metagenome for the repeat-rich workload: genomes with log-normal
    lengths (median, sigma) adding up to about total_bp, per-genome GC
    uniform in 30-70%, of which repeat_frac of the sequence is overwritten by
    repeat families -- units of U{500..5000} bp, each copied U{10..200} times
    to uniformly chosen places of the metagenome, on either strand, every
    copy with its own substitution divergence U(2%, 5%). Copies of one
    family land in different genomes, so SMEMs in repeats have many
    occurrences."""
    rng = np.random.Generator(np.random.PCG64(seed))
    mean_len = median * np.exp(sigma * sigma / 2.0)
    n_genomes = max(1, int(round(total_bp / mean_len)))
    lens = np.maximum(10_000, np.round(median * np.exp(sigma * rng.standard_normal(n_genomes)))).astype(np.int64)
    gcs = rng.uniform(0.3, 0.7, size=n_genomes)
    genomes = [random_genome(rng, int(l), float(g)) for l, g in zip(lens, gcs)]
    ends = np.cumsum(lens)
    budget = int(repeat_frac * ends[-1])
    while budget > 0:
        ul = int(rng.integers(*unit_range))
        unit = _BASES[rng.integers(0, 4, size=ul)]
        for _ in range(int(rng.integers(*copies_range))):
            if budget <= 0:
                break
            gi = int(np.searchsorted(ends, rng.integers(0, ends[-1]), side="right"))
            g = genomes[gi]
            if len(g) <= ul:
                continue
            cp = unit.copy()
            m = rng.random(ul) < rng.uniform(*divergence_range)
            cp[m] = _BASES[(np.searchsorted(_BASES, cp[m]) + rng.integers(1, 4, size=int(m.sum()))) % 4]
            if rng.random() < 0.5:
                cp = revcom(cp)
            at = int(rng.integers(0, len(g) - ul))
            g[at:at + ul] = cp
            budget -= ul
    return genomes


def _indel_read(rng, win: np.ndarray, L: int, n_ev: int) -> np.ndarray:
    """Apply n_ev indels (insertion or deletion of U{1..3} bases, equally
    likely) at uniform read positions to a substituted window; L bases out."""
    pos = np.sort(rng.integers(0, L, size=n_ev))
    parts = []
    i = 0  # position in the window
    o = 0  # bases emitted
    for p in pos:
        take = max(0, int(p) - o)
        parts.append(win[i:i + take])
        i += take
        o += take
        k = int(rng.integers(1, 4))
        if rng.random() < 0.5:
            parts.append(_BASES[rng.integers(0, 4, size=k)])
            o += k
        else:
            i += k
    parts.append(win[i:i + max(0, L - o)])
    out = np.concatenate(parts)[:L]
    if len(out) < L:
        out = np.concatenate([out, _BASES[rng.integers(0, 4, size=L - len(out))]])
    return out


def _apply_errors(rng, windows: np.ndarray, L: int, sub_rate: float, indel_rate: float) -> np.ndarray:
    """Substitutions at sub_rate per base (vectorised over all reads), then
    Binomial(L, indel_rate) indels per read."""
    n, W = windows.shape
    sub = rng.random((n, W)) < sub_rate
    shift = rng.integers(1, 4, size=(n, W), dtype=np.int8)
    idx = np.searchsorted(_BASES, windows).astype(np.int8)
    win = np.where(sub, _BASES[(idx + shift) % 4], windows)
    reads = win[:, :L].copy()
    n_ev = rng.binomial(L, indel_rate, size=n)
    for r in np.nonzero(n_ev)[0]:
        reads[r] = _indel_read(rng, win[r], L, int(n_ev[r]))
    return reads


class ReadSet:
    """Reads as one concatenated nt16 array with offsets, plus Phred scores and
    the true origin (genome index, 0-based forward start, strand 1=FWD 2=REV)."""

    def __init__(self, seqs: np.ndarray, offs: np.ndarray, quals: np.ndarray, truth: np.ndarray):
        self.seqs = seqs
        self.offs = offs
        self.quals = quals
        self.truth = truth

    def __len__(self):
        return len(self.offs) - 1

    def read(self, i: int) -> np.ndarray:
        return self.seqs[self.offs[i]:self.offs[i + 1]]

    def qual(self, i: int) -> np.ndarray:
        return self.quals[self.offs[i]:self.offs[i + 1]]


def sample_reads(genomes, n_reads: int, L: int = 150, seed: int = 3, sub_rate: float = 0.01,
                 indel_rate: float = 0.001, q_lo: int = 20, q_hi: int = 40) -> ReadSet:
    """Single-end reads from uniformly chosen genomes, strands and positions."""
    rng = np.random.Generator(np.random.PCG64(seed))
    slack = 16
    g = rng.integers(0, len(genomes), size=n_reads)
    lens = np.array([len(x) for x in genomes], dtype=np.int64)
    pos = (rng.random(n_reads) * (lens[g] - (L + slack))).astype(np.int64)
    strand = rng.integers(1, 3, size=n_reads)
    windows = np.empty((n_reads, L + slack), dtype=np.uint8)
    for k in range(len(genomes)):
        m = np.nonzero(g == k)[0]
        if len(m) == 0:
            continue
        gi = pos[m, None] + np.arange(L + slack)[None, :]
        windows[m] = genomes[k][gi]
    rev = strand == 2
    windows[rev] = _COMP[windows[rev][:, ::-1]]
    reads = _apply_errors(rng, windows, L, sub_rate, indel_rate)
    quals = rng.integers(q_lo, q_hi + 1, size=(n_reads, L)).astype(np.uint8)
    offs = np.arange(n_reads + 1, dtype=np.int64) * L
    truth = np.stack([g, pos, strand], axis=1).astype(np.int64)
    return ReadSet(reads.reshape(-1), offs, quals.reshape(-1), truth)


def sample_pairs(genomes, n_pairs: int, L: int = 150, seed: int = 4, ins_mean: float = 400.0,
                 ins_sd: float = 50.0, sub_rate: float = 0.01, indel_rate: float = 0.001,
                 random_frac: float = 0.05, q_lo: int = 20, q_hi: int = 40):
    """Paired-end reads: mate 1 is the fragment's first L bases, mate 2 the
    reverse complement of its last L bases; random_frac of pairs are random
    sequence (unmappable). Returns (mate1 ReadSet, mate2 ReadSet)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    frag = np.clip(np.round(rng.normal(ins_mean, ins_sd, size=n_pairs)), L + 10, 4 * ins_mean).astype(np.int64)
    fmax = int(frag.max()) + 16
    g = rng.integers(0, len(genomes), size=n_pairs)
    lens = np.array([len(x) for x in genomes], dtype=np.int64)
    pos = (rng.random(n_pairs) * (lens[g] - fmax)).astype(np.int64)
    strand = rng.integers(1, 3, size=n_pairs)
    w = L + 16
    m1 = np.empty((n_pairs, w), dtype=np.uint8)
    m2 = np.empty((n_pairs, w), dtype=np.uint8)
    for k in range(len(genomes)):
        m = np.nonzero(g == k)[0]
        if len(m) == 0:
            continue
        gi = pos[m, None] + np.arange(w)[None, :]
        m1[m] = genomes[k][gi]
        end = pos[m] + frag[m]
        gi2 = end[:, None] - 1 - np.arange(w)[None, :]
        m2[m] = _COMP[genomes[k][gi2]]
    rev = strand == 2
    m1[rev], m2[rev] = m2[rev].copy(), m1[rev].copy()
    r1 = _apply_errors(rng, m1, L, sub_rate, indel_rate)
    r2 = _apply_errors(rng, m2, L, sub_rate, indel_rate)
    rnd = rng.random(n_pairs) < random_frac
    nr = int(rnd.sum())
    r1[rnd] = _BASES[rng.integers(0, 4, size=(nr, L))]
    r2[rnd] = _BASES[rng.integers(0, 4, size=(nr, L))]
    q1 = rng.integers(q_lo, q_hi + 1, size=(n_pairs, L)).astype(np.uint8)
    q2 = rng.integers(q_lo, q_hi + 1, size=(n_pairs, L)).astype(np.uint8)
    offs = np.arange(n_pairs + 1, dtype=np.int64) * L
    truth = np.stack([g, pos, strand, frag, rnd.astype(np.int64)], axis=1).astype(np.int64)
    return (ReadSet(r1.reshape(-1), offs, q1.reshape(-1), truth),
            ReadSet(r2.reshape(-1), offs.copy(), q2.reshape(-1), truth))


def interleave(m1: ReadSet, m2: ReadSet) -> ReadSet:
    """Mates of each pair as consecutive reads (r1_0, r2_0, r1_1, ...)."""
    n = len(m1)
    L1 = np.diff(m1.offs)
    L2 = np.diff(m2.offs)
    lens = np.empty(2 * n, dtype=np.int64)
    lens[0::2] = L1
    lens[1::2] = L2
    offs = np.zeros(2 * n + 1, dtype=np.int64)
    np.cumsum(lens, out=offs[1:])
    if np.all(L1 == L1[0]) and np.all(L2 == L1[0]):
        L = int(L1[0])
        seqs = np.stack([m1.seqs.reshape(n, L), m2.seqs.reshape(n, L)], axis=1).reshape(-1)
        quals = np.stack([m1.quals.reshape(n, L), m2.quals.reshape(n, L)], axis=1).reshape(-1)
    else:
        parts, qparts = [], []
        for i in range(n):
            parts += [m1.read(i), m2.read(i)]
            qparts += [m1.quals[m1.offs[i]:m1.offs[i + 1]], m2.quals[m2.offs[i]:m2.offs[i + 1]]]
        seqs = np.concatenate(parts)
        quals = np.concatenate(qparts)
    truth = np.repeat(m1.truth, 2, axis=0)
    return ReadSet(seqs, offs, quals, truth)


def repeat_genomes(seed: int = 7, n_genomes: int = 3, length: int = 60_000, unit_range=(300, 2000),
                   copies_range=(5, 30), divergence_range=(0.0, 0.05), repeat_frac: float = 0.3):
    """Genomes where repeat_frac of the sequence is made of repeat families:
    units of U{unit_range} bp copied U{copies_range} times with per-copy
    substitution divergence U{divergence_range}. High-occurrence SMEMs come
    from these."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n_genomes):
        g = _BASES[rng.integers(0, 4, size=length)]
        budget = int(repeat_frac * length)
        while budget > 0:
            ul = int(rng.integers(*unit_range))
            unit = _BASES[rng.integers(0, 4, size=ul)]
            nc = int(rng.integers(*copies_range))
            for _ in range(nc):
                if budget <= 0:
                    break
                div = rng.uniform(*divergence_range)
                cp = unit.copy()
                m = rng.random(ul) < div
                cp[m] = _BASES[rng.integers(0, 4, size=int(m.sum()))]
                if rng.random() < 0.5:
                    cp = revcom(cp)
                at = int(rng.integers(0, length - ul))
                g[at:at + ul] = cp
                budget -= ul
        out.append(g)
    return out
