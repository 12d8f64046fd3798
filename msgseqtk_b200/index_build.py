"""Host-side preparation of an FMD-index view from chromosome sequences.

MSGseqTK builds its DB on the host (msgseqtk-build); the mapping path only
reads it. This module produces the same decoded view of that DB -- BD text
layout, suffix array, BWT, base counts, the reference's SA sample set and the
chromosome table -- so workloads can be generated without the reference
toolchain. The suffix array is unique for a given text, so the BWT and samples
equal the ones FMDIndex(mtg.getBDSeq(), true, 32) would build
(FMDIndex.cpp:29-116, :465-480); tests check this against the reference.

The BD text of a chromosome is [seq][0][revcom(seq)][0] with IUPAC codes
reduced by DNAalphabet::toBasic (MetaGenome.cpp:104-113).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .synth import revcom

SA_SAMPLE_RATE = 32  # FMDIndex.h:347-348
_TO_BASIC = np.array([0, 1, 2, 2, 4, 4, 4, 4, 8, 8, 8, 8, 8, 8, 8, 15], dtype=np.uint8)


@dataclass
class FmdView:
    n: int
    bwt: np.ndarray          # uint8 nt16 codes, length n
    B: np.ndarray            # int64[16] base counts
    sample_rows: np.ndarray  # int64, rows with i % 32 == 0 or bwt[i] == 0
    sample_vals: np.ndarray  # int64 SA values at those rows
    bd_start: np.ndarray     # int64 per chromosome
    bd_end: np.ndarray
    chr_len: np.ndarray
    chr_seq: np.ndarray      # uint8 forward chromosome sequences, concatenated
    chr_off: np.ndarray      # int64, n_chrom + 1
    gap_sa: np.ndarray | None = None  # SA values of the B[0] '$'-suffix rows (FMDIndex::gapSA)


def bd_text(chroms) -> np.ndarray:
    parts = []
    for s in chroms:
        b = _TO_BASIC[s]
        parts += [b, np.zeros(1, np.uint8), revcom(b), np.zeros(1, np.uint8)]
    return np.concatenate(parts)


# Largest array torch.sort and the scans below take in one call (index
# arithmetic in 32 bits); longer arrays go through _sort_keys' partitions.
SORT_LIMIT = 1 << 30


def _sort_keys(key: torch.Tensor, chunk: int, limit: int = SORT_LIMIT):
    """torch.sort(key) (values and source positions) for arrays of any
    length: keys are partitioned by their top bits into ranges of at most
    `limit` elements, each range gathered, sorted and written at its place.
    Equal keys may come out in any order (the callers only need the order of
    distinct keys)."""
    n = key.numel()
    if n <= limit:
        return torch.sort(key)
    dev = key.device
    mx = int(key.max().item())
    shift = max(0, mx.bit_length() - 16)
    nb = (mx >> shift) + 1
    hist = torch.zeros(nb, dtype=torch.int64, device=dev)
    for a in range(0, n, chunk):
        hist += torch.bincount(key[a:a + chunk] >> shift, minlength=nb)
    counts = hist.cpu().numpy()
    # consecutive buckets grouped into ranges of at most `limit` keys
    groups, lo, size = [], 0, 0
    for b in range(nb):
        c = int(counts[b])
        if c > limit:
            raise ValueError("suffix array: one key bucket exceeds the sort limit")
        if size + c > limit:
            groups.append((lo, b, size))
            lo, size = b, 0
        size += c
    groups.append((lo, nb, size))
    out_key = torch.empty_like(key)
    out_idx = torch.empty(n, dtype=torch.int64, device=dev)
    off = 0
    for blo, bhi, size in groups:
        if size == 0:
            continue
        ks, ix = [], []
        for a in range(0, n, chunk):
            kk = key[a:a + chunk]
            bk = kk >> shift
            sel = torch.nonzero((bk >= blo) & (bk < bhi)).flatten()
            ks.append(kk[sel])
            ix.append(sel + a)
            del bk, sel
        kg = torch.cat(ks)
        ig = torch.cat(ix)
        del ks, ix
        sk, perm = torch.sort(kg)
        out_key[off:off + size] = sk
        out_idx[off:off + size] = ig[perm]
        off += size
        del kg, ig, sk, perm
    return out_key, out_idx


def suffix_array(text: np.ndarray, device: str | torch.device = "cpu", chunk: int = 1 << 28,
                 sort_limit: int = SORT_LIMIT) -> torch.Tensor:
    """Suffix array of a byte string by prefix doubling (standard order: a
    suffix that is a proper prefix of another sorts first). Returns int64 on
    `device`. Elementwise work runs in chunks of `chunk` elements and in
    place, so that at most a few n-element int64 arrays are alive at once
    (texts of 3 G symbols on one GPU)."""
    n = int(text.shape[0])
    dev = torch.device(device)
    # 0 = past the end, 1 + distinct symbol index otherwise
    uniq = np.unique(text)
    lut = np.zeros(256, dtype=np.uint8)
    lut[uniq] = np.arange(1, len(uniq) + 1, dtype=np.uint8)
    bits = max(1, int(len(uniq)).bit_length())
    k = 63 // bits
    code = torch.zeros(n + k, dtype=torch.uint8, device=dev)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        code[a:b] = torch.from_numpy(lut[text[a:b]]).to(dev)
    key = torch.zeros(n, dtype=torch.int64, device=dev)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        kk = key[a:b]
        for j in range(k):
            kk <<= bits
            kk |= code[a + j:b + j].to(torch.int64)
    del code
    h = k
    sorted_key, sa = _sort_keys(key, chunk, sort_limit)
    del key
    while True:
        # group number of each sorted position: 1 + count of key changes before it
        grp = torch.empty(n, dtype=torch.int64, device=dev)
        grp[0] = 1
        for a in range(1, n, chunk):
            b = min(n, a + chunk)
            grp[a:b] = (sorted_key[a:b] != sorted_key[a - 1:b - 1]).to(torch.int64)
        del sorted_key
        carry = 0
        for a in range(0, n, chunk):  # running sum, chunk by chunk
            g = grp[a:a + chunk]
            torch.cumsum(g, 0, out=g)
            g += carry
            carry = int(g[-1].item())
        rank = torch.empty(n, dtype=torch.int64, device=dev)
        for a in range(0, n, chunk):
            rank[sa[a:a + chunk]] = grp[a:a + chunk]
        ngroups = int(grp[-1].item())
        del grp
        if ngroups == n:
            break
        # key = rank * (n + 1) + rank of the suffix h further (0 past the end)
        del sa
        key = torch.empty(n, dtype=torch.int64, device=dev)
        for a in range(0, n, chunk):
            b = min(n, a + chunk)
            kk = key[a:b]
            torch.mul(rank[a:b], n + 1, out=kk)
            lo, hi = a + h, min(n, b + h)
            if lo < hi:
                kk[:hi - lo] += rank[lo:hi]
        del rank  # rebuilt from the sorted keys; only key and the sort's buffers live during the sort
        if dev.type == "cuda":
            torch.cuda.empty_cache()
        sorted_key, sa = _sort_keys(key, chunk, sort_limit)
        del key
        h *= 2
    del rank
    return sa


def build_view(chroms, device: str | torch.device = "cpu") -> FmdView:
    text = bd_text(chroms)
    n = int(text.shape[0])
    sa_t = suffix_array(text, device)
    dev = sa_t.device
    text_t = torch.from_numpy(text).to(dev)
    chunk = 1 << 28
    bwt = np.empty(n, dtype=np.uint8)
    rows_l, vals_l = [], []
    for a in range(0, n, chunk):  # BWT and the SA sample set, chunk by chunk
        b = min(n, a + chunk)
        s_c = sa_t[a:b]
        bw = torch.where(s_c == 0, torch.zeros((), dtype=torch.uint8, device=dev), text_t[(s_c - 1).clamp_min(0)])
        r = torch.nonzero((torch.arange(a, b, device=dev) % SA_SAMPLE_RATE == 0) | (bw == 0)).flatten()
        rows_l.append((r + a).cpu().numpy().astype(np.int64))
        vals_l.append(s_c[r].cpu().numpy().astype(np.int64))
        bwt[a:b] = bw.cpu().numpy()
        del s_c, bw, r
    gap_sa = sa_t[: 2 * len(chroms)].cpu().numpy().astype(np.int64)
    rows = np.concatenate(rows_l)
    vals = np.concatenate(vals_l)
    del sa_t, text_t
    if torch.cuda.is_available():
        torch.cuda.empty_cache()
    B = np.bincount(text, minlength=16).astype(np.int64)[:16]
    lens = np.array([len(s) for s in chroms], dtype=np.int64)
    span = 2 * (lens + 1)
    bd_end = np.cumsum(span)
    bd_start = bd_end - span
    chr_off = np.zeros(len(chroms) + 1, dtype=np.int64)
    np.cumsum(lens, out=chr_off[1:])
    chr_seq = np.concatenate(chroms).astype(np.uint8)
    return FmdView(n, bwt, B, rows, vals, bd_start.astype(np.int64), bd_end.astype(np.int64), lens, chr_seq, chr_off,
                   gap_sa)
