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


def suffix_array(text: np.ndarray, device: str | torch.device = "cpu") -> torch.Tensor:
    """Suffix array of a byte string by prefix doubling (standard order: a
    suffix that is a proper prefix of another sorts first). Returns int64 on
    `device`."""
    n = int(text.shape[0])
    dev = torch.device(device)
    sym = torch.from_numpy(text.astype(np.int64)).to(dev)
    # 0 = past the end, 1 + distinct symbol index otherwise
    uniq = torch.unique(sym)
    bits = max(1, int(uniq.numel()).bit_length())
    k = 63 // bits
    code = torch.zeros(n + k, dtype=torch.int64, device=dev)
    code[:n] = torch.searchsorted(uniq, sym) + 1
    key = torch.zeros(n, dtype=torch.int64, device=dev)
    for j in range(k):
        key = (key << bits) | code[j:j + n]
    del code, sym
    h = k
    sorted_key, sa = torch.sort(key)
    del key
    rank = torch.empty(n, dtype=torch.int64, device=dev)
    while True:
        flag = torch.ones(n, dtype=torch.int64, device=dev)
        flag[1:] = (sorted_key[1:] != sorted_key[:-1]).to(torch.int64)
        grp = torch.cumsum(flag, 0)
        del flag
        rank[sa] = grp
        ngroups = int(grp[-1].item())
        del grp, sorted_key
        if ngroups == n:
            break
        nxt = torch.zeros(n, dtype=torch.int64, device=dev)
        if h < n:
            nxt[: n - h] = rank[h:]
        key = rank * (n + 1) + nxt
        del nxt
        sorted_key, sa = torch.sort(key)
        del key
        h *= 2
    return sa


def build_view(chroms, device: str | torch.device = "cpu") -> FmdView:
    text = bd_text(chroms)
    n = int(text.shape[0])
    sa_t = suffix_array(text, device)
    text_t = torch.from_numpy(text).to(sa_t.device)
    prev = (sa_t - 1).clamp_min(0)
    bwt_t = torch.where(sa_t == 0, torch.zeros_like(prev, dtype=torch.uint8), text_t[prev])
    del prev
    rows_t = torch.nonzero((torch.arange(n, device=sa_t.device) % SA_SAMPLE_RATE == 0) | (bwt_t == 0)).flatten()
    vals_t = sa_t[rows_t]
    gap_sa = sa_t[: 2 * len(chroms)].cpu().numpy().astype(np.int64)
    bwt = bwt_t.cpu().numpy()
    rows = rows_t.cpu().numpy().astype(np.int64)
    vals = vals_t.cpu().numpy().astype(np.int64)
    del sa_t, bwt_t, rows_t, vals_t, text_t
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
