"""ctypes bindings for the two CPU checkers (TEST INFRASTRUCTURE):

* ``Oracle`` -- the project's C++ restatement of the reference path
  (oracle/msg_oracle.cpp -> oracle/build/libmsgoracle.so);
* ``Reference`` -- the reference's own sources compiled in place
  (oracle/ref/Makefile -> oracle/_ref/libmsgref.so).

Only tests, the smoke check and the bench's CPU-baseline leg use these.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "build", "libmsgoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmsgref.so")
# the reference's source tree (read-only); MSG_REFERENCE_SRC overrides it
REF_SRC = os.environ.get("MSG_REFERENCE_SRC", "/root/reference/src")

i64p = C.POINTER(C.c_int64)
u8p = C.POINTER(C.c_uint8)


def _p(a, t):
    return a.ctypes.data_as(t)


def build_oracle() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return ORACLE_SO


def build_reference() -> str | None:
    """Compile the reference when its sources are present (this build
    container); elsewhere the prebuilt library is used if it exists."""
    if os.path.isdir(REF_SRC):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(HERE, "ref"), f"REF={REF_SRC}"], check=True)
    return REF_SO if os.path.exists(REF_SO) else None


class OrcAln(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("tid", "strand", "t_start", "t_end", "aln_from", "aln_to",
                                         "aln_start", "aln_end")] + [("aln_score", C.c_double)] + \
               [(n, C.c_int64) for n in ("n_cigar", "cigar_off", "md_off", "md_len", "flags")]


class RefAln(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("tid", "strand", "t_start", "t_end", "aln_from", "aln_to",
                                         "aln_start", "aln_end")] + [("aln_score", C.c_double)] + \
               [(n, C.c_int64) for n in ("n_cigar", "cigar_off", "md_off", "md_len")]


def _aln_records(arr, n, cg, md):
    out = []
    for k in range(n):
        a = arr[k]
        cig = [int(x) for x in cg[a.cigar_off:a.cigar_off + a.n_cigar]]
        mds = bytes(md[a.md_off:a.md_off + a.md_len]).decode()
        out.append(dict(tid=a.tid, strand=a.strand, t_start=a.t_start, t_end=a.t_end, aln_from=a.aln_from,
                        aln_to=a.aln_to, aln_start=a.aln_start, aln_end=a.aln_end, aln_score=a.aln_score,
                        cigar=cig, md=mds))
    return out


class Oracle:
    def __init__(self, view, so: str = ORACLE_SO):
        if not os.path.exists(so):
            build_oracle()
        self.lib = L = C.CDLL(so)
        L.orc_index_create.restype = C.c_void_p
        L.orc_index_create.argtypes = [C.c_int64, u8p, i64p, C.c_int64, i64p, i64p, C.c_int64, i64p, i64p,
                                       i64p, u8p, i64p]
        L.orc_index_free.argtypes = [C.c_void_p]
        L.orc_rank.restype = C.c_int64
        L.orc_rank.argtypes = [C.c_void_p, C.c_int, C.c_int64]
        for f in (L.orc_back_ext, L.orc_fwd_ext):
            f.restype = C.c_int64
            f.argtypes = [C.c_void_p, i64p, i64p, i64p, C.c_int]
        L.orc_access_sa.restype = C.c_int64
        L.orc_access_sa.argtypes = [C.c_void_p, C.c_int64]
        L.orc_loglik.restype = C.c_double
        L.orc_loglik.argtypes = [C.c_void_p, C.c_int]
        L.orc_find_smems.restype = C.c_int64
        L.orc_find_smems.argtypes = [C.c_void_p, u8p, C.c_int64, C.c_int64, C.c_double, i64p, C.c_int64]
        L.orc_find_seeds.restype = C.c_int64
        L.orc_find_seeds.argtypes = [C.c_void_p, u8p, C.c_int64, C.c_int64, C.c_double, C.c_int64, i64p, C.c_int64]
        L.orc_find_mems.restype = C.c_int64
        L.orc_find_mems.argtypes = [C.c_void_p, u8p, C.c_int64, C.c_int64, C.c_double, i64p, C.c_int64,
                                    C.POINTER(C.c_double)]
        L.orc_get_chains.restype = C.c_int64
        L.orc_get_chains.argtypes = [i64p, C.c_int64, C.c_int64, C.c_int64, i64p, i64p, C.c_int64, C.c_int64]
        L.orc_align_read.restype = C.c_int64
        L.orc_align_read.argtypes = [C.c_void_p, u8p, C.c_int64, C.c_int64, C.c_double, C.c_int64, C.c_int,
                                     C.POINTER(C.c_int32), C.POINTER(OrcAln), C.c_int64, C.POINTER(C.c_uint32),
                                     C.c_int64, i64p, C.c_char_p, C.c_int64, i64p]
        L.orc_map_batch.restype = C.c_int64
        L.orc_map_batch.argtypes = [C.c_void_p, C.c_int64, u8p, i64p, C.c_int64, C.c_double, C.c_int64, C.c_int,
                                    i64p, i64p]
        self.view = v = view
        self._keep = [np.ascontiguousarray(x) for x in (v.bwt, v.B, v.sample_rows, v.sample_vals, v.bd_start,
                                                        v.bd_end, v.chr_len, v.chr_seq, v.chr_off)]
        k = self._keep
        self.h = L.orc_index_create(v.n, _p(k[0], u8p), _p(k[1], i64p), len(k[2]), _p(k[2], i64p),
                                    _p(k[3], i64p), len(k[4]), _p(k[4], i64p), _p(k[5], i64p), _p(k[6], i64p),
                                    _p(k[7], u8p), _p(k[8], i64p))

    def __del__(self):
        try:
            self.lib.orc_index_free(self.h)
        except Exception:
            pass

    def rank(self, b, i):
        return self.lib.orc_rank(self.h, b, i)

    def back_ext(self, p, q, s, b):
        P, Q, S = C.c_int64(p), C.c_int64(q), C.c_int64(s)
        r = self.lib.orc_back_ext(self.h, C.byref(P), C.byref(Q), C.byref(S), b)
        return r, P.value, Q.value, S.value

    def fwd_ext(self, p, q, s, b):
        P, Q, S = C.c_int64(p), C.c_int64(q), C.c_int64(s)
        r = self.lib.orc_fwd_ext(self.h, C.byref(P), C.byref(Q), C.byref(S), b)
        return r, P.value, Q.value, S.value

    def access_sa(self, i):
        return self.lib.orc_access_sa(self.h, i)

    def loglik(self, b):
        return self.lib.orc_loglik(self.h, b)

    def smems(self, read, min_len=17, max_evalue=0.01):
        read = np.ascontiguousarray(read, dtype=np.uint8)
        cap = 4 * len(read) + 64
        while True:
            out = np.zeros((cap, 6), dtype=np.int64)
            n = self.lib.orc_find_smems(self.h, _p(read, u8p), len(read), min_len, max_evalue, _p(out, i64p), cap)
            if n <= cap:
                return out[:n]
            cap = n

    def mems(self, read, min_len=17, max_evalue=0.01):
        """SMEM_LIST::findMEMS rows (6 int64) and the list's loglik."""
        read = np.ascontiguousarray(read, dtype=np.uint8)
        cap = len(read) + 2
        out = np.zeros((cap, 6), dtype=np.int64)
        ll = C.c_double(0)
        n = self.lib.orc_find_mems(self.h, _p(read, u8p), len(read), min_len, max_evalue, _p(out, i64p), cap, C.byref(ll))
        assert n <= cap
        return out[:n], ll.value

    def seeds(self, read, min_len=17, max_evalue=0.01, max_nseed=500):
        read = np.ascontiguousarray(read, dtype=np.uint8)
        cap = 4096
        while True:
            out = np.zeros((cap, 6), dtype=np.int64)
            n = self.lib.orc_find_seeds(self.h, _p(read, u8p), len(read), min_len, max_evalue, max_nseed,
                                        _p(out, i64p), cap)
            if n <= cap:
                return out[:n]
            cap = n

    def chains(self, seeds, max_mm, max_indel):
        seeds = np.ascontiguousarray(seeds, dtype=np.int64)
        cc, ci = 1024, 1 << 16
        while True:
            off = np.zeros(cc + 1, dtype=np.int64)
            idx = np.zeros(ci, dtype=np.int64)
            n = self.lib.orc_get_chains(_p(seeds, i64p), len(seeds), max_mm, max_indel, _p(off, i64p),
                                        _p(idx, i64p), cc, ci)
            if n <= cc and off[n] <= ci:
                return [idx[off[k]:off[k + 1]].copy() for k in range(n)]
            cc, ci = max(cc, n) * 2, ci * 4

    def align_read(self, read, min_len=17, max_evalue=0.01, max_nseed=500, mode=0, score=(1, 3, 5, 2)):
        read = np.ascontiguousarray(read, dtype=np.uint8)
        sc = (C.c_int32 * 4)(*score)
        cap, ccap, mcap = 256, 1 << 16, 1 << 16
        while True:
            arr = (OrcAln * cap)()
            cg = np.zeros(ccap, dtype=np.uint32)
            md = C.create_string_buffer(mcap)
            cu, mu = C.c_int64(0), C.c_int64(0)
            n = self.lib.orc_align_read(self.h, _p(read, u8p), len(read), min_len, max_evalue, max_nseed, mode, sc,
                                        arr, cap, cg.ctypes.data_as(C.POINTER(C.c_uint32)), ccap, C.byref(cu),
                                        md, mcap, C.byref(mu))
            if n <= cap and cu.value <= ccap and mu.value <= mcap:
                recs = _aln_records(arr, n, cg, md.raw)
                for k in range(n):
                    recs[k]["flags"] = arr[k].flags
                return recs
            cap, ccap, mcap = max(cap, n) * 2, max(ccap, cu.value) * 2, max(mcap, mu.value) * 2

    def map_batch(self, reads, offs, n_threads=1, min_len=17, max_evalue=0.01, max_nseed=500):
        reads = np.ascontiguousarray(reads, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.int64)
        na, nc = C.c_int64(0), C.c_int64(0)
        m = self.lib.orc_map_batch(self.h, len(offs) - 1, _p(reads, u8p), _p(offs, i64p), min_len, max_evalue,
                                   max_nseed, n_threads, C.byref(na), C.byref(nc))
        return m, na.value, nc.value


class Reference:
    """The reference's own code path (compiled from its sources)."""

    def __init__(self, chroms, so: str = REF_SO, view=None):
        """Build the reference DB for `chroms`: with the reference's own
        FMDIndex constructor (divsufsort), or, when `view` is given, from that
        decoded view through the reference's WaveletTreeRRR/BitSeqRRR."""
        self.lib = L = C.CDLL(so)
        L.ref_db_build.restype = C.c_void_p
        L.ref_db_build.argtypes = [C.c_int64, u8p, i64p]
        L.ref_db_free.argtypes = [C.c_void_p]
        for f in (L.ref_db_length, L.ref_db_num_chroms):
            f.restype = C.c_int64
            f.argtypes = [C.c_void_p]
        L.ref_db_counts.argtypes = [C.c_void_p, i64p, i64p]
        L.ref_db_bwt.argtypes = [C.c_void_p, u8p]
        L.ref_db_bdseq.argtypes = [C.c_void_p, u8p]
        L.ref_db_access_sa.restype = C.c_int64
        L.ref_db_access_sa.argtypes = [C.c_void_p, C.c_int64]
        L.ref_db_rank.restype = C.c_int64
        L.ref_db_rank.argtypes = [C.c_void_p, C.c_int64, C.c_int64]
        L.ref_db_sa_samples.restype = C.c_int64
        L.ref_db_sa_samples.argtypes = [C.c_void_p, i64p, i64p, C.c_int64]
        L.ref_db_chroms.argtypes = [C.c_void_p, i64p, i64p, i64p]
        for f in (L.ref_back_ext, L.ref_fwd_ext):
            f.restype = C.c_int64
            f.argtypes = [C.c_void_p, i64p, i64p, i64p, C.c_int]
        L.ref_loglik.restype = C.c_double
        L.ref_loglik.argtypes = [C.c_void_p, C.c_int]
        L.ref_find_smems.restype = C.c_int64
        L.ref_find_smems.argtypes = [C.c_void_p, u8p, C.c_int64, C.c_int64, C.c_double, i64p, C.c_int64]
        L.ref_find_seeds.restype = C.c_int64
        L.ref_find_seeds.argtypes = [C.c_void_p, u8p, C.c_int64, C.c_int64, C.c_double, C.c_int64, i64p, C.c_int64]
        L.ref_find_mems.restype = C.c_int64
        L.ref_find_mems.argtypes = [C.c_void_p, u8p, C.c_int64, C.c_int64, C.c_double, i64p, C.c_int64,
                                    C.POINTER(C.c_double)]
        L.ref_clean_batch.restype = C.c_int64
        L.ref_clean_batch.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, u8p, i64p, u8p, i64p, C.c_int64, C.c_double,
                                      C.c_double, C.c_int] + [C.POINTER(C.c_double)] * 3 + [u8p,
                                                                                           C.POINTER(C.c_double)]
        L.ref_get_chains.restype = C.c_int64
        L.ref_get_chains.argtypes = [i64p, C.c_int64, C.c_int64, C.c_int64, i64p, i64p, C.c_int64, C.c_int64]
        L.ref_align_read.restype = C.c_int64
        L.ref_align_read.argtypes = [C.c_void_p, u8p, C.c_int64, C.c_int64, C.c_double, C.c_int64, C.c_int,
                                     C.POINTER(RefAln), C.c_int64, C.POINTER(C.c_uint32), C.c_int64, i64p,
                                     C.c_char_p, C.c_int64, i64p]
        L.ref_map_batch.restype = C.c_int64
        L.ref_map_batch.argtypes = [C.c_void_p, C.c_int64, u8p, u8p, i64p, C.c_int64, C.c_double, C.c_int64,
                                    C.c_double, C.c_int, C.POINTER(C.c_double), i64p]
        L.ref_max_threads.restype = C.c_int
        L.ref_db_save.restype = C.c_int
        L.ref_db_save.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p]
        L.ref_sam_batch.restype = C.c_int64
        L.ref_sam_batch.argtypes = [C.c_void_p, C.c_int64, u8p, u8p, i64p, C.c_int64, C.c_double, C.c_int64,
                                    C.c_double, C.c_int, C.c_char_p, C.c_int64]
        ip = C.POINTER(C.c_int)
        L.ref_sam_pe_batch.restype = C.c_int64
        L.ref_sam_pe_batch.argtypes = [C.c_void_p, C.c_int64, u8p, u8p, i64p, C.c_int64, C.c_double, C.c_int64,
                                       C.c_double, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, ip,
                                       C.c_int64, C.c_char_p, C.c_int64]
        L.ref_sam_pe_from_records.restype = C.c_int64
        L.ref_sam_pe_from_records.argtypes = [C.c_void_p, C.c_int64, u8p, u8p, i64p, C.c_void_p,
                                              C.POINTER(C.c_uint32), i64p, C.c_double, C.c_int, C.c_double,
                                              C.c_double, C.c_double, C.c_double, ip, C.c_int64, C.c_char_p,
                                              C.c_int64]
        L.ref_clean_assign.restype = C.c_int64
        L.ref_clean_assign.argtypes = [C.c_void_p, C.c_void_p, C.c_char_p, C.c_int64, C.c_int64, C.c_double,
                                       C.c_char_p, C.c_int64]
        L.ref_fastq_rewrite.restype = C.c_int64
        L.ref_fastq_rewrite.argtypes = [C.c_char_p, C.c_int64, u8p, C.c_char_p, C.c_int64]
        L.ref_fastq_parse.restype = C.c_int64
        L.ref_fastq_parse.argtypes = [C.c_char_p, C.c_int64, C.c_char_p, C.c_int64]
        L.ref_sam_from_records.restype = C.c_int64
        L.ref_sam_from_records.argtypes = [C.c_void_p, C.c_int64, u8p, u8p, i64p, C.c_void_p, C.POINTER(C.c_uint32),
                                           i64p, C.c_double, C.c_int, C.c_char_p, C.c_int64]
        seqs = np.ascontiguousarray(np.concatenate(chroms).astype(np.uint8))
        offs = np.zeros(len(chroms) + 1, dtype=np.int64)
        np.cumsum([len(c) for c in chroms], out=offs[1:])
        L.ref_db_from_view.restype = C.c_void_p
        L.ref_db_from_view.argtypes = [C.c_int64, u8p, i64p, C.c_int64, u8p, i64p, C.c_int64, i64p, i64p, i64p]
        if view is None:
            self.h = L.ref_db_build(len(chroms), _p(seqs, u8p), _p(offs, i64p))
        else:
            k = [np.ascontiguousarray(x) for x in (view.bwt, view.B.astype(np.int64), view.sample_rows,
                                                   view.sample_vals, view.gap_sa)]
            self.h = L.ref_db_from_view(len(chroms), _p(seqs, u8p), _p(offs, i64p), view.n, _p(k[0], u8p),
                                        _p(k[1], i64p), len(k[2]), _p(k[2], i64p), _p(k[3], i64p), _p(k[4], i64p))
        self.n = L.ref_db_length(self.h)

    @classmethod
    def merged(cls, chroms_a, chroms_b, so: str = REF_SO):
        """The DB msgseqtk-mergedb makes from a DB of chroms_a and one of
        chroms_b (MetaGenome/FMDIndex append, updateIndex, buildSA)."""
        self = cls.__new__(cls)
        self.lib = L = cls(chroms_a[:1], so).lib  # declares the signatures
        L.ref_db_merge.restype = C.c_void_p
        L.ref_db_merge.argtypes = [C.c_int64, u8p, i64p, C.c_int64, u8p, i64p]
        keep = []
        args = []
        for ch in (chroms_a, chroms_b):
            seqs = np.ascontiguousarray(np.concatenate(ch).astype(np.uint8))
            offs = np.zeros(len(ch) + 1, dtype=np.int64)
            np.cumsum([len(c) for c in ch], out=offs[1:])
            keep += [seqs, offs]
            args += [len(ch), _p(seqs, u8p), _p(offs, i64p)]
        self.h = L.ref_db_merge(*args)
        self.n = L.ref_db_length(self.h)
        return self

    def __del__(self):
        try:
            self.lib.ref_db_free(self.h)
        except Exception:
            pass

    def counts(self):
        B = np.zeros(256, dtype=np.int64)
        Cc = np.zeros(256, dtype=np.int64)
        self.lib.ref_db_counts(self.h, _p(B, i64p), _p(Cc, i64p))
        return B, Cc

    def bwt(self):
        out = np.zeros(self.n, dtype=np.uint8)
        self.lib.ref_db_bwt(self.h, _p(out, u8p))
        return out

    def bdseq(self):
        out = np.zeros(self.n, dtype=np.uint8)
        self.lib.ref_db_bdseq(self.h, _p(out, u8p))
        return out

    def sa_samples(self):
        cap = self.n // 16 + 1024
        rows = np.zeros(cap, dtype=np.int64)
        vals = np.zeros(cap, dtype=np.int64)
        k = self.lib.ref_db_sa_samples(self.h, _p(rows, i64p), _p(vals, i64p), cap)
        return rows[:k], vals[:k]

    def chroms(self):
        nc = self.lib.ref_db_num_chroms(self.h)
        a, b, c = (np.zeros(nc, dtype=np.int64) for _ in range(3))
        self.lib.ref_db_chroms(self.h, _p(a, i64p), _p(b, i64p), _p(c, i64p))
        return a, b, c

    def rank(self, b, i):
        return self.lib.ref_db_rank(self.h, b, i)

    def access_sa(self, i):
        return self.lib.ref_db_access_sa(self.h, i)

    def back_ext(self, p, q, s, b):
        P, Q, S = C.c_int64(p), C.c_int64(q), C.c_int64(s)
        r = self.lib.ref_back_ext(self.h, C.byref(P), C.byref(Q), C.byref(S), b)
        return r, P.value, Q.value, S.value

    def fwd_ext(self, p, q, s, b):
        P, Q, S = C.c_int64(p), C.c_int64(q), C.c_int64(s)
        r = self.lib.ref_fwd_ext(self.h, C.byref(P), C.byref(Q), C.byref(S), b)
        return r, P.value, Q.value, S.value

    def loglik(self, b):
        return self.lib.ref_loglik(self.h, b)

    def smems(self, read, min_len=17, max_evalue=0.01):
        read = np.ascontiguousarray(read, dtype=np.uint8)
        cap = 4 * len(read) + 64
        while True:
            out = np.zeros((cap, 6), dtype=np.int64)
            n = self.lib.ref_find_smems(self.h, _p(read, u8p), len(read), min_len, max_evalue, _p(out, i64p), cap)
            if n <= cap:
                return out[:n]
            cap = n

    def mems(self, read, min_len=17, max_evalue=0.01):
        """SMEM_LIST::findMEMS rows (6 int64) and the list's loglik."""
        read = np.ascontiguousarray(read, dtype=np.uint8)
        cap = len(read) + 2
        out = np.zeros((cap, 6), dtype=np.int64)
        ll = C.c_double(0)
        n = self.lib.ref_find_mems(self.h, _p(read, u8p), len(read), min_len, max_evalue, _p(out, i64p), cap, C.byref(ll))
        assert n <= cap
        return out[:n], ll.value

    def seeds(self, read, min_len=17, max_evalue=0.01, max_nseed=500):
        read = np.ascontiguousarray(read, dtype=np.uint8)
        cap = 4096
        while True:
            out = np.zeros((cap, 6), dtype=np.int64)
            n = self.lib.ref_find_seeds(self.h, _p(read, u8p), len(read), min_len, max_evalue, max_nseed,
                                        _p(out, i64p), cap)
            if n <= cap:
                return out[:n]
            cap = n

    def chains(self, seeds, max_mm, max_indel):
        seeds = np.ascontiguousarray(seeds, dtype=np.int64)
        cc, ci = 1024, 1 << 16
        while True:
            off = np.zeros(cc + 1, dtype=np.int64)
            idx = np.zeros(ci, dtype=np.int64)
            n = self.lib.ref_get_chains(_p(seeds, i64p), len(seeds), max_mm, max_indel, _p(off, i64p),
                                        _p(idx, i64p), cc, ci)
            if n <= cc and off[n] <= ci:
                return [idx[off[k]:off[k + 1]].copy() for k in range(n)]
            cc, ci = max(cc, n) * 2, ci * 4

    def align_read(self, read, min_len=17, max_evalue=0.01, max_nseed=500, mode=0):
        read = np.ascontiguousarray(read, dtype=np.uint8)
        cap, ccap, mcap = 256, 1 << 16, 1 << 16
        while True:
            arr = (RefAln * cap)()
            cg = np.zeros(ccap, dtype=np.uint32)
            md = C.create_string_buffer(mcap)
            cu, mu = C.c_int64(0), C.c_int64(0)
            n = self.lib.ref_align_read(self.h, _p(read, u8p), len(read), min_len, max_evalue, max_nseed, mode, arr,
                                        cap, cg.ctypes.data_as(C.POINTER(C.c_uint32)), ccap, C.byref(cu), md, mcap,
                                        C.byref(mu))
            if n <= cap and cu.value <= ccap and mu.value <= mcap:
                return _aln_records(arr, n, cg, md.raw)
            cap, ccap, mcap = max(cap, n) * 2, max(ccap, cu.value) * 2, max(mcap, mu.value) * 2

    def save(self, mtg_path, mgs_path, fmd_path):
        """Write the DB files as msgseqtk-build does."""
        rc = self.lib.ref_db_save(self.h, str(mtg_path).encode(), str(mgs_path).encode(), str(fmd_path).encode())
        if rc != 0:
            raise RuntimeError(f"ref_db_save failed ({rc})")

    @staticmethod
    def _text(fn):
        cap = 1 << 20
        while True:
            buf = C.create_string_buffer(cap)
            n = fn(buf, cap)
            if n <= cap:
                return buf.raw[:n].decode().splitlines()
            cap = n + 1

    def sam_batch(self, reads, quals, offs, min_len=17, max_evalue=0.01, max_nseed=500, min_score_rate=0.65,
                  max_report=1):
        """SAM records (text lines, see ref_harness.cpp) of the reference's
        single-end path."""
        reads = np.ascontiguousarray(reads, dtype=np.uint8)
        quals = np.ascontiguousarray(quals, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.int64)
        return self._text(lambda b, cap: self.lib.ref_sam_batch(
            self.h, len(offs) - 1, _p(reads, u8p), _p(quals, u8p), _p(offs, i64p), min_len, max_evalue, max_nseed,
            min_score_rate, max_report, b, cap))

    def sam_from_records(self, reads, quals, offs, aln, cigar, read_aln_off, min_score_rate=0.65, max_report=1):
        """SAM records from alignment records of the CUDA library, through the
        reference's own tail (filter, evaluate, calcMapQ, sort, exportBAM)."""
        reads = np.ascontiguousarray(reads, dtype=np.uint8)
        quals = np.ascontiguousarray(quals, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.int64)
        aln = np.ascontiguousarray(aln)
        cigar = np.ascontiguousarray(cigar, dtype=np.uint32)
        roff = np.ascontiguousarray(read_aln_off, dtype=np.int64)
        return self._text(lambda b, cap: self.lib.ref_sam_from_records(
            self.h, len(offs) - 1, _p(reads, u8p), _p(quals, u8p), _p(offs, i64p), aln.ctypes.data,
            cigar.ctypes.data_as(C.POINTER(C.c_uint32)), _p(roff, i64p), min_score_rate, max_report, b, cap))

    def fastq_parse(self, text: bytes):
        """The reference's FASTQ reading: lines "name\tdesc\tSEQHEX\tQUALHEX"
        (split on '\n' only: names and descriptions may hold '\r')."""
        cap = 4 * len(text) + 1024
        buf = C.create_string_buffer(cap)
        n = self.lib.ref_fastq_parse(text, len(text), buf, cap)
        assert n <= cap
        out = buf.raw[:n].decode("latin-1")
        return out.split("\n")[:-1] if out else []

    def clean_assign(self, bg, text: bytes, min_len=17, max_evalue=0.01) -> bytes:
        """msgseqtk-clean's assignment lines for the reads of a FASTQ text."""
        cap = 4 * len(text) + 1024
        buf = C.create_string_buffer(cap)
        n = self.lib.ref_clean_assign(self.h, bg.h, text, len(text), min_len, max_evalue, buf, cap)
        assert n <= cap
        return buf.raw[:n]

    def fastq_rewrite(self, text: bytes, keep=None) -> bytes:
        """The reference reading FASTQ text and writing the kept reads back."""
        cap = 4 * len(text) + 1024
        buf = C.create_string_buffer(cap)
        kp = None if keep is None else np.ascontiguousarray(keep, dtype=np.uint8)
        n = self.lib.ref_fastq_rewrite(text, len(text), _p(kp, u8p) if kp is not None else None, buf, cap)
        assert n <= cap
        return buf.raw[:n]

    @staticmethod
    def _pairing(pairing):
        """(mean, sd, min, max, opt[5], max_npair) from a dict; defaults are
        PairingScheme's after msgseqtk-align's option handling without -m/-d:
        mean 200, sd 20, range [0, 400], every pair kind allowed."""
        p = dict(mean=200.0, sd=20.0, min=0.0, max=400.0, no_mixed=0, no_discordant=0, no_tail_over=0,
                 no_contain=0, no_overlap=0, max_npair=0)
        p.update(pairing or {})
        opt = (C.c_int * 5)(p["no_mixed"], p["no_discordant"], p["no_tail_over"], p["no_contain"], p["no_overlap"])
        return p["mean"], p["sd"], p["min"], p["max"], opt, p["max_npair"]

    def sam_pe_batch(self, reads, quals, offs, min_len=17, max_evalue=0.01, max_nseed=500, min_score_rate=0.65,
                     max_report=1, pairing=None):
        """SAM records of the reference's paired-end path; reads 2i and 2i+1
        are the mates of pair i."""
        reads = np.ascontiguousarray(reads, dtype=np.uint8)
        quals = np.ascontiguousarray(quals, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.int64)
        m, sd, lo, hi, opt, mx = self._pairing(pairing)
        return self._text(lambda b, cap: self.lib.ref_sam_pe_batch(
            self.h, (len(offs) - 1) // 2, _p(reads, u8p), _p(quals, u8p), _p(offs, i64p), min_len, max_evalue,
            max_nseed, min_score_rate, max_report, m, sd, lo, hi, opt, mx, b, cap))

    def sam_pe_from_records(self, reads, quals, offs, aln, cigar, read_aln_off, min_score_rate=0.65, max_report=1,
                            pairing=None):
        """The reference's paired-end tail on alignment records of the CUDA
        library (mates at reads 2i, 2i+1)."""
        reads = np.ascontiguousarray(reads, dtype=np.uint8)
        quals = np.ascontiguousarray(quals, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.int64)
        aln = np.ascontiguousarray(aln)
        cigar = np.ascontiguousarray(cigar, dtype=np.uint32)
        roff = np.ascontiguousarray(read_aln_off, dtype=np.int64)
        m, sd, lo, hi, opt, mx = self._pairing(pairing)
        return self._text(lambda b, cap: self.lib.ref_sam_pe_from_records(
            self.h, (len(offs) - 1) // 2, _p(reads, u8p), _p(quals, u8p), _p(offs, i64p), aln.ctypes.data,
            cigar.ctypes.data_as(C.POINTER(C.c_uint32)), _p(roff, i64p), min_score_rate, max_report, m, sd, lo, hi,
            opt, mx, b, cap))

    def map_batch(self, reads, quals, offs, n_threads=0, min_len=17, max_evalue=0.01, max_nseed=500,
                  min_score_rate=0.65):
        reads = np.ascontiguousarray(reads, dtype=np.uint8)
        quals = np.ascontiguousarray(quals, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.int64)
        sec = C.c_double(0)
        na = C.c_int64(0)
        m = self.lib.ref_map_batch(self.h, len(offs) - 1, _p(reads, u8p), _p(quals, u8p), _p(offs, i64p), min_len,
                                   max_evalue, max_nseed, min_score_rate, n_threads, C.byref(sec), C.byref(na))
        return m, na.value, sec.value

    def clean_batch(self, bg, reads, offs, rev_reads=None, rev_offs=None, min_len=17, max_evalue=0.01, min_lod=0.0,
                    n_threads=0):
        """msgseqtk-clean's task body over a batch (this DB = reference
        genomes, `bg` = background): per read (pair) refLoglik, bgLoglik,
        lod and the keep decision, plus the OpenMP time in seconds."""
        reads = np.ascontiguousarray(reads, dtype=np.uint8)
        offs = np.ascontiguousarray(offs, dtype=np.int64)
        n = len(offs) - 1
        pe = rev_reads is not None
        rr = np.ascontiguousarray(rev_reads if pe else np.zeros(1), dtype=np.uint8)
        ro = np.ascontiguousarray(rev_offs if pe else np.zeros(1), dtype=np.int64)
        out = [np.zeros(n, dtype=np.float64) for _ in range(3)]
        keep = np.zeros(n, dtype=np.uint8)
        sec = C.c_double(0)
        dp = C.POINTER(C.c_double)
        self.lib.ref_clean_batch(self.h, bg.h, n, _p(reads, u8p), _p(offs, i64p), _p(rr, u8p) if pe else None,
                                 _p(ro, i64p) if pe else None, min_len, max_evalue, min_lod, n_threads,
                                 out[0].ctypes.data_as(dp), out[1].ctypes.data_as(dp), out[2].ctypes.data_as(dp),
                                 _p(keep, u8p), C.byref(sec))
        return out[0], out[1], out[2], keep.astype(bool), sec.value
