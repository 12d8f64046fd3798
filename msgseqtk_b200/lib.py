"""ctypes binding of the C ABI in include/msg_b200.h (libmsg_b200.so).

The shared library is built in-tree by msgseqtk_b200/csrc/Makefile; there is
no CPU fallback -- loading fails loudly when the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmsg_b200.so")

MSG_OK, MSG_EINVAL, MSG_ENOMEM, MSG_EUNSUPPORTED, MSG_ETIMEOUT, MSG_ECUDA, MSG_ESTATE, MSG_EINTERNAL = range(8)

i64p = C.POINTER(C.c_int64)
u8p = C.POINTER(C.c_uint8)

ALN_DTYPE = np.dtype([("read", "<i8"), ("tid", "<i4"), ("strand", "<i4"), ("t_start", "<i8"), ("t_end", "<i8"),
                      ("aln_from", "<i8"), ("aln_to", "<i8"), ("aln_start", "<i8"), ("aln_end", "<i8"),
                      ("aln_score", "<i4"), ("flags", "<i4"), ("cigar_off", "<i8"), ("n_cigar", "<i4"),
                      ("pad", "<i4")])
assert ALN_DTYPE.itemsize == 88

# symbols of the C ABI, in include/msg_b200.h order
EXPORTS = ["msg_strerror", "msg_last_error", "msg_ctx_create", "msg_ctx_destroy", "msg_index_load", "msg_db_read",
           "msg_db_views", "msg_db_free", "msg_db_read_device", "msg_db_read_cached", "msg_index_bytes", "msg_ctx_share_index",
           "msg_map_params_default", "msg_map_batch", "msg_map_batches", "msg_seed_batch", "msg_locate_batch",
           "msg_chain_batch", "msg_align_batch", "msg_map_batch_device", "msg_last_stats",
           "msg_result_device", "msg_ctx_stream", "msg_ctx_set_scratch_limit", "msg_ctx_set_dp_shape", "msg_ctx_set_dp_lanes", "msg_ctx_set_dp_occupancy", "msg_ctx_set_smem_shape", "msg_autotune", "msg_smem_batch_noalloc", "msg_band_model_set", "msg_band_collect",
           "msg_band_train", "msg_band_grad", "msg_tail_params_default", "msg_tail_batch", "msg_pair_params_default", "msg_tail_pe_batch",
           "msg_fastq_parse", "msg_fastq_format", "msg_clean_format", "msg_sam_format", "msg_bam_header",
           "msg_bam_format", "msg_bgzf_compress",
           "msg_mem_params_default", "msg_mem_batch", "msg_clean_batch",
           "msg_clean_batch_device", "msg_occ_query", "msg_bi_ext_query", "msg_sa_query"]

SAM_DTYPE = np.dtype([("read", "<i8"), ("flag", "<i4"), ("tid", "<i4"), ("pos", "<i8"), ("mapq", "<i4"),
                      ("as", "<i4"), ("xh", "<f4"), ("xp", "<f4"), ("nh", "<i4"), ("xn", "<i4"),
                      ("cigar_off", "<i8"), ("n_cigar", "<i4"), ("md_len", "<i4"), ("md_off", "<i8"),
                      ("isize", "<i4"), ("pad", "<i4")])
assert SAM_DTYPE.itemsize == 80

# band model (include/msg_b200.h)
BAND_FEATURES, BAND_HIDDEN, BAND_CLASSES, BAND_NPARAMS = 16, 64, 4, 5540
BAND_WIDTHS = (7, 15, 31, None)  # class -> band half-width (None: whole rectangles)


class FmdView(C.Structure):
    _fields_ = [("n", C.c_int64), ("bwt", u8p), ("base_count", i64p), ("n_samples", C.c_int64),
                ("sample_rows", i64p), ("sample_vals", i64p)]


class MtgView(C.Structure):
    _fields_ = [("n_chrom", C.c_int64), ("bd_start", i64p), ("bd_end", i64p), ("chr_len", i64p), ("chr_seq", u8p),
                ("chr_off", i64p)]


class MapParams(C.Structure):
    _fields_ = [("min_len", C.c_int64), ("max_evalue", C.c_double), ("max_nseed", C.c_int64), ("mode", C.c_int32),
                ("match", C.c_double), ("mismatch", C.c_double), ("gap_open", C.c_double), ("gap_ext", C.c_double),
                ("min_score_rate", C.c_double), ("band_mode", C.c_int32), ("band_w", C.c_int32)]


class BandTrainParams(C.Structure):
    _fields_ = [("epochs", C.c_int32), ("batch", C.c_int32), ("lr", C.c_float), ("seed", C.c_uint64)]


class TailParams(C.Structure):
    _fields_ = [("min_score_rate", C.c_double), ("max_report", C.c_uint32), ("n_threads", C.c_int32),
                ("gap_open", C.c_double), ("gap_ext", C.c_double), ("clip", C.c_double)]


class PairParams(C.Structure):
    _fields_ = [("mean", C.c_double), ("sd", C.c_double), ("min_ins", C.c_double), ("max_ins", C.c_double),
                ("no_mixed", C.c_int32), ("no_discordant", C.c_int32), ("no_tail_over", C.c_int32),
                ("no_contain", C.c_int32), ("no_overlap", C.c_int32), ("pad", C.c_int32), ("max_npair", C.c_int64)]


class FastqBatch(C.Structure):
    _fields_ = [("cap_reads", C.c_int64), ("cap_bases", C.c_int64), ("cap_text", C.c_int64), ("seq", u8p),
                ("qual", u8p), ("off", i64p), ("text", C.c_char_p), ("name_off", i64p), ("n_reads", C.c_int64),
                ("n_bases", C.c_int64), ("n_text", C.c_int64)]


class MemParams(C.Structure):
    _fields_ = [("min_len", C.c_int64), ("max_evalue", C.c_double)]


class ReadBatch(C.Structure):
    _fields_ = [("n_reads", C.c_int64), ("seq", u8p), ("off", i64p)]


class AlnOut(C.Structure):
    _fields_ = [("aln_cap", C.c_int64), ("aln", C.c_void_p), ("cigar_cap", C.c_int64), ("cigar", C.c_void_p),
                ("n_aln", C.c_int64), ("n_cigar", C.c_int64), ("read_aln_off", i64p)]


class StageDump(C.Structure):
    _fields_ = [("smem_cap", C.c_int64), ("smem", i64p), ("smem_off", i64p), ("seed_cap", C.c_int64),
                ("seed", i64p), ("seed_off", i64p), ("n_smem", C.c_int64), ("n_seed", C.c_int64)]


class Tune(C.Structure):
    _fields_ = [("stripe_rows", C.c_int32), ("n_tried", C.c_int32), ("small_area", C.c_int64),
                ("warp_area", C.c_int64), ("ms_dp", C.c_double), ("ms_dp_default", C.c_double),
                ("smem_variant", C.c_int32), ("dp_lanes", C.c_int32), ("ms_smem", C.c_double),
                ("ms_smem_default", C.c_double), ("dp_stripe_blocks", C.c_int32), ("pad2", C.c_int32)]


class MapStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("n_reads", "n_smem", "n_seed", "n_chain", "n_aln", "n_ext", "n_sa",
                                         "dp_cells", "host_sorted", "n_launch")] + \
               [(n, C.c_double) for n in ("ms_total", "ms_smem", "ms_locate", "ms_chain", "ms_dp")] + \
               [(n, C.c_int64) for n in ("dp_cells_done", "n_band_exact", "n_band_drop", "n_band_fallback",
                                         "n_filtered", "n_dp_warp")] + \
               [("n_dp_class", C.c_int64 * 5), ("dp_class_cells", C.c_int64 * 5), ("n_smem_rerun", C.c_int64),
                ("smem_retries", C.c_int64), ("n_ext_ff", C.c_int64), ("n_ff_steps", C.c_int64),
                ("ms_dp_part", C.c_double * 4)]


def build(force: bool = False) -> str:
    """Compile the CUDA library for sm_100a in-tree (nvcc cross-compiles
    without a GPU)."""
    args = ["make", "-s", "-j4", "-C", os.path.join(HERE, "csrc")]
    if force:
        subprocess.run(args + ["clean"], check=True)
    subprocess.run(args, check=True)
    return LIB_PATH


_lib = None


def load_library(path: str = LIB_PATH):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library {path} is missing; run msgseqtk_b200.lib.build()")
    L = C.CDLL(path)
    L.msg_strerror.restype = C.c_char_p
    L.msg_strerror.argtypes = [C.c_int]
    L.msg_last_error.restype = C.c_char_p
    L.msg_last_error.argtypes = [C.c_void_p]
    L.msg_ctx_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
    L.msg_ctx_destroy.argtypes = [C.c_void_p]
    L.msg_index_load.argtypes = [C.c_void_p, C.POINTER(FmdView), C.POINTER(MtgView)]
    L.msg_index_bytes.argtypes = [C.c_void_p, i64p]
    L.msg_ctx_share_index.argtypes = [C.c_void_p, C.c_void_p]
    L.msg_db_read.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]
    L.msg_db_views.argtypes = [C.c_void_p, C.POINTER(FmdView), C.POINTER(MtgView)]
    L.msg_db_free.argtypes = [C.c_void_p]
    L.msg_db_read_device.argtypes = [C.c_int, C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(C.c_void_p)]
    L.msg_db_read_cached.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.POINTER(C.c_void_p),
                                     C.POINTER(C.c_int)]
    L.msg_db_free.restype = None
    L.msg_map_params_default.argtypes = [C.POINTER(MapParams)]
    L.msg_map_params_default.restype = None
    L.msg_map_batch.argtypes = [C.c_void_p, C.POINTER(ReadBatch), C.POINTER(MapParams), C.POINTER(AlnOut),
                                C.POINTER(StageDump)]
    L.msg_map_batch_device.argtypes = L.msg_map_batch.argtypes
    i32p_ = C.POINTER(C.c_int32)
    L.msg_seed_batch.argtypes = [C.c_void_p, C.POINTER(ReadBatch), C.POINTER(MapParams), i64p, C.c_int64, i64p, i64p]
    L.msg_locate_batch.argtypes = [C.c_void_p, C.POINTER(ReadBatch), i64p, i64p, i64p, C.c_int64, i64p, i64p]
    L.msg_chain_batch.argtypes = [C.c_void_p, C.POINTER(ReadBatch), i64p, i64p, i32p_, C.c_int64, i64p, C.c_int64,
                                  i64p, i64p, i64p]
    L.msg_align_batch.argtypes = [C.c_void_p, C.POINTER(ReadBatch), i64p, i64p, i32p_, i64p, i64p,
                                  C.POINTER(MapParams), C.POINTER(AlnOut)]
    L.msg_map_batches.argtypes = [C.c_void_p, C.c_int64, C.POINTER(ReadBatch), C.POINTER(MapParams),
                                  C.POINTER(AlnOut)]
    L.msg_last_stats.argtypes = [C.c_void_p, C.POINTER(MapStats)]
    L.msg_result_device.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
    L.msg_ctx_stream.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    L.msg_ctx_set_scratch_limit.argtypes = [C.c_void_p, C.c_int64]
    L.msg_ctx_set_dp_shape.argtypes = [C.c_void_p, C.c_int32, C.c_int64, C.c_int64]
    L.msg_ctx_set_smem_shape.argtypes = [C.c_void_p, C.c_int32]
    L.msg_ctx_set_dp_lanes.argtypes = [C.c_void_p, C.c_int32]
    L.msg_ctx_set_dp_occupancy.argtypes = [C.c_void_p, C.c_int32]
    L.msg_autotune.argtypes = [C.c_void_p, C.POINTER(ReadBatch), C.POINTER(MapParams), C.POINTER(Tune)]
    L.msg_smem_batch_noalloc.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.POINTER(MapParams),
                                         C.c_void_p, C.c_int64, C.c_void_p]
    f32p = C.POINTER(C.c_float)
    i32p = C.POINTER(C.c_int32)
    L.msg_band_model_set.argtypes = [C.c_void_p, f32p, C.c_int64]
    L.msg_band_collect.argtypes = [C.c_void_p, C.POINTER(ReadBatch), C.POINTER(MapParams), f32p, i32p, C.c_int64, i64p]
    L.msg_band_train.argtypes = [C.c_void_p, f32p, i32p, C.c_int64, C.POINTER(BandTrainParams), f32p, f32p]
    L.msg_band_grad.argtypes = [C.c_void_p, f32p, f32p, i32p, C.c_int64, f32p, f32p]
    L.msg_tail_params_default.argtypes = [C.POINTER(TailParams)]
    L.msg_tail_params_default.restype = None
    L.msg_tail_batch.argtypes = [C.POINTER(MtgView), C.POINTER(ReadBatch), u8p, C.c_void_p, C.POINTER(C.c_uint32),
                                 i64p, C.POINTER(TailParams), C.c_void_p, C.c_int64, C.c_char_p, C.c_int64, i64p,
                                 i64p]
    L.msg_pair_params_default.argtypes = [C.POINTER(PairParams)]
    L.msg_pair_params_default.restype = None
    L.msg_tail_pe_batch.argtypes = L.msg_tail_batch.argtypes[:7] + [C.POINTER(PairParams)] + \
        L.msg_tail_batch.argtypes[7:]
    L.msg_fastq_parse.argtypes = [C.c_char_p, C.c_int64, C.c_int, C.POINTER(FastqBatch), i64p]
    L.msg_fastq_format.argtypes = [C.POINTER(ReadBatch), u8p, C.c_char_p, i64p, u8p, C.c_char_p, C.c_int64, i64p]
    L.msg_clean_format.argtypes = [C.c_char_p, i64p, C.c_int64] + [C.POINTER(C.c_double)] * 3 + \
        [C.c_char_p, C.c_int64, i64p]
    L.msg_sam_format.argtypes = [C.c_void_p, C.c_int64, C.c_char_p, C.POINTER(ReadBatch), u8p,
                                 C.POINTER(C.c_uint32), C.c_char_p, i64p, C.POINTER(C.c_char_p), C.c_int64, C.c_char_p,
                                 C.c_int64, i64p]
    L.msg_bam_header.argtypes = [C.c_char_p, C.c_int64, C.POINTER(C.c_char_p), i64p, C.c_int64, u8p, C.c_int64, i64p]
    L.msg_bam_format.argtypes = [C.c_void_p, C.c_int64, C.c_char_p, C.POINTER(ReadBatch), u8p,
                                 C.POINTER(C.c_uint32), C.c_char_p, i64p, C.c_int64, u8p, C.c_int64, i64p]
    L.msg_bgzf_compress.argtypes = [u8p, C.c_int64, C.c_int, C.c_int, C.c_int, u8p, C.c_int64, i64p]
    f64p = C.POINTER(C.c_double)
    L.msg_mem_params_default.argtypes = [C.POINTER(MemParams)]
    L.msg_mem_params_default.restype = None
    L.msg_mem_batch.argtypes = [C.c_void_p, C.POINTER(ReadBatch), C.POINTER(MemParams), f64p, i32p, i64p, C.c_int64,
                                i64p]
    L.msg_clean_batch.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(ReadBatch), C.POINTER(ReadBatch),
                                  C.POINTER(MemParams), C.c_double, f64p, f64p, f64p, u8p]
    L.msg_clean_batch_device.argtypes = L.msg_clean_batch.argtypes
    L.msg_occ_query.argtypes = [C.c_void_p, C.c_int64, u8p, i64p, i64p]
    L.msg_bi_ext_query.argtypes = [C.c_void_p, C.c_int64, C.c_int, u8p, i64p, i64p, i64p, i64p]
    L.msg_sa_query.argtypes = [C.c_void_p, C.c_int64, i64p, i64p]
    _lib = L
    return L


class MsgError(RuntimeError):
    def __init__(self, code, detail=""):
        self.code = code
        lib = load_library()
        super().__init__(f"{lib.msg_strerror(code).decode()} ({code}): {detail}")


def _p(a, t):
    return a.ctypes.data_as(t)


def default_params(**kw) -> MapParams:
    p = MapParams()
    load_library().msg_map_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def tail_params(**kw) -> TailParams:
    p = TailParams()
    load_library().msg_tail_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def mtg_view(view):
    """(MtgView, arrays to keep alive) from an index view."""
    k = [np.ascontiguousarray(x) for x in (view.bd_start, view.bd_end, view.chr_len, view.chr_seq, view.chr_off)]
    return MtgView(len(k[0]), _p(k[0], i64p), _p(k[1], i64p), _p(k[2], i64p), _p(k[3], u8p), _p(k[4], i64p)), k


def pair_params(**kw) -> PairParams:
    q = PairParams()
    load_library().msg_pair_params_default(C.byref(q))
    for k, v in kw.items():
        setattr(q, k, v)
    return q


def tail(view, seq, off, qual, aln, cigar, read_aln_off, params: TailParams | None = None,
         pairing: PairParams | None = None):
    """msgseqtk-align's tail on host threads: single-end (filter, evaluate,
    calcMapQ, sort, output), or paired-end when `pairing` is given (mates at
    reads 2i and 2i+1). Returns (records as SAM_DTYPE, MD text bytes)."""
    L = load_library()
    params = params or tail_params()
    m, keep = mtg_view(view)
    seq = np.ascontiguousarray(seq, dtype=np.uint8)
    off = np.ascontiguousarray(off, dtype=np.int64)
    qual = None if qual is None else np.ascontiguousarray(qual, dtype=np.uint8)
    aln = np.ascontiguousarray(aln, dtype=ALN_DTYPE)
    cigar = np.ascontiguousarray(cigar, dtype=np.uint32)
    roff = np.ascontiguousarray(read_aln_off, dtype=np.int64)
    rb = ReadBatch(len(off) - 1, _p(seq, u8p), _p(off, i64p))
    n_out, md_len = C.c_int64(0), C.c_int64(0)
    # a first guess that fits: one record per read or per alignment, an MD text
    # of at most two characters per query base plus the counts
    n = len(off) - 1
    cap = n + (len(aln) if params.max_report != 1 or pairing is not None else 0)
    mcap = 2 * int(off[-1] - off[0]) * max(1, min(int(params.max_report) or len(aln) + 1, len(aln) + 1)) + 16 * cap
    while True:
        out = np.empty(max(cap, 1), dtype=SAM_DTYPE)  # untouched pages cost nothing
        md = np.empty(max(mcap, 1), dtype=np.uint8)
        args = [C.byref(m), C.byref(rb), _p(qual, u8p) if qual is not None else None, aln.ctypes.data,
                cigar.ctypes.data_as(C.POINTER(C.c_uint32)), _p(roff, i64p), C.byref(params)]
        if pairing is not None:
            args.append(C.byref(pairing))
        args += [out.ctypes.data, cap, md.ctypes.data_as(C.c_char_p), mcap, C.byref(n_out), C.byref(md_len)]
        rc = (L.msg_tail_pe_batch if pairing is not None else L.msg_tail_batch)(*args)
        if rc == MSG_EINVAL and (n_out.value > cap or md_len.value > mcap):
            cap, mcap = n_out.value, md_len.value
            continue
        if rc != MSG_OK:
            raise MsgError(rc, "msg_tail_batch")
        return out[:n_out.value], md[:md_len.value].tobytes()


def fastq_parse(text: bytes, at_eof: bool = True, max_reads: int | None = None):
    """msg_fastq_parse on a bytes object: dict(seq, qual, off, text, name_off,
    consumed), text holding "name\tdescription\n" per read."""
    L = load_library()
    cap_r = max_reads if max_reads is not None else text.count(b"\n") // 4 + 2
    cap_b = len(text) + 1
    seq = np.empty(cap_b, np.uint8)
    qual = np.empty(cap_b, np.uint8)
    off = np.empty(cap_r + 1, np.int64)
    nm = np.empty(len(text) + 2 * cap_r + 1, np.uint8)
    noff = np.empty(cap_r + 1, np.int64)
    b = FastqBatch(cap_r, cap_b, len(nm), _p(seq, u8p), _p(qual, u8p), _p(off, i64p),
                   nm.ctypes.data_as(C.c_char_p), _p(noff, i64p), 0, 0, 0)
    used = C.c_int64(0)
    rc = L.msg_fastq_parse(text, len(text), int(at_eof), C.byref(b), C.byref(used))
    if rc != MSG_OK:
        raise MsgError(rc, "msg_fastq_parse")
    n = b.n_reads
    return dict(seq=seq[:b.n_bases].copy(), qual=qual[:b.n_bases].copy(), off=off[:n + 1].copy(),
                text=nm[:b.n_text].tobytes(), name_off=noff[:n + 1].copy(), consumed=used.value)


def fastq_format(seq, off, qual, text: bytes, name_off, keep=None) -> bytes:
    """msg_fastq_format: FASTQ text of the kept reads (all when keep is None)."""
    L = load_library()
    seq = np.ascontiguousarray(seq, dtype=np.uint8)
    off = np.ascontiguousarray(off, dtype=np.int64)
    qual = np.ascontiguousarray(qual, dtype=np.uint8)
    name_off = np.ascontiguousarray(name_off, dtype=np.int64)
    kp = None if keep is None else np.ascontiguousarray(keep, dtype=np.uint8)
    rb = ReadBatch(len(off) - 1, _p(seq, u8p), _p(off, i64p))
    n = C.c_int64(0)
    cap = 2 * len(seq) + len(text) + 8 * (len(off) - 1) + 16
    buf = C.create_string_buffer(cap)
    rc = L.msg_fastq_format(C.byref(rb), _p(qual, u8p), text, _p(name_off, i64p),
                            _p(kp, u8p) if kp is not None else None, buf, cap, C.byref(n))
    if rc != MSG_OK:
        raise MsgError(rc, "msg_fastq_format")
    return buf.raw[:n.value]


def clean_format(text: bytes, name_off, ref_ll, bg_ll, lod) -> bytes:
    """msg_clean_format: msgseqtk-clean's assignment lines."""
    L = load_library()
    name_off = np.ascontiguousarray(name_off, dtype=np.int64)
    arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (ref_ll, bg_ll, lod)]
    dp = C.POINTER(C.c_double)
    n = C.c_int64(0)
    cap = len(text) + 96 * (len(name_off) - 1) + 16
    buf = C.create_string_buffer(cap)
    rc = L.msg_clean_format(text, _p(name_off, i64p), len(name_off) - 1, *[a.ctypes.data_as(dp) for a in arrs], buf,
                            cap, C.byref(n))
    if rc != MSG_OK:
        raise MsgError(rc, "msg_clean_format")
    return buf.raw[:n.value]


def sam_format(recs, md: bytes, seq, off, qual, cigar, names: bytes, name_off, chrom_names) -> bytes:
    """msg_sam_format: SAM text lines of tail records."""
    L = load_library()
    recs = np.ascontiguousarray(recs, dtype=SAM_DTYPE)
    seq = np.ascontiguousarray(seq, dtype=np.uint8)
    off = np.ascontiguousarray(off, dtype=np.int64)
    qual = np.ascontiguousarray(qual, dtype=np.uint8)
    cigar = np.ascontiguousarray(cigar, dtype=np.uint32)
    name_off = np.ascontiguousarray(name_off, dtype=np.int64)
    cn = (C.c_char_p * max(1, len(chrom_names)))(*[c.encode() for c in chrom_names])
    rb = ReadBatch(len(off) - 1, _p(seq, u8p), _p(off, i64p))
    n = C.c_int64(0)
    cap = 1 << 16
    while True:
        buf = C.create_string_buffer(cap)
        rc = L.msg_sam_format(recs.ctypes.data, len(recs), md, C.byref(rb), _p(qual, u8p),
                              cigar.ctypes.data_as(C.POINTER(C.c_uint32)), names, _p(name_off, i64p), cn,
                              len(chrom_names), buf, cap, C.byref(n))
        if rc == MSG_EINVAL and n.value > cap:
            cap = n.value
            continue
        if rc != MSG_OK:
            raise MsgError(rc, "msg_sam_format")
        return buf.raw[:n.value]


def _grow(call, cap, what):
    """Runs call(buf, cap, n) with a buffer that grows to the size it asks for."""
    n = C.c_int64(0)
    while True:
        buf = np.empty(max(cap, 1), dtype=np.uint8)
        rc = call(_p(buf, u8p), cap, C.byref(n))
        if rc == MSG_EINVAL and n.value > cap:
            cap = n.value
            continue
        if rc != MSG_OK:
            raise MsgError(rc, what)
        return buf[:n.value].tobytes()


def bam_header(text: bytes, chrom_names, chrom_len) -> bytes:
    """msg_bam_header: the uncompressed binary BAM header."""
    L = load_library()
    cn = (C.c_char_p * max(1, len(chrom_names)))(*[c.encode() for c in chrom_names])
    cl = np.ascontiguousarray(chrom_len, dtype=np.int64)
    return _grow(lambda b, cap, n: L.msg_bam_header(text, len(text), cn, _p(cl, i64p), len(chrom_names), b, cap, n),
                 len(text) + 64 * len(chrom_names) + 64, "msg_bam_header")


def bam_format(recs, md: bytes, seq, off, qual, cigar, names: bytes, name_off, n_chrom: int) -> bytes:
    """msg_bam_format: uncompressed binary BAM records of tail records."""
    L = load_library()
    recs = np.ascontiguousarray(recs, dtype=SAM_DTYPE)
    seq = np.ascontiguousarray(seq, dtype=np.uint8)
    off = np.ascontiguousarray(off, dtype=np.int64)
    qual = None if qual is None else np.ascontiguousarray(qual, dtype=np.uint8)
    cigar = np.ascontiguousarray(cigar, dtype=np.uint32)
    name_off = np.ascontiguousarray(name_off, dtype=np.int64)
    rb = ReadBatch(len(off) - 1, _p(seq, u8p), _p(off, i64p))
    return _grow(lambda b, cap, n: L.msg_bam_format(recs.ctypes.data, len(recs), md, C.byref(rb),
                                                    _p(qual, u8p) if qual is not None else None,
                                                    cigar.ctypes.data_as(C.POINTER(C.c_uint32)), names,
                                                    _p(name_off, i64p), int(n_chrom), b, cap, n),
                 1 << 16, "msg_bam_format")


def bgzf_compress(data: bytes, level: int = 6, n_threads: int = 1, eof: bool = True) -> bytes:
    """msg_bgzf_compress: BGZF members of data (and the EOF member)."""
    L = load_library()
    a = np.frombuffer(data, dtype=np.uint8) if len(data) else np.zeros(1, np.uint8)
    a = np.ascontiguousarray(a)
    return _grow(lambda b, cap, n: L.msg_bgzf_compress(_p(a, u8p), len(data), level, n_threads, int(eof), b, cap, n),
                 len(data) + len(data) // 8 + 1024, "msg_bgzf_compress")


def mem_params(**kw) -> MemParams:
    p = MemParams()
    load_library().msg_mem_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Context:
    """One device context: a CUDA stream, a loaded index and batch buffers."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.msg_ctx_create(device, C.byref(h))
        if rc != MSG_OK:
            raise MsgError(rc, "msg_ctx_create")
        self.h = h
        self._keep = []

    def close(self):
        if getattr(self, "h", None):
            self.lib.msg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != MSG_OK:
            raise MsgError(rc, f"{what}: {self.lib.msg_last_error(self.h).decode()}")

    def load_index(self, view):
        k = [np.ascontiguousarray(x) for x in (view.bwt, view.B.astype(np.int64), view.sample_rows, view.sample_vals,
                                               view.bd_start, view.bd_end, view.chr_len, view.chr_seq, view.chr_off)]
        f = FmdView(view.n, _p(k[0], u8p), _p(k[1], i64p), len(k[2]), _p(k[2], i64p), _p(k[3], i64p))
        m = MtgView(len(k[4]), _p(k[4], i64p), _p(k[5], i64p), _p(k[6], i64p), _p(k[7], u8p), _p(k[8], i64p))
        self._check(self.lib.msg_index_load(self.h, C.byref(f), C.byref(m)), "msg_index_load")

    def load_database(self, db: "Database"):
        """msg_index_load from a database read with msg_db_read."""
        self._check(self.lib.msg_index_load(self.h, C.byref(db.fmd), C.byref(db.mtg)), "msg_index_load")

    def share_index(self, owner: "Context"):
        """Map against the index `owner` loaded, without a second device
        copy (msg_ctx_share_index); the memory lives while any holder does."""
        self._check(self.lib.msg_ctx_share_index(self.h, owner.h), "msg_ctx_share_index")

    def apply_shapes(self, shapes: dict):
        """Set the kernel shapes an autotune() result names on this context."""
        self.set_smem_shape(shapes["smem_variant"])
        self.set_dp_shape(shapes["stripe_rows"], shapes["small_area"], shapes["warp_area"])
        self.set_dp_lanes(shapes["dp_lanes"])
        self.set_dp_occupancy(shapes["dp_stripe_blocks"])

    def index_bytes(self) -> int:
        b = C.c_int64(0)
        self._check(self.lib.msg_index_bytes(self.h, C.byref(b)), "msg_index_bytes")
        return b.value

    def occ(self, b, i):
        b = np.ascontiguousarray(b, dtype=np.uint8)
        i = np.ascontiguousarray(i, dtype=np.int64)
        out = np.zeros(len(i), dtype=np.int64)
        self._check(self.lib.msg_occ_query(self.h, len(i), _p(b, u8p), _p(i, i64p), _p(out, i64p)), "msg_occ_query")
        return out

    def bi_ext(self, direction, b, p, q, s):
        b = np.ascontiguousarray(b, dtype=np.uint8)
        p, q, s = (np.array(x, dtype=np.int64) for x in (p, q, s))
        ret = np.zeros(len(b), dtype=np.int64)
        self._check(self.lib.msg_bi_ext_query(self.h, len(b), direction, _p(b, u8p), _p(p, i64p), _p(q, i64p),
                                              _p(s, i64p), _p(ret, i64p)), "msg_bi_ext_query")
        return ret, p, q, s

    def sa(self, rows):
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        out = np.zeros(len(rows), dtype=np.int64)
        self._check(self.lib.msg_sa_query(self.h, len(rows), _p(rows, i64p), _p(out, i64p)), "msg_sa_query")
        return out

    def map(self, seq, off, params: MapParams | None = None, dump: bool = False, device_ptrs=None,
            aln_cap: int | None = None, cigar_cap: int | None = None):
        """Map reads (nt16 codes `seq`, offsets `off`). Returns a dict with the
        alignment records, CIGAR words and per-read alignment offsets; with
        dump=True also the SMEM and seed lists."""
        params = params or default_params()
        n = len(off) - 1
        if device_ptrs is None:
            seq = np.ascontiguousarray(seq, dtype=np.uint8)
            off = np.ascontiguousarray(off, dtype=np.int64)
            batch = ReadBatch(n, _p(seq, u8p), _p(off, i64p))
            fn = self.lib.msg_map_batch
        else:
            batch = ReadBatch(n, C.cast(C.c_void_p(device_ptrs[0]), u8p), C.cast(C.c_void_p(device_ptrs[1]), i64p))
            fn = self.lib.msg_map_batch_device
        aln_cap = aln_cap or max(16, 4 * n)
        cigar_cap = cigar_cap or max(64, 16 * aln_cap)
        while True:
            aln = np.zeros(aln_cap, dtype=ALN_DTYPE)
            cig = np.zeros(cigar_cap, dtype=np.uint32)
            roff = np.zeros(n + 1, dtype=np.int64)
            out = AlnOut(aln_cap, aln.ctypes.data, cigar_cap, cig.ctypes.data, 0, 0, _p(roff, i64p))
            d = None
            if dump:
                smem_cap = 64 * n + 64
                seed_cap = 64 * n + 64
                sm = np.zeros((smem_cap, 6), dtype=np.int64)
                so = np.zeros(n + 1, dtype=np.int64)
                sd = np.zeros((seed_cap, 6), dtype=np.int64)
                sdo = np.zeros(n + 1, dtype=np.int64)
                d = StageDump(smem_cap, _p(sm, i64p), _p(so, i64p), seed_cap, _p(sd, i64p), _p(sdo, i64p), 0, 0)
            rc = fn(self.h, C.byref(batch), C.byref(params), C.byref(out), C.byref(d) if d is not None else None)
            if rc == MSG_EINVAL and (out.n_aln > aln_cap or out.n_cigar > cigar_cap):
                aln_cap = max(aln_cap, out.n_aln) * 2
                cigar_cap = max(cigar_cap, out.n_cigar) * 2
                continue
            self._check(rc, "msg_map_batch")
            res = dict(aln=aln[:out.n_aln].copy(), cigar=cig[:out.n_cigar].copy(), read_aln_off=roff)
            if dump:
                if d.n_smem > smem_cap or d.n_seed > seed_cap:
                    raise MsgError(MSG_EINVAL, "dump capacity")
                res.update(smem=sm[:d.n_smem].copy(), smem_off=so, seed=sd[:d.n_seed].copy(), seed_off=sdo)
            return res

    # ---- the stages of map() one call each (msg_seed/locate/chain/align_batch) ----
    @staticmethod
    def _batch(seq, off):
        seq = np.ascontiguousarray(seq, dtype=np.uint8)
        off = np.ascontiguousarray(off, dtype=np.int64)
        return seq, off, ReadBatch(len(off) - 1, _p(seq, u8p), _p(off, i64p))

    def seed_batch(self, seq, off, params: MapParams | None = None):
        """SMEM rows (n, 6) in emission order and per-read offsets."""
        params = params or default_params()
        seq, off, b = self._batch(seq, off)
        n = len(off) - 1
        cap = 8 * n + 16
        while True:
            rows = np.zeros((cap, 6), dtype=np.int64)
            roff = np.zeros(n + 1, dtype=np.int64)
            cnt = C.c_int64(0)
            rc = self.lib.msg_seed_batch(self.h, C.byref(b), C.byref(params), _p(rows, i64p), cap, _p(roff, i64p),
                                         C.byref(cnt))
            if rc == MSG_EINVAL and cnt.value > cap:
                cap = cnt.value
                continue
            self._check(rc, "msg_seed_batch")
            return rows[:cnt.value].copy(), roff

    def locate_batch(self, seq, off, smem, smem_off):
        """Seeds (n, 6) of the given SMEM rows after removeRedundant, per-read offsets."""
        seq, off, b = self._batch(seq, off)
        smem = np.ascontiguousarray(smem, dtype=np.int64).reshape(-1, 6)
        smem_off = np.ascontiguousarray(smem_off, dtype=np.int64)
        n = len(off) - 1
        cap = int(smem[:, 4].sum()) + 16 if len(smem) else 16
        rows = np.zeros((cap, 6), dtype=np.int64)
        roff = np.zeros(n + 1, dtype=np.int64)
        cnt = C.c_int64(0)
        self._check(self.lib.msg_locate_batch(self.h, C.byref(b), _p(smem, i64p), _p(smem_off, i64p), _p(rows, i64p),
                                              cap, _p(roff, i64p), C.byref(cnt)), "msg_locate_batch")
        return rows[:cnt.value].copy(), roff

    def chain_batch(self, seq, off, seed, seed_off):
        """Chains: seed indices within each read's seed rows, per-chain and per-read offsets."""
        seq, off, b = self._batch(seq, off)
        seed = np.ascontiguousarray(seed, dtype=np.int64).reshape(-1, 6)
        seed_off = np.ascontiguousarray(seed_off, dtype=np.int64)
        n = len(off) - 1
        ccap, scap = len(seed) + 16, 4 * len(seed) + 16
        while True:
            cs = np.zeros(scap, dtype=np.int32)
            cso = np.zeros(ccap + 1, dtype=np.int64)
            rco = np.zeros(n + 1, dtype=np.int64)
            nc, ns = C.c_int64(0), C.c_int64(0)
            rc = self.lib.msg_chain_batch(self.h, C.byref(b), _p(seed, i64p), _p(seed_off, i64p),
                                          cs.ctypes.data_as(C.POINTER(C.c_int32)), scap, _p(cso, i64p), ccap,
                                          _p(rco, i64p), C.byref(nc), C.byref(ns))
            if rc == MSG_EINVAL and (nc.value > ccap or ns.value > scap):
                ccap, scap = max(ccap, nc.value), max(scap, ns.value)
                continue
            self._check(rc, "msg_chain_batch")
            return cs[:ns.value].copy(), cso[:nc.value + 1].copy(), rco

    def align_batch(self, seq, off, seed, seed_off, chain_seed, chain_seed_off, read_chain_off,
                    params: MapParams | None = None):
        """Records of the given chains, as map() returns them."""
        params = params or default_params()
        seq, off, b = self._batch(seq, off)
        seed = np.ascontiguousarray(seed, dtype=np.int64).reshape(-1, 6)
        seed_off = np.ascontiguousarray(seed_off, dtype=np.int64)
        chain_seed = np.ascontiguousarray(chain_seed, dtype=np.int32)
        chain_seed_off = np.ascontiguousarray(chain_seed_off, dtype=np.int64)
        read_chain_off = np.ascontiguousarray(read_chain_off, dtype=np.int64)
        n = len(off) - 1
        aln_cap = max(16, len(chain_seed_off))
        cigar_cap = 16 * aln_cap + 64
        while True:
            aln = np.zeros(aln_cap, dtype=ALN_DTYPE)
            cig = np.zeros(cigar_cap, dtype=np.uint32)
            roff = np.zeros(n + 1, dtype=np.int64)
            out = AlnOut(aln_cap, aln.ctypes.data, cigar_cap, cig.ctypes.data, 0, 0, _p(roff, i64p))
            rc = self.lib.msg_align_batch(self.h, C.byref(b), _p(seed, i64p), _p(seed_off, i64p),
                                          chain_seed.ctypes.data_as(C.POINTER(C.c_int32)), _p(chain_seed_off, i64p),
                                          _p(read_chain_off, i64p), C.byref(params), C.byref(out))
            if rc == MSG_EINVAL and (out.n_aln > aln_cap or out.n_cigar > cigar_cap):
                aln_cap, cigar_cap = max(aln_cap, out.n_aln) * 2, max(cigar_cap, out.n_cigar) * 2
                continue
            self._check(rc, "msg_align_batch")
            return dict(aln=aln[:out.n_aln].copy(), cigar=cig[:out.n_cigar].copy(), read_aln_off=roff)

    def stream_handle(self) -> int:
        h = C.c_void_p()
        self._check(self.lib.msg_ctx_stream(self.h, C.byref(h)), "msg_ctx_stream")
        return h.value or 0

    def map_device(self, seq_ptr: int, off_ptr: int, n_reads: int, params: MapParams | None = None):
        """Map reads already in device memory; results stay on the device.
        Returns (n_aln, n_cigar)."""
        params = params or default_params()
        batch = ReadBatch(n_reads, C.cast(C.c_void_p(seq_ptr), u8p), C.cast(C.c_void_p(off_ptr), i64p))
        out = AlnOut(0, None, 0, None, 0, 0, None)
        self._check(self.lib.msg_map_batch_device(self.h, C.byref(batch), C.byref(params), C.byref(out), None),
                    "msg_map_batch_device")
        return out.n_aln, out.n_cigar

    def map_into(self, seq: np.ndarray, off: np.ndarray, aln: np.ndarray, cig: np.ndarray, roff: np.ndarray,
                 params: MapParams | None = None):
        """Map host reads into caller-owned (e.g. pinned) host buffers.
        Returns (n_aln, n_cigar)."""
        params = params or default_params()
        batch = ReadBatch(len(off) - 1, _p(seq, u8p), _p(off, i64p))
        out = AlnOut(len(aln), aln.ctypes.data, len(cig), cig.ctypes.data, 0, 0, _p(roff, i64p))
        self._check(self.lib.msg_map_batch(self.h, C.byref(batch), C.byref(params), C.byref(out), None),
                    "msg_map_batch")
        return out.n_aln, out.n_cigar

    def map_batches(self, batches, outs, params: MapParams | None = None):
        """msg_map_batches: batches = [(seq, off)], outs = [(aln, cigar,
        read_aln_off)] host arrays (pinned for overlapped copies). Returns
        [(n_aln, n_cigar)] per batch."""
        params = params or default_params()
        n = len(batches)
        rb = (ReadBatch * n)(*[ReadBatch(len(o) - 1, _p(q, u8p), _p(o, i64p)) for q, o in batches])
        ao = (AlnOut * n)(*[AlnOut(len(a), a.ctypes.data, len(c), c.ctypes.data, 0, 0, _p(r, i64p))
                            for a, c, r in outs])
        self._check(self.lib.msg_map_batches(self.h, n, rb, C.byref(params), ao), "msg_map_batches")
        return [(ao[k].n_aln, ao[k].n_cigar) for k in range(n)]

    def smem_noalloc(self, seq_ptr: int, off_ptr: int, n_reads: int, out_ptr: int, cap_per_read: int,
                     count_ptr: int, params: MapParams | None = None) -> int:
        """msg_smem_batch_noalloc on caller-owned device buffers; returns the
        status code (MSG_EINVAL when a count exceeded cap_per_read)."""
        params = params or default_params()
        return self.lib.msg_smem_batch_noalloc(self.h, n_reads, seq_ptr, off_ptr, C.byref(params), out_ptr,
                                               cap_per_read, count_ptr)

    # ---- MEM search and read cleaning ----
    def mems(self, seq, off, params: MemParams | None = None, rows: bool = True):
        """SMEM_LIST::findMEMS per read: (loglik[n], n_mem[n], rows[m, 6] or
        None) with rows in read order."""
        params = params or mem_params()
        seq = np.ascontiguousarray(seq, dtype=np.uint8)
        off = np.ascontiguousarray(off, dtype=np.int64)
        n = len(off) - 1
        batch = ReadBatch(n, _p(seq, u8p), _p(off, i64p))
        ll = np.zeros(n, dtype=np.float64)
        cnt = np.zeros(n, dtype=np.int32)
        nr = C.c_int64(0)
        f64p, i32p = C.POINTER(C.c_double), C.POINTER(C.c_int32)
        if not rows:
            self._check(self.lib.msg_mem_batch(self.h, C.byref(batch), C.byref(params), _p(ll, f64p), _p(cnt, i32p),
                                               None, 0, C.byref(nr)), "msg_mem_batch")
            return ll, cnt, None
        cap = max(16, n)
        while True:
            out = np.zeros((cap, 6), dtype=np.int64)
            rc = self.lib.msg_mem_batch(self.h, C.byref(batch), C.byref(params), _p(ll, f64p), _p(cnt, i32p),
                                        _p(out, i64p), cap, C.byref(nr))
            if rc == MSG_EINVAL and nr.value > cap:
                cap = nr.value
                continue
            self._check(rc, "msg_mem_batch")
            return ll, cnt, out[:nr.value].copy()

    def clean(self, bg: "Context", seq, off, rev_seq=None, rev_off=None, params: MemParams | None = None,
              min_lod: float = 0.0):
        """msgseqtk-clean's decision with this context's index as the
        reference genomes and bg's as the background, reads in host memory:
        (ref_loglik, bg_loglik, lod, keep)."""
        seq = np.ascontiguousarray(seq, dtype=np.uint8)
        off = np.ascontiguousarray(off, dtype=np.int64)
        n = len(off) - 1
        fb = ReadBatch(n, _p(seq, u8p), _p(off, i64p))
        rb = None
        if rev_seq is not None:
            rev_seq = np.ascontiguousarray(rev_seq, dtype=np.uint8)
            rev_off = np.ascontiguousarray(rev_off, dtype=np.int64)
            rb = ReadBatch(len(rev_off) - 1, _p(rev_seq, u8p), _p(rev_off, i64p))  # the library checks the counts
        return self._clean(self.lib.msg_clean_batch, bg, n, fb, rb, params, min_lod)

    def clean_device(self, bg: "Context", seq_ptr: int, off_ptr: int, n: int, rev_seq_ptr: int | None = None,
                     rev_off_ptr: int | None = None, params: MemParams | None = None, min_lod: float = 0.0):
        """clean() with the reads already in device memory (pointers)."""
        fb = ReadBatch(n, C.cast(C.c_void_p(seq_ptr), u8p), C.cast(C.c_void_p(off_ptr), i64p))
        rb = None
        if rev_seq_ptr is not None:
            rb = ReadBatch(n, C.cast(C.c_void_p(rev_seq_ptr), u8p), C.cast(C.c_void_p(rev_off_ptr), i64p))
        return self._clean(self.lib.msg_clean_batch_device, bg, n, fb, rb, params, min_lod)

    def _clean(self, fn, bg, n, fb, rb, params, min_lod):
        params = params or mem_params()
        f64p = C.POINTER(C.c_double)
        out = [np.zeros(n, dtype=np.float64) for _ in range(3)]
        keep = np.zeros(n, dtype=np.uint8)
        self._check(fn(self.h, bg.h, C.byref(fb), C.byref(rb) if rb is not None else None, C.byref(params), min_lod,
                       _p(out[0], f64p), _p(out[1], f64p), _p(out[2], f64p), _p(keep, u8p)), "msg_clean_batch")
        return out[0], out[1], out[2], keep.astype(bool)

    # ---- band model ----
    def band_model_set(self, params: np.ndarray):
        params = np.ascontiguousarray(params, dtype=np.float32)
        self._check(self.lib.msg_band_model_set(self.h, _p(params, C.POINTER(C.c_float)), params.size),
                    "msg_band_model_set")

    def band_collect(self, seq: np.ndarray, off: np.ndarray, params: MapParams | None = None):
        """Per-chain features (n x 16 float32) and cheapest certified band
        class (int32; -1 for chains that never get a band) of a host read
        batch."""
        params = params or default_params()
        seq = np.ascontiguousarray(seq, dtype=np.uint8)
        off = np.ascontiguousarray(off, dtype=np.int64)
        rb = ReadBatch(len(off) - 1, _p(seq, u8p), _p(off, i64p))
        cap = max(16, 4 * (len(off) - 1))
        while True:
            feat = np.zeros((cap, BAND_FEATURES), dtype=np.float32)
            lab = np.zeros(cap, dtype=np.int32)
            n = C.c_int64(0)
            rc = self.lib.msg_band_collect(self.h, C.byref(rb), C.byref(params), _p(feat, C.POINTER(C.c_float)),
                                           _p(lab, C.POINTER(C.c_int32)), cap, C.byref(n))
            if rc == 1 and n.value > cap:  # MSG_EINVAL: capacity
                cap = n.value
                continue
            self._check(rc, "msg_band_collect")
            return feat[:n.value], lab[:n.value]

    def band_train(self, feat: np.ndarray, label: np.ndarray, epochs=20, batch=4096, lr=2e-3, seed=1):
        """Train the band model on the GPU; returns (params, per-epoch loss)."""
        feat = np.ascontiguousarray(feat, dtype=np.float32)
        label = np.ascontiguousarray(label, dtype=np.int32)
        tp = BandTrainParams(epochs, batch, lr, seed)
        params = np.zeros(BAND_NPARAMS, dtype=np.float32)
        loss = np.zeros(epochs, dtype=np.float32)
        self._check(self.lib.msg_band_train(self.h, _p(feat, C.POINTER(C.c_float)), _p(label, C.POINTER(C.c_int32)),
                                            len(label), C.byref(tp), _p(params, C.POINTER(C.c_float)),
                                            _p(loss, C.POINTER(C.c_float))), "msg_band_train")
        return params, loss

    def band_grad(self, params: np.ndarray, feat: np.ndarray, label: np.ndarray):
        params = np.ascontiguousarray(params, dtype=np.float32)
        feat = np.ascontiguousarray(feat, dtype=np.float32)
        label = np.ascontiguousarray(label, dtype=np.int32)
        grad = np.zeros(BAND_NPARAMS - 2 * BAND_FEATURES, dtype=np.float32)
        loss = C.c_float(0)
        self._check(self.lib.msg_band_grad(self.h, _p(params, C.POINTER(C.c_float)), _p(feat, C.POINTER(C.c_float)),
                                           _p(label, C.POINTER(C.c_int32)), len(label),
                                           _p(grad, C.POINTER(C.c_float)), C.byref(loss)), "msg_band_grad")
        return grad, loss.value

    def set_scratch_limit(self, nbytes: int):
        self._check(self.lib.msg_ctx_set_scratch_limit(self.h, int(nbytes)), "msg_ctx_set_scratch_limit")

    def autotune(self, seq, off, params: MapParams | None = None) -> dict:
        """msg_autotune on a sample batch: sets the fastest SMEM and DP shapes."""
        params = params or default_params()
        seq, off, b = self._batch(seq, off)
        r = Tune()
        self._check(self.lib.msg_autotune(self.h, C.byref(b), C.byref(params), C.byref(r)), "msg_autotune")
        return dict(smem_variant=r.smem_variant, stripe_rows=r.stripe_rows, small_area=r.small_area,
                    warp_area=r.warp_area, ms_smem=r.ms_smem, ms_smem_default=r.ms_smem_default, ms_dp=r.ms_dp,
                    ms_dp_default=r.ms_dp_default, n_tried=r.n_tried, dp_lanes=r.dp_lanes,
                    dp_stripe_blocks=r.dp_stripe_blocks)

    def set_dp_occupancy(self, blocks: int = 3):
        """Register budget of the stripe DP kernel (msg_ctx_set_dp_occupancy); records do not depend on it."""
        self._check(self.lib.msg_ctx_set_dp_occupancy(self.h, int(blocks)), "msg_ctx_set_dp_occupancy")

    def set_dp_lanes(self, bits: int = 16):
        """Lane width of the stripe DP fill (msg_ctx_set_dp_lanes); records do not depend on it."""
        self._check(self.lib.msg_ctx_set_dp_lanes(self.h, int(bits)), "msg_ctx_set_dp_lanes")

    def set_smem_shape(self, variant: int = 0):
        """SMEM thread-path variant (msg_ctx_set_smem_shape); records do not depend on it."""
        self._check(self.lib.msg_ctx_set_smem_shape(self.h, int(variant)), "msg_ctx_set_smem_shape")

    def set_dp_shape(self, stripe_rows: int = 16, small_area: int = 256, warp_area: int = 65536):
        """DP work split (msg_ctx_set_dp_shape); records do not depend on it."""
        self._check(self.lib.msg_ctx_set_dp_shape(self.h, int(stripe_rows), int(small_area), int(warp_area)),
                    "msg_ctx_set_dp_shape")

    def stats(self) -> dict:
        s = MapStats()
        self._check(self.lib.msg_last_stats(self.h, C.byref(s)), "msg_last_stats")
        d = {k: getattr(s, k) for k, _ in MapStats._fields_}
        d["n_dp_class"] = list(s.n_dp_class)
        d["dp_class_cells"] = list(s.dp_class_cells)
        d["ms_dp_part"] = list(s.ms_dp_part)
        return d


_ASCII = np.frombuffer(b"$ACMGRSVTWYHKDBN", dtype=np.uint8)
_COMP = np.array([0, 8, 4, 12, 2, 10, 6, 14, 1, 9, 5, 13, 3, 11, 7, 15], dtype=np.uint8)


def md_tag(cigar_words, query: np.ndarray, target_at, aln_from: int, aln_start: int) -> str:
    """Alignment::getAlnMDTag (Alignment.cpp:305-353) from CIGAR runs: '='/'X'
    by (query & target) != 0, insertions written as '^' + query bases."""
    md = []
    prev = -1
    ln = 0
    i, j = aln_from, aln_start
    for w in cigar_words:
        op, n = int(w) & 15, int(w) >> 4
        if op == 4:
            continue
        for _ in range(n):
            if op == 0:
                qb, tb = int(query[i]), int(target_at(j))
                o = 7 if (qb & tb) else 8
            else:
                o = op
            if o == 7:
                i += 1; j += 1; ln += 1
            elif o == 8:
                md.append(str(ln)); ln = 0
                md.append(chr(_ASCII[int(target_at(j))]))
                i += 1; j += 1
            elif o == 1:
                if prev != 1:
                    md.append(str(ln))
                ln = 0
                if o != prev:
                    md.append("^")
                md.append(chr(_ASCII[int(query[i])]))
                i += 1
            elif o == 2:
                j += 1
            prev = o
    md.append(str(ln))
    return "".join(md)


class Database:
    """A database read from msgseqtk-build files (msg_db_read): host arrays of
    the FMD-index and the MetaGenome, as numpy views."""

    def __init__(self, mtg_path, mgs_path, fmd_path, n_threads: int = 8, image=None, device=None):
        """With `image` (a path), msg_db_read_cached: read the decoded image
        there when it matches the files, else decode and write it;
        `from_image` tells which (1 read, 0 written, -1 not writable). With
        `device`, msg_db_read_device: the BWT decoded on that GPU."""
        self.lib = load_library()
        self.h = C.c_void_p()
        self.from_image = None
        paths = [str(x).encode() for x in (mtg_path, mgs_path, fmd_path)]
        if device is not None:
            rc = self.lib.msg_db_read_device(int(device), *paths, C.byref(self.h))
            if rc != MSG_OK:
                raise MsgError(rc, "msg_db_read_device")
        elif image is None:
            rc = self.lib.msg_db_read(*paths, n_threads, C.byref(self.h))
        else:
            hit = C.c_int(0)
            rc = self.lib.msg_db_read_cached(*paths, str(image).encode(), n_threads, C.byref(self.h), C.byref(hit))
            self.from_image = hit.value
        if rc != MSG_OK:
            raise MsgError(rc, "msg_db_read" if image is None else "msg_db_read_cached")
        self.fmd = FmdView()
        self.mtg = MtgView()
        self.lib.msg_db_views(self.h, C.byref(self.fmd), C.byref(self.mtg))

    def arrays(self):
        f, m = self.fmd, self.mtg
        arr = lambda p, n: np.ctypeslib.as_array(p, shape=(n,)).copy() if n > 0 else np.zeros(0)
        return dict(bwt=arr(f.bwt, f.n), B=arr(f.base_count, 16), sample_rows=arr(f.sample_rows, f.n_samples),
                    sample_vals=arr(f.sample_vals, f.n_samples), bd_start=arr(m.bd_start, m.n_chrom),
                    bd_end=arr(m.bd_end, m.n_chrom), chr_len=arr(m.chr_len, m.n_chrom),
                    chr_off=arr(m.chr_off, m.n_chrom + 1), chr_seq=arr(m.chr_seq, int(m.chr_off[m.n_chrom])))

    def view(self):
        """The database as an index view (msgseqtk_b200.index_build.FmdView),
        e.g. for Context.load_index or the oracle."""
        from .index_build import FmdView as View
        a = self.arrays()
        return View(int(self.fmd.n), a["bwt"].astype(np.uint8), a["B"].astype(np.int64),
                    a["sample_rows"].astype(np.int64), a["sample_vals"].astype(np.int64),
                    a["bd_start"].astype(np.int64), a["bd_end"].astype(np.int64), a["chr_len"].astype(np.int64),
                    a["chr_seq"].astype(np.uint8), a["chr_off"].astype(np.int64))

    def close(self):
        if self.h:
            self.lib.msg_db_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
