"""The C-ABI library loads and exports every function include/msg_b200.h
declares; calls that need no GPU behave."""
import ctypes as C
import os
import re

from msgseqtk_b200 import lib

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "msg_b200.h")


def declared_functions():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(msg_[a-z_0-9]+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    L = lib.load_library()
    names = declared_functions()
    assert len(names) >= 13
    for n in names:
        assert hasattr(L, n), n
    assert sorted(lib.EXPORTS) == names


def test_status_strings_and_defaults():
    L = lib.load_library()
    assert L.msg_strerror(0) == b"ok"
    assert L.msg_strerror(3).startswith(b"unsupported")
    p = lib.default_params()
    assert (p.min_len, p.max_evalue, p.max_nseed, p.mode) == (17, 0.01, 500, 0)
    assert (p.match, p.mismatch, p.gap_open, p.gap_ext) == (1, 3, 5, 2)
    m = lib.mem_params()  # msgseqtk-clean defaults: --min-seed 17, --max-evalue 0.01
    assert (m.min_len, m.max_evalue) == (17, 0.01)


def test_null_arguments_rejected_without_device():
    L = lib.load_library()
    assert L.msg_ctx_create(0, None) == lib.MSG_EINVAL
    assert L.msg_index_load(None, None, None) == lib.MSG_EINVAL
    assert L.msg_ctx_share_index(None, None) == lib.MSG_EINVAL
    assert L.msg_db_read_device(0, None, None, None, None) == lib.MSG_EINVAL
    assert L.msg_map_batch(None, None, None, None, None) == lib.MSG_EINVAL
    assert L.msg_last_stats(None, None) == lib.MSG_EINVAL
    assert L.msg_mem_batch(None, None, None, None, None, None, 0, None) == lib.MSG_EINVAL
    assert L.msg_clean_batch(None, None, None, None, None, 0.0, None, None, None, None) == lib.MSG_EINVAL
    assert L.msg_clean_batch_device(None, None, None, None, None, 0.0, None, None, None, None) == lib.MSG_EINVAL
