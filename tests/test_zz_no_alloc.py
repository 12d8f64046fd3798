"""msg_smem_batch_noalloc: seeding for callers that cannot allocate device
memory while mapping (their GPU memory belongs to another allocator). It must
give exactly the SMEM lists the allocating entry point (msg_map_batch) gives,
on two calls in a row, since the static working array keeps the previous
call's contents. Collected last so that a failure here leaves every other
test already run."""
import os

import numpy as np
import pytest

from msgseqtk_b200 import lib

pytestmark = pytest.mark.gpu


def test_noalloc_seeding_matches_allocating_entry_point():
    import torch
    from conftest import Case

    case = Case("repeats")
    ctx = lib.Context(0)
    try:
        ctx.load_index(case.view)
        n = len(case.read_off) - 1
        d_seq = torch.from_numpy(case.reads).cuda()
        d_off = torch.from_numpy(case.read_off).cuda()
        for k in range(case.n_params):
            ps = case.params(k)
            params = lib.default_params(min_len=ps["min_len"], max_evalue=ps["max_evalue"],
                                        max_nseed=ps["max_nseed"], mode=ps["mode"])
            ref = ctx.map(case.reads, case.read_off, params, dump=True)  # allocating entry point
            want_cnt = np.diff(ref["smem_off"])
            cap = int(want_cnt.max()) + 3
            out = torch.empty(n * cap * 6, dtype=torch.int64, device="cuda")
            cnt = torch.empty(n, dtype=torch.int32, device="cuda")
            for call in range(2):
                out.fill_(-11 - call)
                cnt.fill_(-1)
                torch.cuda.synchronize()
                rc = ctx.smem_noalloc(d_seq.data_ptr(), d_off.data_ptr(), n, out.data_ptr(), cap, cnt.data_ptr(),
                                      params)
                assert rc == lib.MSG_OK, (k, call, rc)
                got_cnt = cnt.cpu().numpy()
                rows = out.view(n, cap, 6).cpu().numpy()
                assert np.array_equal(got_cnt, want_cnt), (k, call)
                for i in range(n):
                    want = ref["smem"][ref["smem_off"][i]:ref["smem_off"][i + 1]]
                    assert np.array_equal(rows[i, :got_cnt[i]], want), (k, call, i)
        # too small an output reports the needed counts
        out = torch.empty(n * 1 * 6, dtype=torch.int64, device="cuda")
        rc = ctx.smem_noalloc(d_seq.data_ptr(), d_off.data_ptr(), n, out.data_ptr(), 1, cnt.data_ptr(),
                              lib.default_params())
        ref = ctx.map(case.reads, case.read_off, lib.default_params(), dump=True)
        if np.diff(ref["smem_off"]).max() > 1:
            assert rc == lib.MSG_EINVAL
            assert np.array_equal(cnt.cpu().numpy(), np.diff(ref["smem_off"]))
        # reads above the static length limit are rejected
        long_seq = torch.from_numpy(np.concatenate([case.reads[:100], np.ones(400, np.uint8)])).cuda()
        long_off = torch.tensor([0, 100, 500], dtype=torch.int64, device="cuda")
        out = torch.empty(2 * 8 * 6, dtype=torch.int64, device="cuda")
        rc = ctx.smem_noalloc(long_seq.data_ptr(), long_off.data_ptr(), 2, out.data_ptr(), 8, cnt.data_ptr(),
                              lib.default_params())
        assert rc == lib.MSG_EINVAL
    finally:
        ctx.close()
