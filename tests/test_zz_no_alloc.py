"""amj_bucket_build_static, the allocation-free bucket build, against
amj_bucket_build through the C ABI.

It exists for callers that may not allocate device memory (engines that own
every device byte through their own pool, loops that may not wait on the
driver's allocator); its scratch is a fixed area compiled into the library and
shared by every call.  The file name sorts last so a run that stops at the
first failure has run everything else.
"""
import ctypes as C

import numpy as np
import pytest

from accmultiwayjoins_b200 import Context, _lib as L, data

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 20


def run_both(ctx, keys, buckets):
    import torch
    lib = L.load()
    n = keys.shape[0]
    dk = torch.from_numpy(keys).cuda()
    outs = []
    for static in (False, True):
        hk = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
        idx = torch.full((max(n, 1),), -7, dtype=torch.int32, device="cuda")
        bp = torch.full((buckets + 1,), -7, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        if static:
            st = torch.cuda.current_stream().cuda_stream
            rc = lib.amj_bucket_build_static(dk.data_ptr(), n, buckets, hk.data_ptr(), idx.data_ptr(), bp.data_ptr(),
                                             C.c_void_p(st))
        else:
            rc = lib.amj_bucket_build(ctx.handle, dk.data_ptr(), n, buckets, hk.data_ptr(), idx.data_ptr(),
                                      bp.data_ptr())
        L.check(rc, "bucket build")
        torch.cuda.synchronize()
        outs.append((hk.cpu().numpy()[:n], idx.cpu().numpy()[:n], bp.cpu().numpy()))
    return outs


def test_static_scratch_bucket_build_matches_allocating_build():
    with Context(0) as ctx:
        # two full-size calls in a row on the shared scratch, then the edges:
        # one bucket (no sort pass), no keys, and a small call after a large one
        cases = [(300_000, 1 << 18, -(1 << 30), 1 << 30, 1), (MAX_KEYS, 1 << 20, 0, 1 << 18, 2),
                 (5000, 1, -100, 100, 3), (0, 1 << 4, 0, 16, 4), (0, 1, 0, 16, 5), (777, 1 << 20, 0, 1 << 24, 6)]
        for n, buckets, lo, hi, seed in cases:
            keys = data.uniform(n, lo, hi, seed=seed)
            (hk0, ix0, bp0), (hk1, ix1, bp1) = run_both(ctx, keys, buckets)
            assert np.array_equal(bp0, bp1)
            assert np.array_equal(hk0, hk1)
            assert np.array_equal(ix0, ix1)


def test_static_scratch_rejects_sizes_beyond_its_limit():
    import torch
    lib = L.load()
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = buf.data_ptr()
    assert lib.amj_bucket_build_static(p, MAX_KEYS + 1, 1 << 10, p, p, p, None) == L.AMJ_EINVAL
    assert b"fixed scratch limit" in lib.amj_last_error()
    assert lib.amj_bucket_build_static(p, 16, 1 << 21, p, p, p, None) == L.AMJ_EINVAL
