"""tc_thumbnail_noalloc: the thumbnail stages computed with a fixed scratch
array instead of device allocations, for callers that cannot call cudaMalloc
(another framework owns the allocator, or the path must not synchronize the
device).  Its output must equal tc_getsdf's stages, which allocate their
scratch, on two calls in a row.  Collected last so that a run stopping at the
first failure has run every other test first."""
import ctypes as C

import numpy as np
import pytest

from tests.golden import cases

pytestmark = pytest.mark.gpu


def stages_allocating(tc, M, N, drp, dcol, W):
    mF, Wv, nc = C.c_int(), C.c_int(), C.c_int()
    st = np.zeros((5, 512, W), np.uint8)
    corners = np.zeros((256, 4), np.int32)
    tc.check(tc.lib().tc_getsdf(M, N, drp.data_ptr(), dcol.data_ptr(), None, C.byref(mF),
                                C.byref(Wv), corners.ctypes.data, 256, C.byref(nc), st.ctypes.data,
                                None))
    assert Wv.value == W
    return st


def stages_noalloc(tc, M, N, drp, dcol, dev):
    import torch
    W = int(512.0 / M * N)
    out = torch.full((5 * 512 * W,), 7, dtype=torch.uint8, device=dev)
    Wv = C.c_int()
    tc.check(tc.lib().tc_thumbnail_noalloc(M, N, drp.data_ptr(), dcol.data_ptr(), None,
                                           out.data_ptr(), C.byref(Wv), None))
    assert Wv.value == W
    return out.cpu().numpy().reshape(5, 512, W)


def test_noalloc_matches_allocating_entry(tc, dev):
    import torch
    for name in ("multi_shape", "rmat16_selfloops"):
        case = next(c for c in cases.MATRIX_CASES if c["name"] == name)
        M, N, rp, col = cases.matrix(case)
        drp = torch.from_numpy(rp).to(dev)
        dcol = torch.from_numpy(col).to(dev)
        W = int(512.0 / M * N)
        want = stages_allocating(tc, M, N, drp, dcol, W)
        for _ in range(2):                       # two calls in a row share the scratch
            got = stages_noalloc(tc, M, N, drp, dcol, dev)
            np.testing.assert_array_equal(got, want, err_msg=name)


def test_noalloc_limits(tc, dev):
    import torch
    # too small for a thumbnail: nothing written, W = 0
    Wv = C.c_int(-1)
    rp = torch.zeros(101, dtype=torch.int32, device=dev)
    col = torch.zeros(1, dtype=torch.int32, device=dev)
    tc.check(tc.lib().tc_thumbnail_noalloc(100, 100, rp.data_ptr(), col.data_ptr(), None, None,
                                           C.byref(Wv), None))
    assert Wv.value == 0
    # wider than the fixed scratch: refused before touching anything
    M, N = 1024, 1024 * 3
    rp = torch.zeros(M + 1, dtype=torch.int32, device=dev)
    st = tc.lib().tc_thumbnail_noalloc(M, N, rp.data_ptr(), col.data_ptr(), None, col.data_ptr(),
                                       C.byref(Wv), None)
    assert st == 6                              # TC_ERR_CAPACITY
