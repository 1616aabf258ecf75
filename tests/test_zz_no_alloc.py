"""The allocation-free BFS entry point (gsw_bfs_strict_noalloc), called through
the C ABI with device buffers the caller owns, gives the same levels as the
regular entry point (gsw_bfs with the STRICT push expand forced) - integer
levels, so bit for bit - on two calls in a row, and rejects sizes beyond its
fixed working memory.  It is for callers that cannot allocate device memory
(a host framework's memory pool owns the device, or cudaMalloc's device-wide
synchronisation is unaffordable).  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

import gswitch_b200 as gs
import oracle

pytestmark = pytest.mark.gpu


def _noalloc_call(torch, off, col, root):
    dev = torch.device("cuda", 0)
    d_off = torch.from_numpy(off).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    n = len(off) - 1
    d_lv = torch.full((n,), 7, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = gs.lib().gsw_bfs_strict_noalloc(n, len(col), d_off.data_ptr(), d_col.data_ptr(), root, d_lv.data_ptr(),
                                         ctypes.c_void_p(stream))
    torch.cuda.synchronize(dev)
    return rc, d_lv.cpu().numpy()


def _noalloc_levels(torch, h, root):
    rc, lv = _noalloc_call(torch, h.off, h.col, root)
    assert rc == 0, gs.lib().gsw_last_error_string()
    return lv


def test_noalloc_matches_regular_entry_point_twice():
    import torch

    graphs = [(oracle.rmat(14, 16, seed=1), 0), (oracle.grid(60, 70, 100, seed=4), 17)]
    with gs.Context(0) as ctx:
        for h, root in graphs:
            g = ctx.upload(h.off, h.col)
            ref, _ = g.bfs(root, "Push-Queue-STRICT-Standalone")
            assert np.array_equal(ref, oracle.bfs(h, root))
            first = _noalloc_levels(torch, h, root)
            second = _noalloc_levels(torch, h, root)  # reuses the same fixed memory
            assert np.array_equal(first, ref)
            assert np.array_equal(second, ref)
            g.close()


def test_noalloc_rejects_sizes_beyond_its_fixed_memory():
    # rejected before any device access, so no buffers are needed
    rc = gs.lib().gsw_bfs_strict_noalloc((1 << 18) + 1, 10, ctypes.c_void_p(16), ctypes.c_void_p(16), 0,
                                         ctypes.c_void_p(16), None)
    assert rc == 6
    assert b"2^18" in gs.lib().gsw_last_error_string()
    rc = gs.lib().gsw_bfs_strict_noalloc(100, (1 << 28) + 1, ctypes.c_void_p(16), ctypes.c_void_p(16), 0,
                                         ctypes.c_void_p(16), None)
    assert rc == 6


def test_noalloc_reports_out_of_range_column_as_invalid_argument():
    """A column index >= n in the caller's CSR is an argument error, not a
    capacity problem; the kernel skips that arc (it checks every index before
    touching the levels) and the call still works afterwards."""
    import torch

    h = oracle.rmat(10, 8, seed=3)
    col = h.col.copy()
    col[h.off[0]] = h.n + 5  # the root's first arc, so the search reaches it
    rc, _ = _noalloc_call(torch, h.off, col, 0)
    assert rc == 1
    assert b"column index out of range" in gs.lib().gsw_last_error_string()
    assert np.array_equal(_noalloc_levels(torch, h, 0), oracle.bfs(h, 0))
