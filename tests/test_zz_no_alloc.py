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


def _noalloc_levels(torch, h, root):
    dev = torch.device("cuda", 0)
    d_off = torch.from_numpy(h.off).to(dev)
    d_col = torch.from_numpy(h.col).to(dev)
    d_lv = torch.full((h.n,), 7, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = gs.lib().gsw_bfs_strict_noalloc(h.n, h.m, d_off.data_ptr(), d_col.data_ptr(), root, d_lv.data_ptr(),
                                         ctypes.c_void_p(stream))
    assert rc == 0, gs.lib().gsw_last_error_string()
    torch.cuda.synchronize(dev)
    return d_lv.cpu().numpy()


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
