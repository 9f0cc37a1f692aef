"""cee_jv_screen_noalloc: the JV screen for callers that cannot allocate device memory (a host
whose own pool owns all device memory, or a path that must not allocate while it runs). The
caller hands over a snapshot already in device memory; the entry point keeps its working
memory in fixed file-scope device arrays and allocates nothing.

Its witnesses must equal those of the regular entry point (cee_jv_screen) exactly -- the
integer screen has no tolerance -- on two calls in a row with different snapshots, since the
calls share the file-scope arrays. This file is collected last so that a run stopping at the
first failure has run every other test first; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from cudaedgeelimination_b200 import _native, synth
from helpers import random_graph

pytestmark = pytest.mark.gpu


def device_snapshot(g):
    """The caller-side device copy of a snapshot (allocated by the test, not by the library)."""
    import torch
    xy = np.stack([g.x - g.x.min(), g.y - g.y.min()], axis=1).astype(np.int32)
    arrays = {
        "xy": xy.reshape(-1), "edge_uv": np.stack([g.edge_u, g.edge_v], axis=1).astype(np.int32).reshape(-1),
        "edge_w": g.edge_w.astype(np.int32), "active": g.active.astype(np.uint8),
        "row_offsets": g.row_offsets.astype(np.int32), "neighbors": g.neighbors.astype(np.int32),
        "csr_edge_ids": g.csr_edge_ids.astype(np.int32),
    }
    tensors = {k: torch.from_numpy(np.ascontiguousarray(v)).to("cuda:0") for k, v in arrays.items()}
    view = _native.DeviceGraph()
    view.n, view.dist_type, view.m, view.adjacency = g.n, g.dist_type, g.m, int(g.row_offsets[-1])
    for name, t in tensors.items():
        setattr(view, name, t.data_ptr())
    return view, tensors


def screen_noalloc(g):
    import torch
    view, keep = device_snapshot(g)
    out = torch.full((g.m,), -7, dtype=torch.int32, device="cuda:0")
    stream = torch.cuda.current_stream(0).cuda_stream
    _native.check(None, _native.lib().cee_jv_screen_noalloc(ctypes.byref(view), ctypes.c_void_p(out.data_ptr()),
                                                            ctypes.c_void_p(stream)))
    return out.cpu().numpy()


def test_noalloc_matches_regular_entry_point_twice(ctx):
    import torch
    torch.cuda.set_device(0)
    first = synth.jv_clustered()                      # ~39k CSR slots
    second = random_graph(400, 3000, 21, shuffle=True, active_frac=0.9)
    expected_first, _ = ctx.jv_screen(first)
    expected_second, _ = ctx.jv_screen(second)
    got_first = screen_noalloc(first)
    got_second = screen_noalloc(second)                # reuses the arrays the first call left behind
    np.testing.assert_array_equal(got_first, expected_first)
    np.testing.assert_array_equal(got_second, expected_second)
    assert (got_first >= 0).any() and (got_second >= 0).any()


def test_noalloc_rejects_unsorted_row():
    """A device snapshot whose CSR row is not ascending by neighbour fails validation
    (CEE_ERR_INVALID) instead of screening with the wrong N(a) membership."""
    import torch
    torch.cuda.set_device(0)
    g = synth.jv_small()
    bad = g.copy()
    bad.neighbors = g.neighbors.copy()
    bad.csr_edge_ids = g.csr_edge_ids.copy()
    row = int(np.flatnonzero(np.diff(g.row_offsets) >= 3)[0])
    lo = int(g.row_offsets[row])
    for arr in (bad.neighbors, bad.csr_edge_ids):
        arr[lo], arr[lo + 1] = arr[lo + 1], arr[lo]
    view, keep = device_snapshot(bad)
    out = torch.full((g.m,), -7, dtype=torch.int32, device="cuda:0")
    stream = torch.cuda.current_stream(0).cuda_stream
    status = _native.lib().cee_jv_screen_noalloc(ctypes.byref(view), ctypes.c_void_p(out.data_ptr()),
                                                 ctypes.c_void_p(stream))
    assert status == _native.CEE_ERR_INVALID
    assert b"failed validation" in _native.lib().cee_last_error(None)
    # the next call with a valid snapshot still matches the regular entry point
    np.testing.assert_array_equal(screen_noalloc(g), regular_screen(g))


def regular_screen(g):
    """The regular entry point's witnesses (cee_jv_screen) on a fresh context."""
    from cudaedgeelimination_b200 import Context
    c = Context(0)
    try:
        return c.jv_screen(g)[0]
    finally:
        c.close()


def test_noalloc_rejects_oversize_adjacency():
    view = _native.DeviceGraph()
    view.n, view.dist_type, view.m, view.adjacency = 10, 0, 5, (1 << 22) + 2
    status = _native.lib().cee_jv_screen_noalloc(ctypes.byref(view), ctypes.c_void_p(1), None)
    assert status == _native.CEE_ERR_RANGE
    assert b"exceeds the no-alloc scratch" in _native.lib().cee_last_error(None)
