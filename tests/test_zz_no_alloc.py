"""The allocation-free gauge-action sums (qgb_gf_action_sums_noalloc).

Callers that cannot allocate GPU memory -- a host whose device memory belongs
to its own pool, or code recording into a CUDA graph, where cudaMalloc during
capture fails -- call this entry point with their own device buffers: the
links in the reference memory image and two doubles of output.  Its scratch is
a fixed array inside the library.  Here the test itself allocates the caller's
buffers (with torch), calls the entry point twice in a row through the C ABI,
and checks both results against the regular entry points that compute the same
sums from a library-owned field.  This file is collected last so that a run
stopping at the first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_action_sums_match_regular_entry_points(q):
    import torch
    from qlat_b200 import _lib

    lib = _lib.load()
    torch.cuda.set_device(0)
    ts = (6, 4, 8, 10)
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState("noalloc").split("gf-init"), 0.4, 2)
    sp_ref = q.gf_sum_re_tr_plaq_node_no_comm(gf)
    sr_ref = q.gf_sum_re_tr_rect_node_no_comm(gf)
    links = torch.from_numpy(np.ascontiguousarray(np.asarray(gf)).view(np.float64).reshape(-1)).cuda()
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    dims = _lib.i32x4(*ts)
    for call in range(2):
        for rect in (1, 0):
            rc = lib.qgb_gf_action_sums_noalloc(ctypes.c_void_p(links.data_ptr()), dims, rect,
                                                ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
            assert rc == 0, lib.qgb_last_error()
            torch.cuda.synchronize()
            sp, sr = out.tolist()
            assert abs(sp - sp_ref) <= 1e-12 * abs(sp_ref), (call, rect, sp, sp_ref)
            if rect:
                assert abs(sr - sr_ref) <= 1e-12 * abs(sr_ref), (call, sr, sr_ref)
            else:
                assert sr == 0.0


def test_noalloc_rejects_lattices_beyond_its_scratch(q):
    import torch
    from qlat_b200 import _lib

    lib = _lib.load()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    links = torch.zeros(8, dtype=torch.float64, device="cuda")  # never read: the size check comes first
    rc = lib.qgb_gf_action_sums_noalloc(ctypes.c_void_p(links.data_ptr()), _lib.i32x4(128, 128, 128, 16), 1,
                                        ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1
    assert b"at most 16777216 sites" in lib.qgb_last_error()
