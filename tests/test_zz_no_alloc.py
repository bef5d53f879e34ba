"""The allocation-free gauge-action sums (qgb_gf_action_sums_noalloc).

Callers that cannot allocate GPU memory -- a host whose device memory belongs
to its own pool, or one that cannot take the device-wide synchronisation an
allocation may cause -- call this entry point with their own device buffers:
the links in the reference memory image and two doubles of output.  Its
scratch is a fixed array inside the library.

The GPU test allocates the caller's buffers itself (with torch), calls the
entry point twice in a row through the C ABI, and checks both results against
the regular entry points that compute the same sums from a library-owned field.
The CPU tests check the argument checks that run before anything touches the
GPU: extents whose product would wrap a 64-bit integer, lattices beyond the
scratch, and misaligned buffers.  Their pointers are never dereferenced: every
one of these calls is refused before the entry point makes any CUDA call.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest

QGB_ERR_INVALID_ARG = 1
QGB_ERR_BAD_GEOMETRY = 2

# stand-ins for device addresses; the refused calls never use them
FAKE_LINKS = 1 << 20
FAKE_OUT = 1 << 21


def _lib():
    from qlat_b200 import _lib as L
    return L, L.load()


def _call(lib, L, dims, links=FAKE_LINKS, out=FAKE_OUT):
    return lib.qgb_gf_action_sums_noalloc(ctypes.c_void_p(links), L.i32x4(*dims), 1, ctypes.c_void_p(out), None)


@pytest.mark.parametrize("dims", [(1 << 20, 1 << 20, 1 << 20, 16),    # product 2^64: wraps to 0
                                  (1 << 20, 1 << 20, 1 << 20, 17),    # product 17 * 2^60: wraps to 2^60
                                  (1 << 20, 1 << 20, 1 << 4, 1 << 20),
                                  (4096, 4096, 2, 1),                  # 2^25 sites, no wrap
                                  (128, 128, 128, 16)])
def test_noalloc_refuses_lattices_beyond_its_scratch_without_overflow(dims):
    L, lib = _lib()
    assert _call(lib, L, dims) == QGB_ERR_INVALID_ARG
    assert b"at most 16777216 sites" in lib.qgb_last_error()


def test_noalloc_refuses_bad_extents_and_misaligned_buffers():
    L, lib = _lib()
    assert _call(lib, L, (0, 4, 4, 4)) == QGB_ERR_BAD_GEOMETRY
    assert _call(lib, L, (4, 4, 4, (1 << 20) + 1)) == QGB_ERR_BAD_GEOMETRY
    assert _call(lib, L, (4, 4, 4, 4), links=FAKE_LINKS + 8) == QGB_ERR_INVALID_ARG
    assert b"16-byte" in lib.qgb_last_error()
    assert _call(lib, L, (4, 4, 4, 4), out=FAKE_OUT + 4) == QGB_ERR_INVALID_ARG
    assert _call(lib, L, (4, 4, 4, 4), links=0) == QGB_ERR_INVALID_ARG


@pytest.mark.gpu
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
    l0 = q.launch_count()
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
    assert q.launch_count() - l0 == 8  # two kernels per call, counted like every other launch

