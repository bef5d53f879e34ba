"""Failures made on the host, as the library's callers meet them: NaN links,
a geometry out of range, an allocation the device cannot serve.  Each comes
back as a QlatB200Error with its status code (the reference raises
RuntimeError through `except +`), and the library stays usable afterwards.
Nothing here faults or stalls the GPU: the bad values are ordinary data and
the failing cudaMalloc returns an error code.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

QGB_ERR_BAD_GEOMETRY, QGB_ERR_ALLOC, QGB_ERR_NAN = 2, 3, 5


def _create(dims, precision=64):
    from qlat_b200._lib import call
    h = ctypes.c_void_p()
    call("qgb_field_create", ctypes.byref(h), (ctypes.c_int32 * 4)(*dims), 4, 0, precision)
    return h


def test_nan_links_are_reported(q):
    geo = q.Geometry((4, 4, 4, 8))
    gf = q.GaugeField(geo)
    q.set_unit(gf)
    arr = np.asarray(gf).copy()
    arr[5, 1, 0, 0] = np.nan
    gf.from_numpy(arr)
    with pytest.raises(q.QlatB200Error) as e:
        q.gf_avg_plaq(gf)
    assert e.value.code == QGB_ERR_NAN
    gm = q.GaugeMomentum(geo)
    gm.set_rand(q.RngState("nan"), 1.0)
    with pytest.raises(q.QlatB200Error) as e:
        q.run_hmc_evolve_pure_gauge(gm, gf, q.GaugeAction(2.13, -0.331), None, 2)
    assert e.value.code == QGB_ERR_NAN
    q.set_unit(gf)  # the library goes on working
    assert q.gf_avg_plaq(gf) == 1.0


def test_bad_geometry_is_reported(q):
    for dims in ((0, 4, 4, 4), (4, 4, 4, 1 << 21)):
        with pytest.raises(q.QlatB200Error) as e:
            _create(dims)
        assert e.value.code == QGB_ERR_BAD_GEOMETRY


def test_failed_allocation_is_reported(q):
    # 2^31 sites of FP64 links: 1.2 TB, far beyond the device
    with pytest.raises(q.QlatB200Error) as e:
        _create((256, 256, 256, 128))
    assert e.value.code == QGB_ERR_ALLOC
    gf = q.GaugeField(q.Geometry((4, 4, 4, 4)))  # the next allocation succeeds
    q.set_unit(gf)
    assert q.gf_avg_plaq(gf) == 1.0
