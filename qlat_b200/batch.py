"""Batches of independent pure-gauge HMC chains on one GPU.

A ``ChainBatch`` holds many chains -- each with its own lattice, beta and c1 --
in one concatenated GPU field, and advances all of them together: every
phase of a trajectory is one kernel launch over all chains, recorded once as a
CUDA graph and replayed.  Each chain follows run_hmc_pure_gauge
(hmc.pyx:190-216): ``rs_c.split(f"{traj}")`` for the trajectory,
``.split("set_rand_gauge_momentum")`` for its momenta and
``.split("metropolis_accept")`` for its Metropolis draw.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import call
from .field import RngState

INTEGRATORS = {"force-gradient": 0, "leapfrog": 1}


class ChainBatch:
    def __init__(self, total_sites, betas, c1s=None):
        self.total_sites = [tuple(int(v) for v in ts) for ts in total_sites]
        n = len(self.total_sites)
        self.n = n
        self.betas = [float(b) for b in betas]
        self.c1s = [0.0] * n if c1s is None else [float(c) for c in c1s]
        assert len(self.betas) == n and len(self.c1s) == n
        dims = (ctypes.c_int32 * (4 * n))(*[v for ts in self.total_sites for v in ts])
        beta = (ctypes.c_double * n)(*self.betas)
        c1 = (ctypes.c_double * n)(*self.c1s)
        h = ctypes.c_void_p()
        call("qgb_batch_create", ctypes.byref(h), n, dims, beta, c1)
        self._h = h
        self.volumes = [int(np.prod(ts)) for ts in self.total_sites]

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            try:
                _lib.load().qgb_batch_destroy(self._h)
            except Exception:
                pass
            self._h = None

    @staticmethod
    def _rs_array(rs_list):
        arr = (ctypes.c_uint32 * (24 * len(rs_list)))()
        for i, r in enumerate(rs_list):
            for k in range(24):
                arr[24 * i + k] = r.c[k]
        return arr

    def set_rand(self, rs_list, sigma=0.5, n_step=1):
        """GaugeField.set_rand(rs_c, sigma, n_step) for every chain."""
        call("qgb_batch_set_rand", self._h, self._rs_array(rs_list), float(sigma), int(n_step))

    def trajectory(self, rs_momentum, n_step, md_time=1.0, *, integrator="leapfrog", precision="fp64",
                   reunit_interval=4, use_graph=True):
        """Proposals of every chain; returns the delta_h array."""
        dh = np.zeros(self.n, dtype=np.float64)
        call("qgb_batch_trajectory", self._h, self._rs_array(rs_momentum), int(n_step), float(md_time),
             INTEGRATORS[integrator], 1 if precision == "mixed" else 0, int(reunit_interval), int(bool(use_graph)),
             dh.ctypes.data_as(_lib.c_dbl_p))
        return dh

    def accept(self, flags):
        f = (ctypes.c_int32 * self.n)(*[1 if x else 0 for x in flags])
        call("qgb_batch_accept", self._h, f)

    def run_hmc(self, traj, rs_list, n_step, md_time=1.0, *, integrator="leapfrog", precision="fp64",
                reunit_interval=4, is_always_accept=False):
        """One trajectory of every chain with run_hmc_pure_gauge's RNG splits and
        Metropolis (hmc.pyx:139-155, 190-216), all in the library.
        Returns (flags, delta_h)."""
        dh = np.zeros(self.n, dtype=np.float64)
        flags = np.zeros(self.n, dtype=np.int32)
        call("qgb_batch_run_hmc", self._h, self._rs_array(rs_list), int(traj), int(n_step), float(md_time),
             INTEGRATORS[integrator], 1 if precision == "mixed" else 0, int(reunit_interval),
             int(bool(is_always_accept)), dh.ctypes.data_as(_lib.c_dbl_p),
             flags.ctypes.data_as(_lib.c_i32_p))
        return [bool(f) for f in flags], dh

    def autotune(self, precision="mixed", reps=3):
        """Time the batched force's launch shapes on the current links in the
        precision of `precision`'s molecular dynamics and keep the fastest
        (qgb_batch_autotune); returns (variant, ms per launch)."""
        from .field import F32, F64
        best = ctypes.c_int32()
        ms = ctypes.c_double()
        call("qgb_batch_autotune", self._h, F32 if precision == "mixed" else F64, int(reps), ctypes.byref(best),
             ctypes.byref(ms))
        return best.value, ms.value

    def set_force_variant(self, precision, variant):
        from .field import F32, F64
        call("qgb_batch_set_force_variant", self._h, F32 if precision == "mixed" else F64, int(variant))

    def plaq(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.float64)
        call("qgb_batch_plaq", self._h, out.ctypes.data_as(_lib.c_dbl_p))
        return out

    def chain_to_numpy(self, c: int) -> np.ndarray:
        a = np.empty((self.volumes[c], 4, 3, 3), dtype=np.complex128)
        call("qgb_batch_download_chain", self._h, int(c), a.ctypes.data_as(_lib.c_dbl_p))
        return a

    def chain_from_numpy(self, c: int, arr) -> None:
        a = np.ascontiguousarray(np.asarray(arr, dtype=np.complex128).reshape(self.volumes[c], 4, 3, 3))
        call("qgb_batch_upload_chain", self._h, int(c), a.ctypes.data_as(_lib.c_dbl_p))
