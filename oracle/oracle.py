"""ctypes front end of the CPU oracle (``oracle/qgauge_oracle.c``).

TEST INFRASTRUCTURE ONLY.  The parity tests, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` use this module as the checker; the
``qlat_b200`` package never imports it.

Fields are numpy ``complex128`` arrays of shape ``(V, 4, 3, 3)`` in the
reference's site-major order (x fastest), exactly the memory image of a
Qlattice ``GaugeField`` / ``GaugeMomentum`` (core.h:753-861).  The Python
functions below mirror the reference's Python API where one exists
(hmc.pyx, wilson_flow.pyx, topology.pyx) so that tests read like the
reference's own example scripts.
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_LIB_PATH = os.path.join(_BUILD, "libqgauge_oracle.so")

_dbl_p = ctypes.POINTER(ctypes.c_double)
_int4 = ctypes.c_int * 4


def build(force: bool = False) -> str:
    """Compile the oracle with gcc (no FMA contraction, like the reference's
    x86-64 baseline build).  Returns the path of the shared library."""
    src = os.path.join(_HERE, "qgauge_oracle.c")
    if (not force and os.path.exists(_LIB_PATH)
            and os.path.getmtime(_LIB_PATH) >= os.path.getmtime(src)
            and os.path.getmtime(_LIB_PATH) >= os.path.getmtime(os.path.join(_HERE, "qgauge_oracle.h"))):
        return _LIB_PATH
    os.makedirs(_BUILD, exist_ok=True)
    tmp = _LIB_PATH + f".tmp{os.getpid()}"
    cmd = ["gcc", "-std=gnu11", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           src, "-o", tmp, "-lquadmath", "-lm"]
    subprocess.check_call(cmd)
    os.replace(tmp, _LIB_PATH)
    return _LIB_PATH


class _Rng(ctypes.Structure):
    _fields_ = [
        ("numBytes", ctypes.c_uint64),
        ("hash", ctypes.c_uint32 * 8),
        ("type", ctypes.c_uint64),
        ("index", ctypes.c_uint64),
        ("cache", ctypes.c_uint64 * 3),
        ("gaussian", ctypes.c_double),
        ("cacheAvail", ctypes.c_int32),
        ("gaussianAvail", ctypes.c_int32),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        L = _lib
        R = ctypes.POINTER(_Rng)
        sig = {
            "or_set_log_mode": (None, [ctypes.c_int]),
            "or_rng_reset": (None, [R]),
            "or_rng_seed": (None, [R, ctypes.c_char_p]),
            "or_rng_split": (None, [R, R, ctypes.c_char_p]),
            "or_rng_split_long": (None, [R, R, ctypes.c_int64]),
            "or_rand_gen": (ctypes.c_uint64, [R]),
            "or_u_rand_gen": (ctypes.c_double, [R, ctypes.c_double, ctypes.c_double]),
            "or_g_rand_gen": (ctypes.c_double, [R, ctypes.c_double, ctypes.c_double]),
            "or_rng_export": (None, [ctypes.POINTER(ctypes.c_uint32), R]),
            "or_sha256_final": (None, [ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                                       ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint64]),
            "or_sha256_initial": (None, [ctypes.POINTER(ctypes.c_uint32)]),
            "or_set_unit": (None, [_dbl_p, _int4]),
            "or_set_rand_gauge_momentum": (None, [_dbl_p, _int4, R, ctypes.c_double]),
            "or_set_g_rand_color_matrix_field": (None, [_dbl_p, _int4, R, ctypes.c_double, ctypes.c_int]),
            "or_gf_avg_plaq": (ctypes.c_double, [_dbl_p, _int4]),
            "or_gm_hamilton_node": (ctypes.c_double, [_dbl_p, _int4]),
            "or_gf_sum_re_tr_plaq": (ctypes.c_double, [_dbl_p, _int4]),
            "or_gf_sum_re_tr_rect": (ctypes.c_double, [_dbl_p, _int4]),
            "or_gf_hamilton_node": (ctypes.c_double, [_dbl_p, _int4, ctypes.c_double, ctypes.c_double]),
            "or_set_gm_force": (None, [_dbl_p, _dbl_p, _int4, ctypes.c_double, ctypes.c_double]),
            "or_gf_evolve": (None, [_dbl_p, _dbl_p, _int4, ctypes.c_double]),
            "or_unitarize_field": (None, [_dbl_p, _int4]),
            "or_gf_wilson_flow_step": (None, [_dbl_p, _int4, ctypes.c_double, ctypes.c_double]),
            "or_gf_wilson_flow_step_euler": (None, [_dbl_p, _int4, ctypes.c_double, ctypes.c_double]),
            "or_gf_energy_density_field": (None, [_dbl_p, _dbl_p, _int4]),
            "or_gf_energy_density": (ctypes.c_double, [_dbl_p, _int4]),
            "or_clf_topology_field": (None, [_dbl_p, _dbl_p, _int4]),
            "or_gf_topology_clf": (ctypes.c_double, [_dbl_p, _int4]),
            "or_clf_topology_field_5_terms": (None, [_dbl_p, _dbl_p, _int4]),
            "or_gf_topology": (ctypes.c_double, [_dbl_p, _int4]),
            "or_run_hmc_evolve_fg": (ctypes.c_double, [_dbl_p, _dbl_p, _int4, ctypes.c_double, ctypes.c_double,
                                                       ctypes.c_int, ctypes.c_double]),
            "or_run_hmc_evolve_leapfrog": (ctypes.c_double, [_dbl_p, _dbl_p, _int4, ctypes.c_double,
                                                             ctypes.c_double, ctypes.c_int, ctypes.c_double]),
            "or_field_set_u_rand": (None, [_dbl_p, _int4, ctypes.c_int, R, ctypes.c_double, ctypes.c_double]),
            "or_field_set_g_rand": (None, [_dbl_p, _int4, ctypes.c_int, R, ctypes.c_double, ctypes.c_double]),
            "or_set_rand_gauge_momentum_fa": (None, [_dbl_p, _dbl_p, _int4, R]),
            "or_gm_hamilton_node_fa": (ctypes.c_double, [_dbl_p, _dbl_p, _int4]),
            "or_gf_evolve_fa": (None, [_dbl_p, _dbl_p, _dbl_p, _int4, ctypes.c_double, ctypes.c_int]),
            "or_set_gm_force_dual": (None, [_dbl_p, _dbl_p, _dbl_p, _int4]),
            "or_project_gauge_transform": (ctypes.c_double, [_dbl_p, _dbl_p, _dbl_p, _dbl_p, _int4]),
            "or_set_gauge_transform_momentum": (None, [_dbl_p, _dbl_p, _dbl_p, _int4]),
            "or_dot_gauge_momentum": (None, [_dbl_p, _dbl_p, _dbl_p, _int4]),
            "or_gf_plaq_field": (None, [_dbl_p, _dbl_p, _int4]),
            "or_gf_energy_density_dir_field": (None, [_dbl_p, _dbl_p, _int4]),
            "or_gf_avg_wilson_loop_normalized_tr": (ctypes.c_double, [_dbl_p, _int4, ctypes.c_int, ctypes.c_int]),
            "or_clf_plaq_action_density_field": (None, [_dbl_p, _dbl_p, _int4, ctypes.c_int]),
            "or_set_plaq_flow_z": (None, [_dbl_p, _dbl_p, _dbl_p, _int4]),
            "or_gf_flow_topo_plaq": (ctypes.c_double, [_dbl_p, _int4, ctypes.c_double, ctypes.c_int]),
            "or_make_matrix_exp": (None, [_dbl_p, _dbl_p, ctypes.c_int]),
            "or_unitarize": (None, [_dbl_p]),
            "or_make_tr_less_anti_herm": (None, [_dbl_p, _dbl_p]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def set_log_mode(mode: int) -> None:
    """0: C library log (the reference); 1: correctly rounded log (binary128)."""
    lib().or_set_log_mode(int(mode))


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    assert a.dtype in (np.complex128, np.float64)
    return a.ctypes.data_as(_dbl_p)


def _dims(total_site) -> "ctypes.Array":
    return _int4(*[int(v) for v in total_site])


class RngState:
    """Mirror of the reference ``RngState`` (rng-state.h:38-99)."""

    def __init__(self, seed: str | None = None):
        self._s = _Rng()
        if seed is None:
            lib().or_rng_reset(ctypes.byref(self._s))
        else:
            lib().or_rng_seed(ctypes.byref(self._s), str(seed).encode())

    def split(self, sindex) -> "RngState":
        r = RngState.__new__(RngState)
        r._s = _Rng()
        if isinstance(sindex, int):
            lib().or_rng_split_long(ctypes.byref(r._s), ctypes.byref(self._s), sindex)
        else:
            lib().or_rng_split(ctypes.byref(r._s), ctypes.byref(self._s), str(sindex).encode())
        return r

    def copy(self) -> "RngState":
        r = RngState.__new__(RngState)
        r._s = _Rng()
        ctypes.memmove(ctypes.byref(r._s), ctypes.byref(self._s), ctypes.sizeof(_Rng))
        return r

    def rand_gen(self) -> int:
        return int(lib().or_rand_gen(ctypes.byref(self._s)))

    def u_rand_gen(self, upper: float = 1.0, lower: float = 0.0) -> float:
        return lib().or_u_rand_gen(ctypes.byref(self._s), upper, lower)

    def g_rand_gen(self, center: float = 0.0, sigma: float = 1.0) -> float:
        return lib().or_g_rand_gen(ctypes.byref(self._s), center, sigma)

    def export(self) -> np.ndarray:
        v = (ctypes.c_uint32 * 24)()
        lib().or_rng_export(v, ctypes.byref(self._s))
        return np.array(list(v), dtype=np.uint32)

    @property
    def ptr(self):
        return ctypes.byref(self._s)


def sha256_hex(data: bytes) -> str:
    h0 = (ctypes.c_uint32 * 8)()
    lib().or_sha256_initial(h0)
    out = (ctypes.c_uint32 * 8)()
    lib().or_sha256_final(out, h0, 0, data, len(data))
    return "".join(f"{w:08x}" for w in out)


def volume(total_site) -> int:
    return int(np.prod([int(v) for v in total_site]))


def new_field(total_site) -> np.ndarray:
    return np.zeros((volume(total_site), 4, 3, 3), dtype=np.complex128)


def set_unit(gf: np.ndarray, total_site) -> None:
    lib().or_set_unit(_p(gf), _dims(total_site))


def set_rand_gauge_momentum(gm, total_site, rs: RngState, sigma: float = 1.0) -> None:
    lib().or_set_rand_gauge_momentum(_p(gm), _dims(total_site), rs.ptr, sigma)


def gf_set_rand(gf, total_site, rs: RngState, sigma: float = 0.5, n_step: int = 1) -> None:
    lib().or_set_g_rand_color_matrix_field(_p(gf), _dims(total_site), rs.ptr, sigma, n_step)


def gf_avg_plaq(gf, total_site) -> float:
    return lib().or_gf_avg_plaq(_p(gf), _dims(total_site))


def gm_hamilton_node(gm, total_site) -> float:
    return lib().or_gm_hamilton_node(_p(gm), _dims(total_site))


def gf_sum_re_tr_plaq(gf, total_site) -> float:
    return lib().or_gf_sum_re_tr_plaq(_p(gf), _dims(total_site))


def gf_sum_re_tr_rect(gf, total_site) -> float:
    return lib().or_gf_sum_re_tr_rect(_p(gf), _dims(total_site))


def gf_hamilton_node(gf, total_site, beta: float, c1: float) -> float:
    return lib().or_gf_hamilton_node(_p(gf), _dims(total_site), beta, c1)


def set_gm_force(gm_force, gf, total_site, beta: float, c1: float) -> None:
    lib().or_set_gm_force(_p(gm_force), _p(gf), _dims(total_site), beta, c1)


def gf_evolve(gf, gm, total_site, step_size: float) -> None:
    lib().or_gf_evolve(_p(gf), _p(gm), _dims(total_site), step_size)


def unitarize(gf, total_site) -> None:
    lib().or_unitarize_field(_p(gf), _dims(total_site))


def gf_wilson_flow_step(gf, total_site, epsilon: float, c1: float = 0.0, integrator: str = "runge-kutta"):
    if integrator == "runge-kutta":
        lib().or_gf_wilson_flow_step(_p(gf), _dims(total_site), epsilon, c1)
    elif integrator == "euler":
        lib().or_gf_wilson_flow_step_euler(_p(gf), _dims(total_site), epsilon, c1)
    else:
        raise ValueError(integrator)


def gf_energy_density_field(gf, total_site) -> np.ndarray:
    fd = np.zeros(volume(total_site), dtype=np.float64)
    lib().or_gf_energy_density_field(_p(fd), _p(gf), _dims(total_site))
    return fd


def gf_energy_density(gf, total_site) -> float:
    return lib().or_gf_energy_density(_p(gf), _dims(total_site))


def gf_wilson_flow(gf, total_site, flow_time: float, steps: int, c1: float = 0.0,
                   existing_flow_time: float = 0.0, integrator: str = "runge-kutta") -> list:
    """wilson_flow.pyx:111-122"""
    eps = flow_time / steps
    out = []
    for _ in range(steps):
        gf_wilson_flow_step(gf, total_site, eps, c1, integrator)
        out.append(gf_energy_density(gf, total_site))
    return out


def clf_topology_field(gf, total_site) -> np.ndarray:
    tf = np.zeros(volume(total_site), dtype=np.float64)
    lib().or_clf_topology_field(_p(tf), _p(gf), _dims(total_site))
    return tf


def gf_topology_clf(gf, total_site) -> float:
    return lib().or_gf_topology_clf(_p(gf), _dims(total_site))


def clf_topology_field_5_terms(gf, total_site) -> np.ndarray:
    """qcd.cpp:425-489: (V, 5) terms of the improved charge density."""
    tf = np.zeros((volume(total_site), 5), dtype=np.float64)
    lib().or_clf_topology_field_5_terms(_p(tf), _p(gf), _dims(total_site))
    return tf


def gf_topology(gf, total_site) -> float:
    """topology.pyx:98-108: the 5-loop improved charge."""
    return lib().or_gf_topology(_p(gf), _dims(total_site))


# ---- field-accelerated HMC (hmc.cpp:121-201, 330-396, 492-645) ----------------
# mass fields: float64 arrays of shape (V, 4); +inf freezes a link


def field_set_u_rand(f: np.ndarray, total_site, rs: RngState, upper: float = 1.0, lower: float = 0.0) -> None:
    """set_u_rand (core.h:1585-1603): f is (V, n) float64 or (V, m, 3, 3) complex128."""
    n = f.size // volume(total_site) * (2 if f.dtype == np.complex128 else 1)
    lib().or_field_set_u_rand(_p(f), _dims(total_site), n, rs.ptr, upper, lower)


def field_set_g_rand(f: np.ndarray, total_site, rs: RngState, center: float = 0.0, sigma: float = 1.0) -> None:
    """set_g_rand (core.h:1617-1636)."""
    n = f.size // volume(total_site) * (2 if f.dtype == np.complex128 else 1)
    lib().or_field_set_g_rand(_p(f), _dims(total_site), n, rs.ptr, center, sigma)


def set_rand_gauge_momentum_fa(gm, mf, total_site, rs: RngState) -> None:
    lib().or_set_rand_gauge_momentum_fa(_p(gm), _p(mf), _dims(total_site), rs.ptr)


def gm_hamilton_node_fa(gm, mf, total_site) -> float:
    return lib().or_gm_hamilton_node_fa(_p(gm), _p(mf), _dims(total_site))


def gf_evolve_fa(gf, gm, mf, total_site, step_size: float) -> None:
    lib().or_gf_evolve_fa(_p(gf), _p(gm), _p(mf), _dims(total_site), step_size, 0)


def gf_evolve_fa_dual(gf, gm_dual, mf_dual, total_site, step_size: float) -> None:
    lib().or_gf_evolve_fa(_p(gf), _p(gm_dual), _p(mf_dual), _dims(total_site), step_size, 1)


def gf_evolve_dual(gf, gm_dual, total_site, step_size: float) -> None:
    lib().or_gf_evolve_fa(_p(gf), _p(gm_dual), None, _dims(total_site), step_size, 1)


def set_gm_force_dual(fd, gf, f, total_site) -> None:
    lib().or_set_gm_force_dual(_p(fd), _p(gf), _p(f), _dims(total_site))


def project_gauge_transform(gm, gm_dual, mf, mf_dual, total_site) -> float:
    return lib().or_project_gauge_transform(_p(gm), _p(gm_dual), _p(mf), _p(mf_dual), _dims(total_site))


def set_gauge_transform_momentum(gm, gm_dual, gtm, total_site) -> None:
    lib().or_set_gauge_transform_momentum(_p(gm), _p(gm_dual), _p(gtm), _dims(total_site))


def dot_gauge_momentum(gm1, gm2, total_site) -> np.ndarray:
    f = np.zeros((volume(total_site), 4), dtype=np.float64)
    lib().or_dot_gauge_momentum(_p(f), _p(gm1), _p(gm2), _dims(total_site))
    return f


# ---- topology-measurement flows (qcd.cpp, wilson-flow.cpp:164-236, instanton_map.py) ----

PLAQ_FLOW_KINDS = {"Shrink": 1, "Freeze": 2, "Localize": 3, "Preserve": 4}


def gf_plaq_field(gf, total_site) -> np.ndarray:
    """qcd.cpp:295-341: (V, 6)."""
    f = np.zeros((volume(total_site), 6), dtype=np.float64)
    lib().or_gf_plaq_field(_p(f), _p(gf), _dims(total_site))
    return f


def gf_energy_density_dir_field(gf, total_site) -> np.ndarray:
    """wilson-flow.cpp:53-95: (V, 6)."""
    f = np.zeros((volume(total_site), 6), dtype=np.float64)
    lib().or_gf_energy_density_dir_field(_p(f), _p(gf), _dims(total_site))
    return f


def gf_avg_wilson_loop_normalized_tr(gf, total_site, l: int, t: int) -> float:
    """qcd-utils.cpp:359-400"""
    return lib().or_gf_avg_wilson_loop_normalized_tr(_p(gf), _dims(total_site), int(l), int(t))


def clf_plaq_action_density_field(gf, total_site, spatial: bool = False) -> np.ndarray:
    """qcd.cpp:33-62, 391-414: (V,)."""
    f = np.zeros(volume(total_site), dtype=np.float64)
    lib().or_clf_plaq_action_density_field(_p(f), _p(gf), _dims(total_site), int(spatial))
    return f


def set_plaq_flow_z(gf, plaq_factor, total_site) -> np.ndarray:
    z = new_field(total_site)
    lib().or_set_plaq_flow_z(_p(z), _p(gf), _p(np.ascontiguousarray(plaq_factor)), _dims(total_site))
    return z


def gf_flow_topo(gf, total_site, step_size: float, flow_type=None, integrator: str = "euler") -> float:
    """instanton_map.py:91-191 on the oracle: returns the flow time taken."""
    if flow_type is None:
        flow_type = "Wilson"
    if flow_type in PLAQ_FLOW_KINDS:
        return lib().or_gf_flow_topo_plaq(_p(gf), _dims(total_site), step_size, PLAQ_FLOW_KINDS[flow_type])
    c1 = {"Wilson": 0.0, "Iwasaki": -0.331, "DBW2": -1.4008}.get(flow_type, flow_type)
    gf_wilson_flow_step(gf, total_site, step_size, float(c1), integrator)
    return step_size


def run_hmc_evolve(gm, gf, total_site, beta, c1, n_step, md_time=1.0, integrator="force-gradient") -> float:
    if integrator == "force-gradient":
        return lib().or_run_hmc_evolve_fg(_p(gm), _p(gf), _dims(total_site), beta, c1, n_step, md_time)
    if integrator == "leapfrog":
        return lib().or_run_hmc_evolve_leapfrog(_p(gm), _p(gf), _dims(total_site), beta, c1, n_step, md_time)
    raise ValueError(integrator)


def metropolis_accept_py(delta_h: float, rs: RngState):
    """hmc.pyx:139-155 (Python API): accept if delta_h <= 0 or u <= exp(-delta_h)."""
    if delta_h <= 0.0:
        return True, 1.0
    accept_prob = math.exp(-delta_h)
    rand_num = rs.u_rand_gen(1.0, 0.0)
    return rand_num <= accept_prob, accept_prob


def metropolis_accept_cpp(delta_h: float, rs: RngState):
    """hmc.cpp:77-105 (C++ API).  The C++ draw is u_rand_gen(rs, 0.0, 1.0),
    i.e. upper=0, lower=1, which yields 1 - u."""
    if delta_h <= 0.0:
        return True, 1.0
    rand_num = rs.u_rand_gen(0.0, 1.0)
    accept_prob = math.exp(-delta_h)
    return rand_num <= accept_prob, accept_prob


def run_hmc_pure_gauge(gf, total_site, beta, c1, traj, rs: RngState, *, n_step=6, md_time=1.0,
                       is_always_accept=False, integrator="force-gradient"):
    """hmc.pyx:190-216 (without the optional reversibility print)."""
    rs = rs.split(f"{traj}")
    gf0 = gf.copy()
    gm = new_field(total_site)
    set_rand_gauge_momentum(gm, total_site, rs.split("set_rand_gauge_momentum"), 1.0)
    delta_h = run_hmc_evolve(gm, gf0, total_site, beta, c1, n_step, md_time, integrator)
    flag, accept_prob = metropolis_accept_py(delta_h, rs.split("metropolis_accept"))
    if flag or is_always_accept:
        gf[...] = gf0
    return flag, delta_h


def make_matrix_exp(a: np.ndarray, max_order: int = 20) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex128).reshape(3, 3)
    out = np.zeros((3, 3), dtype=np.complex128)
    lib().or_make_matrix_exp(_p(out), _p(a), max_order)
    return out
