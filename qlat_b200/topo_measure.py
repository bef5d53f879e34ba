"""Topology measurement along gradient flows, with qlat's Python API
(qlat/qlat/instanton_map.py:91-224, 1327-1569; qcd.pyx:209-213;
wilson_flow.pyx:65-75; topology.pyx:26-75).

``gf_flow_topo`` takes one step of the Wilson / Iwasaki / DBW2 flow (or a flow
with any c1), or of a plaquette-weighted flow (Shrink, Freeze, Localize,
Preserve) on the GPU.  ``smear_measure_topo`` measures plaquettes, energy
densities, its derivative along the flow, and the clover and 5-loop charges
(totals and per timeslice) before and after each stage of a list of flows, and
records the energy density after every flow step.
"""

from __future__ import annotations

import ctypes
import json
import os
import pickle

import numpy as np

from ._lib import call
from .field import FieldRealD, GaugeField, GaugeMomentum
from .wilson_flow import gf_energy_density_field, gf_topology_field, gf_topology_field_clf, gf_topology_terms

FLOW_TOPO_C1 = 0
_PLAQ_KINDS = {"Shrink": 1, "Freeze": 2, "Localize": 3, "Preserve": 4}
_C1 = {"Wilson": 0.0, "Iwasaki": -0.331, "DBW2": -1.4008}
_INTEGRATORS = {"euler": 0, "runge-kutta": 1}


# ---- site fields and reductions -------------------------------------------------------


def gf_plaq_field(gf: GaugeField) -> FieldRealD:
    """qcd.pyx:209-213 -> gf_plaq_field (qcd.cpp:295-341): Re tr P / 3 per site in
    the planes (0,1) (0,2) (0,3) (1,2) (1,3) (2,3); multiplicity 6."""
    f = FieldRealD(gf.geo, 6)
    call("qgb_gf_plaq_field", f.handle, gf.handle)
    return f


def gf_plaq_action_density_field(gf: GaugeField) -> FieldRealD:
    """topology.pyx:26-40 -> clf_plaq_action_density_field (qcd.cpp:391-403):
    sum over the planes of 1 - Re tr(clover) / 3."""
    f = FieldRealD(gf.geo, 1)
    call("qgb_gf_plaq_action_density_field", f.handle, gf.handle, 0)
    return f


def gf_spatial_plaq_action_density_field(gf: GaugeField) -> FieldRealD:
    """topology.pyx:42-52 -> clf_spatial_plaq_action_density_field (qcd.cpp:405-414)."""
    f = FieldRealD(gf.geo, 1)
    call("qgb_gf_plaq_action_density_field", f.handle, gf.handle, 1)
    return f


def gf_plaq_action_density(gf: GaugeField) -> float:
    """topology.pyx:54-63"""
    return float(glb_sum(gf_plaq_action_density_field(gf))[0, 0]) / gf.geo.total_volume


def gf_spatial_plaq_action_density(gf: GaugeField) -> float:
    """topology.pyx:65-75"""
    return float(glb_sum(gf_spatial_plaq_action_density_field(gf))[0, 0]) / gf.geo.total_volume


def glb_sum_tslice(f: FieldRealD, *, t_dir: int = 3) -> np.ndarray:
    """field_base.pyx:750-762: per-timeslice sums, shape (T, multiplicity)."""
    nt = f.geo.total_site[t_dir]
    out = np.zeros((nt, f.multiplicity), dtype=np.float64)
    call("qgb_field_glb_sum_tslice", f.handle, int(t_dir), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out


def glb_sum(f: FieldRealD) -> np.ndarray:
    """Sum over the lattice of each component, shape (1, multiplicity)."""
    return glb_sum_tslice(f).sum(axis=0, keepdims=True)


def glb_min(f: FieldRealD) -> np.ndarray:
    """Smallest value of each component, shape (1, multiplicity)."""
    out = np.zeros((1, f.multiplicity), dtype=np.float64)
    call("qgb_field_glb_min_max", f.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None)
    return out


def glb_max(f: FieldRealD) -> np.ndarray:
    """Largest value of each component, shape (1, multiplicity)."""
    out = np.zeros((1, f.multiplicity), dtype=np.float64)
    call("qgb_field_glb_min_max", f.handle, None, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out


def field_abs(f: FieldRealD) -> FieldRealD:
    """A copy of f with every entry replaced by its absolute value."""
    g = f.copy()
    call("qgb_field_abs", g.handle)
    return g


# ---- flows ------------------------------------------------------------------------------


def gf_plaq_flow_force(gf: GaugeField, plaq_factor: FieldRealD) -> GaugeMomentum:
    """wilson_flow.pyx:65-75 -> set_plaq_flow_z (wilson-flow.cpp:164-236): the
    Wilson-flow force with each plaquette weighted by plaq_factor (multiplicity
    6, planes as in gf_plaq_field)."""
    z = GaugeMomentum(gf.geo, precision=gf.precision)
    call("qgb_set_plaq_flow_z", z.handle, gf.handle, plaq_factor.handle)
    return z


def _flow_kind(flow_type):
    if flow_type is None:
        flow_type = "Wilson"
    if isinstance(flow_type, (int, float)) and not isinstance(flow_type, bool):
        return FLOW_TOPO_C1, float(flow_type)
    if flow_type in _C1:
        return FLOW_TOPO_C1, _C1[flow_type]
    if flow_type in _PLAQ_KINDS:
        return _PLAQ_KINDS[flow_type], 0.0
    raise ValueError(f"gf_flow_topo: flow_type={flow_type!r}")


def gf_flow_topo(gf: GaugeField, step_size: float, flow_type=None, wilson_flow_integrator_type=None) -> float:
    """instanton_map.py:91-191: one flow step of gf in place; returns the flow
    time taken (step_size, or step_size / norm for the plaquette-weighted
    flows).  flow_type: None / "Wilson" / "Iwasaki" / "DBW2" / a number (c1) /
    "Shrink" / "Freeze" / "Localize" / "Preserve"; integrator "euler" (default)
    or "runge-kutta" (the c1 flows only)."""
    kind, c1 = _flow_kind(flow_type)
    integ = _INTEGRATORS[wilson_flow_integrator_type or "euler"]
    adv = ctypes.c_double()
    call("qgb_gf_flow_topo", gf.handle, float(step_size), kind, c1, integ, ctypes.byref(adv))
    return adv.value


def gf_energy_derivative_density_field_topo(gf: GaugeField, *, epsilon: float = 0.0125, flow_typw=None,
                                            wilson_flow_integrator_type=None) -> FieldRealD:
    """instanton_map.py:193-224: (E(flow(+eps)) - E(flow(-eps))) / (2 eps) per site."""
    gf1 = gf.copy()
    gf_flow_topo(gf1, epsilon, flow_typw, wilson_flow_integrator_type)
    fd1 = gf_energy_density_field(gf1)
    gf1 @= gf
    gf_flow_topo(gf1, -epsilon, flow_typw, wilson_flow_integrator_type)
    fd2 = gf_energy_density_field(gf1)
    fd1 -= fd2
    fd1 *= 1 / (2 * epsilon)
    return fd1


# ---- the measurement driver --------------------------------------------------------------

DEFAULT_SMEAR_INFO_LIST = ([[0.05, 20, "Wilson", "euler"]] * 3 + [[0.01, 50, "DBW2", "euler"]] * 4)


def smear_measure_topo(gf: GaugeField, smear_info_list=None, *, energy_derivative_info=None, info_path=None,
                       density_field_path=None, is_show_topo_terms=False, log=None):
    """instanton_map.py:1327-1569: returns (topo_list, energy_list); gf is
    flowed in place.  topo_list holds one record per measurement (before the
    first stage and after each), energy_list one per flow step.  With
    info_path, the stage list (JSON) and both lists (pickles) are written there
    as the reference does; with density_field_path, the energy density, charge
    density and energy-derivative fields of each measurement are written as
    numpy arrays (the reference writes its own field format)."""
    if smear_info_list is None:
        smear_info_list = [list(v) for v in DEFAULT_SMEAR_INFO_LIST]
    if energy_derivative_info is None:
        energy_derivative_info = [0.0125, 0.0, "euler"]
    geo = gf.geo
    total_volume = geo.total_volume
    spatial_volume = total_volume / geo.total_site[3]
    state = {"flow_time": 0.0}
    topo_list, energy_list = [], []

    def plaq_extremes():
        f_plaq = gf_plaq_field(gf)
        return float(np.min(glb_min(f_plaq))), float(np.max(glb_max(f_plaq)))

    def smear(step_size, n_step, flow_type="Wilson", wilson_flow_integrator_type="euler"):
        flow_time_target = state["flow_time"] + n_step * step_size
        while state["flow_time"] < flow_time_target - step_size / 3:
            state["flow_time"] += gf_flow_topo(gf, step_size, flow_type, wilson_flow_integrator_type)
            plaq = gf.plaq()
            plaq_min, plaq_max = plaq_extremes()
            edf = gf_energy_density_field(gf)
            ed_ts = glb_sum_tslice(edf)
            energy_list.append({
                "flow_time": state["flow_time"], "plaq": plaq, "plaq_min": plaq_min, "plaq_max": plaq_max,
                "energy_density": float(ed_ts.sum()) / total_volume,
                "energy_density_tslice": (ed_ts.ravel() / spatial_volume).tolist(),
            })

    def measure():
        plaq = gf.plaq()
        plaq_min, plaq_max = plaq_extremes()
        paf_ts = glb_sum_tslice(gf_plaq_action_density_field(gf))
        edf = gf_energy_density_field(gf)
        ed_ts = glb_sum_tslice(edf)
        tclf_ts = glb_sum_tslice(gf_topology_field_clf(gf))
        topo_field = gf_topology_field(gf)
        topo_ts = glb_sum_tslice(topo_field)
        abs_topo_ts = glb_sum_tslice(field_abs(topo_field))
        edd = gf_energy_derivative_density_field_topo(gf, epsilon=energy_derivative_info[0],
                                                      flow_typw=energy_derivative_info[1],
                                                      wilson_flow_integrator_type=energy_derivative_info[2])
        edd_ts = glb_sum_tslice(edd)
        rec = {
            "flow_time": state["flow_time"], "plaq": plaq, "plaq_min": plaq_min, "plaq_max": plaq_max,
            "energy_density": float(ed_ts.sum()) / total_volume,
            "energy_density_tslice": (ed_ts.ravel() / spatial_volume).tolist(),
            "energy_deriv": float(edd_ts.sum()) / total_volume,
            "energy_deriv_tslice": (edd_ts.ravel() / spatial_volume).tolist(),
            "topo": float(topo_ts.sum()), "topo_tslice": topo_ts.ravel().tolist(),
            "topo_clf": float(tclf_ts.sum()), "topo_clf_tslice": tclf_ts.ravel().tolist(),
            "abs_topo": float(abs_topo_ts.sum()), "abs_topo_tslice": abs_topo_ts.ravel().tolist(),
            "plaq_action_density": float(paf_ts.sum()) / total_volume,
            "plaq_action_density_tslice": (paf_ts.ravel() / spatial_volume).tolist(),
        }
        if log is not None:
            log(f"smear_measure_topo: t={rec['flow_time']} ; energy_density={rec['energy_density']} ; "
                f"energy_deriv={rec['energy_deriv']} ; topo={rec['topo']}")
        if is_show_topo_terms and log is not None:
            terms = gf_topology_terms(gf)
            log(f"smear_measure_topo: t={rec['flow_time']} ; topo={rec['topo']} ; {float(terms.sum())}")
        if density_field_path is not None:
            d = os.path.join(density_field_path, f"smear-step-{len(topo_list)}")
            os.makedirs(d, exist_ok=True)
            np.save(os.path.join(d, "energy_density.npy"), edf.to_numpy())
            np.save(os.path.join(d, "topo.npy"), topo_field.to_numpy())
            np.save(os.path.join(d, "energy_deriv_density_field.npy"), edd.to_numpy())
        topo_list.append(rec)

    measure()
    for si in smear_info_list:
        smear(*si)
        measure()
    if info_path is not None:
        os.makedirs(info_path, exist_ok=True)
        with open(os.path.join(info_path, "smear-info-list.json"), "w") as f:
            json.dump(smear_info_list, f, indent=2)
        with open(os.path.join(info_path, "info.pickle"), "wb") as f:
            pickle.dump(topo_list, f)
        with open(os.path.join(info_path, "energy-list.pickle"), "wb") as f:
            pickle.dump(energy_list, f)
    return topo_list, energy_list
