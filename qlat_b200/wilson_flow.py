"""Gradient flow and clover observables with qlat's Python API
(qlat/qlat/wilson_flow.pyx:38-122, topology.pyx:75-96).
"""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import call
from .field import FieldRealD, GaugeField, GaugeMomentum


def gf_wilson_flow_force(gf: GaugeField, c1: float = 0.0) -> GaugeMomentum:
    """wilson_flow.pyx:75-79 -> set_wilson_flow_z (force at beta = 3)."""
    z = GaugeMomentum(gf.geo, precision=gf.precision)
    call("qgb_set_wilson_flow_z", z.handle, gf.handle, float(c1))
    return z


def gf_wilson_flow_step(gf: GaugeField, epsilon: float, *, c1: float = 0.0,
                        wilson_flow_integrator_type: str | None = None):
    """wilson_flow.pyx:81-93: modifies gf in place (Runge-Kutta by default)."""
    t = wilson_flow_integrator_type or "runge-kutta"
    if t == "runge-kutta":
        call("qgb_gf_wilson_flow_step", gf.handle, float(epsilon), float(c1))
    elif t == "euler":
        call("qgb_gf_wilson_flow_step_euler", gf.handle, float(epsilon), float(c1))
    else:
        raise ValueError(f"unknown wilson_flow_integrator_type {t!r}")


def gf_energy_density(gf: GaugeField) -> float:
    """wilson-flow.cpp:131-141"""
    o = ctypes.c_double()
    call("qgb_gf_energy_density", gf.handle, ctypes.byref(o))
    return o.value


def gf_energy_density_field(gf: GaugeField) -> FieldRealD:
    """wilson-flow.cpp:118-129"""
    fd = FieldRealD(gf.geo, 1, precision=gf.precision)
    call("qgb_gf_energy_density_field", fd.handle, gf.handle)
    return fd


def gf_wilson_flow(gf: GaugeField, flow_time: float, steps: int, *, c1: float = 0.0,
                   existing_flow_time: float = 0.0, wilson_flow_integrator_type: str | None = None) -> list:
    """wilson_flow.pyx:111-122: returns the energy density after each step."""
    t = wilson_flow_integrator_type or "runge-kutta"
    if t == "runge-kutta":
        out = np.zeros(int(steps), dtype=np.float64)
        call("qgb_gf_wilson_flow", gf.handle, float(flow_time), int(steps), float(c1),
             out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return [float(v) for v in out]
    eps = flow_time / steps
    out = []
    for _ in range(int(steps)):
        gf_wilson_flow_step(gf, eps, c1=c1, wilson_flow_integrator_type=t)
        out.append(gf_energy_density(gf))
    return out


def gf_energy_density_dir_field(gf: GaugeField) -> FieldRealD:
    """wilson_flow.pyx:49-63 -> gf_energy_density_dir_field (wilson-flow.cpp:53-95):
    -Re tr(G G) per plane (0,1) (0,2) (0,3) (1,2) (1,3) (2,3), G = TA(clover);
    multiplicity 6, summing to gf_energy_density_field."""
    fd = FieldRealD(gf.geo, 6)
    call("qgb_gf_energy_density_dir_field", fd.handle, gf.handle)
    return fd


def topology_charge_5(gf: GaugeField) -> float:
    """topology_charge_5 (qcd.cpp:376-389): the 5-loop improved charge."""
    o = ctypes.c_double()
    call("qgb_topology_charge_5", gf.handle, ctypes.byref(o))
    return o.value


def gf_energy_derivative_density_field(gf: GaugeField, *, epsilon: float = 0.0125, c1: float = 0.0,
                                       wilson_flow_integrator_type: str | None = None) -> FieldRealD:
    """wilson_flow.pyx:96-108: central difference of the energy density field."""
    gf1 = gf.copy()
    gf_wilson_flow_step(gf1, epsilon, c1=c1, wilson_flow_integrator_type=wilson_flow_integrator_type)
    fd1 = gf_energy_density_field(gf1)
    gf1 @= gf
    gf_wilson_flow_step(gf1, -epsilon, c1=c1, wilson_flow_integrator_type=wilson_flow_integrator_type)
    fd2 = gf_energy_density_field(gf1)
    fd1 -= fd2
    fd1 *= 1 / (2 * epsilon)
    return fd1


def gf_topology_field_clf(gf: GaugeField) -> FieldRealD:
    """topology.pyx:75-86 -> clf_topology_field (qcd.cpp:416-423)."""
    topf = FieldRealD(gf.geo, 1, precision=gf.precision)
    call("qgb_clf_topology_field", topf.handle, gf.handle)
    return topf


def gf_topology_clf(gf: GaugeField) -> float:
    """topology.pyx:89-96"""
    o = ctypes.c_double()
    call("qgb_gf_topology_clf", gf.handle, ctypes.byref(o))
    return o.value


def gf_topology_field(gf: GaugeField) -> FieldRealD:
    """topology.pyx:98-108 -> clf_topology_field_5 (qcd.cpp:491-509): the 5-loop
    improved charge density (hep-lat/9701012 Eq. 2-7), multiplicity 1."""
    topf = FieldRealD(gf.geo, 1, precision=gf.precision)
    call("qgb_clf_topology_field_5", topf.handle, gf.handle)
    return topf


def gf_topology(gf: GaugeField) -> float:
    """topology.pyx:110-118: the 5-loop improved charge."""
    o = ctypes.c_double()
    call("qgb_gf_topology", gf.handle, ctypes.byref(o))
    return o.value


def gf_topology_terms_field(gf: GaugeField) -> FieldRealD:
    """topology.pyx:120-128 -> clf_topology_field_5_terms (qcd.cpp:425-489):
    the five terms per site, multiplicity 5; their sum is gf_topology_field."""
    topf = FieldRealD(gf.geo, 5, precision=gf.precision)
    call("qgb_clf_topology_field_5_terms", topf.handle, gf.handle)
    return topf


def gf_topology_terms(gf: GaugeField) -> np.ndarray:
    """topology.pyx:130-140: the five terms summed over the lattice, shape (5,)."""
    out = np.zeros(5, dtype=np.float64)
    call("qgb_gf_topology_terms", gf.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out
