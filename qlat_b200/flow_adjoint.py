"""Differentiating through the gradient flow.

Convention: tangents and gradients are su(3) fields acting by left
multiplication, U -> exp(s X) U; a gradient is the su(3) field
sum_a (dL/domega_a) T_a in the basis of matrix-hmc.h:76-106 (tr T_a T_b = -2
delta_ab).  The gauge action's gradient is then -2 x set_gm_force, because
Qlattice's momenta have kinetic energy sum_a p_a^2 (hmc.cpp:151-173).

- ``gf_wilson_flow_vjp``: cotangent at the flowed field -> cotangent at the
  initial field, through RK3 Wilson-flow steps (checkpoints every k steps).
- ``gf_flow_action_grad``: L = gauge action of the flowed field, and dL/dU.
- ``FlowedWilsonAction``: a torch.autograd.Function of the su(3) coordinates
  omega (shape (V, 4, 8)) of U = exp(omega . T) U0.
- ``run_flowed_hmc_pure_gauge``: HMC whose action is the gauge action of the
  flowed field, with the flow adjoint as its force.
"""

from __future__ import annotations

import ctypes
import math

from . import _lib
from ._lib import call
from .field import F64, FieldRealD, GaugeAction, GaugeField, GaugeMomentum, RngState


def set_anti_hermitian_matrix_from_basis(fc, basis: FieldRealD):
    """fc[x, m] = sum_a T_a basis[x, 8 m + a] (hmc.pyx set_anti_hermitian_matrix_from_basis)."""
    call("qgb_set_anti_hermitian_matrix_from_basis", fc.handle, basis.handle)


def set_basis_from_anti_hermitian_matrix(basis: FieldRealD, fc):
    """basis[x, 8 m + a] = coefficient of T_a in fc[x, m] (hmc.pyx set_basis_from_anti_hermitian_matrix)."""
    call("qgb_set_basis_from_anti_hermitian_matrix", basis.handle, fc.handle)


def gf_wilson_flow_vjp(gf: GaugeField, epsilon: float, steps: int, cotangent, *, c1: float = 0.0,
                       checkpoint_every: int = 8) -> GaugeMomentum:
    grad = GaugeMomentum(gf.geo, precision=gf.precision)
    call("qgb_gf_wilson_flow_vjp", gf.handle, float(epsilon), int(steps), float(c1), int(checkpoint_every),
         cotangent.handle, grad.handle)
    return grad


def gf_flow_action_grad(gf: GaugeField, epsilon: float, steps: int, beta: float, *, c1: float = 0.0,
                        c1_loss: float = 0.0, checkpoint_every: int = 8):
    """(L, dL/dU) for L = gf_hamilton_node(V_t, GaugeAction(beta, c1_loss)), V_t the
    field after `steps` RK3 flow steps of size epsilon."""
    grad = GaugeMomentum(gf.geo, precision=gf.precision)
    loss = ctypes.c_double()
    call("qgb_gf_flow_action_grad", gf.handle, float(epsilon), int(steps), float(c1), int(checkpoint_every),
         float(beta), float(c1_loss), grad.handle, ctypes.byref(loss))
    return loss.value, grad


def gf_flow_action(gf: GaugeField, epsilon: float, steps: int, beta: float, *, c1: float = 0.0,
                   c1_loss: float = 0.0) -> float:
    from .hmc import gf_hamilton_node
    from .wilson_flow import gf_wilson_flow_step
    v = gf.copy()
    for _ in range(int(steps)):
        gf_wilson_flow_step(v, epsilon, c1=c1)
    return gf_hamilton_node(v, GaugeAction(beta, c1_loss))


def _omega_field(omega, geo):
    """torch (V, 4, 8) float64 CUDA tensor -> su(3) field."""
    basis = FieldRealD(geo, 32)
    basis.upload_device(omega.contiguous().data_ptr())
    om = GaugeMomentum(geo)
    set_anti_hermitian_matrix_from_basis(om, basis)
    return om


def _basis_tensor(field, V):
    import torch
    basis = FieldRealD(field.geo, 32)
    set_basis_from_anti_hermitian_matrix(basis, field)
    out = torch.empty((V, 32), dtype=torch.float64, device="cuda")
    basis.download_device(out.data_ptr())
    return out.view(V, 4, 8)


def _flowed_point(omega, base):
    u = base.copy()
    om = _omega_field(omega, base.geo)
    call("qgb_gf_evolve", u.handle, om.handle, 1.0)  # u = unitarize(exp(Omega) U0)
    return u, om


def _make_function():
    import torch

    class FlowedWilsonAction(torch.autograd.Function):
        """L(omega) = gf_hamilton_node(V_t(exp(omega . T) U0), GaugeAction(beta, c1_loss)),
        V_t = `steps` RK3 Wilson-flow steps of size epsilon.  omega: (V, 4, 8)
        float64 CUDA tensor of su(3) coordinates; returns a 0-d tensor.  The
        backward pass is the hand-written flow adjoint with checkpointing."""

        @staticmethod
        def forward(ctx, omega, base, epsilon, steps, beta, c1_loss=0.0, checkpoint_every=8):
            torch.cuda.synchronize()
            u, om = _flowed_point(omega.detach(), base)
            loss = gf_flow_action(u, epsilon, steps, beta, c1_loss=c1_loss)
            ctx.save_for_backward(omega.detach())
            ctx.args = (base, epsilon, steps, beta, c1_loss, checkpoint_every)
            return torch.tensor(loss, dtype=torch.float64, device=omega.device)

        @staticmethod
        def backward(ctx, gout):
            (omega,) = ctx.saved_tensors
            base, epsilon, steps, beta, c1_loss, every = ctx.args
            torch.cuda.synchronize()
            u, om = _flowed_point(omega, base)
            _, lam = gf_flow_action_grad(u, epsilon, steps, beta, c1_loss=c1_loss, checkpoint_every=every)
            g = GaugeMomentum(base.geo)
            call("qgb_su3_dexp_adjoint", g.handle, om.handle, lam.handle)
            grad = _basis_tensor(g, base.geo.total_volume)
            return gout * grad, None, None, None, None, None, None

    return FlowedWilsonAction


_fn = None


def FlowedWilsonAction():
    """The torch.autograd.Function class (built on first use, so importing this
    package does not import torch)."""
    global _fn
    if _fn is None:
        _fn = _make_function()
    return _fn


def run_flowed_hmc_pure_gauge(gf: GaugeField, beta: float, traj: int, rs: RngState, *, epsilon: float = 0.05,
                              flow_steps: int = 40, n_step: int = 10, md_time: float = 1.0,
                              checkpoint_every: int = 8, is_always_accept: bool = False):
    """HMC with action S(U) = gf_hamilton_node(V_t(U), GaugeAction(beta, 0)) of the
    flowed field V_t (Wilson flow to t = epsilon * flow_steps), leapfrog molecular
    dynamics with the force -1/2 dS/dU from the flow adjoint, and the RNG splits
    and Metropolis step of run_hmc_pure_gauge (hmc.pyx:190-216).
    Returns (flag, delta_h)."""
    from .hmc import gf_evolve, gm_hamilton_node, metropolis_accept
    rs = rs.split(f"{traj}")
    geo = gf.geo
    u = gf.copy()
    gm = GaugeMomentum(geo)
    gm.set_rand(rs.split("set_rand_gauge_momentum"), 1.0)
    s0 = gf_flow_action(u, epsilon, flow_steps, beta)
    h0 = gm_hamilton_node(gm) + s0
    dt = md_time / n_step
    for _ in range(n_step):
        gf_evolve(u, gm, 0.5 * dt)
        _, grad = gf_flow_action_grad(u, epsilon, flow_steps, beta, checkpoint_every=checkpoint_every)
        call("qgb_field_axpby", gm.handle, -0.5 * dt, grad.handle, 1.0)  # gm += dt * (-1/2 grad)
        gf_evolve(u, gm, 0.5 * dt)
    u.unitarize()
    s1 = gf_flow_action(u, epsilon, flow_steps, beta)
    delta_h = gm_hamilton_node(gm) + s1 - h0
    flag, _ = metropolis_accept(delta_h, traj, rs.split("metropolis_accept"))
    if flag or is_always_accept:
        gf @= u
    return flag, delta_h
