"""The hand-written adjoint of the Wilson flow (qgb_gf_wilson_flow_vjp,
qgb_gf_flow_action_grad) against finite differences, the zero-flow identity
grad = -2 set_gm_force, the reference's forward flow (oracle), the
torch.autograd.Function over su(3) coordinates, and the flowed-field HMC."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def ip(a, b):
    """<A, B> = sum_a A^a B^a = -1/2 Re tr(A B), summed over links."""
    A, B = np.asarray(a), np.asarray(b)
    return float(-0.5 * np.einsum("smij,smji->", A, B).real)


def fd4(f, h):
    return (8 * (f(h) - f(-h)) - (f(2 * h) - f(-2 * h))) / (12 * h)


def setup(q, ts=(4, 4, 4, 6), sigma=0.3):
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState("flow-adjoint").split("gf-init"), sigma, 2)
    return gf


def test_zero_flow_gradient_is_minus_two_force(q):
    gf = setup(q)
    loss, grad = q.gf_flow_action_grad(gf, 0.05, 0, 2.0)
    F = q.GaugeMomentum(gf.geo)
    q.set_gm_force(F, gf, q.GaugeAction(2.0, 0.0))
    assert np.allclose(np.asarray(grad), -2.0 * np.asarray(F), rtol=0, atol=1e-13)
    assert abs(loss - q.gf_hamilton_node(gf, q.GaugeAction(2.0, 0.0))) < 1e-9


@pytest.mark.parametrize("every", [4, 8])
def test_flow_vjp_matches_finite_differences(q, every):
    gf = setup(q)
    eps, steps, beta = 0.05, 6, 2.0
    loss, grad = q.gf_flow_action_grad(gf, eps, steps, beta, checkpoint_every=every)
    assert abs(loss - q.gf_flow_action(gf, eps, steps, beta)) < 1e-10 * abs(loss)
    worst = 0.0
    for k in range(16):
        X = q.GaugeMomentum(gf.geo)
        X.set_rand(q.RngState(f"direction-{k}"), 1.0)

        def L(h):
            u = gf.copy()
            q.gf_evolve(u, X, h)
            return q.gf_flow_action(u, eps, steps, beta)

        fd = fd4(L, 1e-4)
        worst = max(worst, abs(fd - ip(grad, X)) / abs(fd))
    assert worst < 1e-7, worst


def test_flow_vjp_at_the_differentiation_workload(q):
    """The differentiation workload itself: 16^4, hot start at scale 0.4,
    40 RK3 steps of 0.05 to t = 2, checkpoints every 8, loss = Wilson gauge
    action (beta 5.8) of the flowed field; the adjoint against 4-point central
    finite differences (h = 1e-4, FP64) along 4 random su(3) directions."""
    ts = (16, 16, 16, 16)
    gf = q.GaugeField(q.Geometry(ts))
    gf.set_rand(q.RngState("b200-c4-adjoint").split("gf-init"), 0.4, 1)
    eps, steps, beta = 0.05, 40, 5.8
    loss, grad = q.gf_flow_action_grad(gf, eps, steps, beta, checkpoint_every=8)
    assert abs(loss - q.gf_flow_action(gf, eps, steps, beta)) < 1e-10 * abs(loss)
    for k in range(4):
        X = q.GaugeMomentum(gf.geo)
        X.set_rand(q.RngState(f"c4-direction-{k}"), 1.0)

        def L(h):
            u = gf.copy()
            q.gf_evolve(u, X, h)
            return q.gf_flow_action(u, eps, steps, beta)

        fd = fd4(L, 1e-4)
        assert abs(fd - ip(grad, X)) < 1e-7 * abs(fd), (k, fd, ip(grad, X))


@pytest.mark.parametrize("c1,eps", [(-0.331, 0.03), (-1.4008, 0.01)])
def test_rectangle_flow_vjp_matches_finite_differences(q, c1, eps):
    """Iwasaki and DBW2 flows (flow force GaugeAction(3, c1)), loss with the
    same rectangle coefficient: the adjoint against finite differences.  The
    DBW2 flow of this rough start is unstable at eps = 0.03 (the action grows
    a hundredfold in 5 steps; there the order-20 exponential and the exact one
    whose derivative the adjoint takes part at 2e-7), so it runs at 0.01."""
    gf = setup(q)
    steps, beta = 5, 2.0
    loss, grad = q.gf_flow_action_grad(gf, eps, steps, beta, c1=c1, c1_loss=c1, checkpoint_every=2)
    assert abs(loss - q.gf_flow_action(gf, eps, steps, beta, c1=c1, c1_loss=c1)) < 1e-10 * abs(loss)
    for k in range(8):
        X = q.GaugeMomentum(gf.geo)
        X.set_rand(q.RngState(f"rect-direction-{k}"), 1.0)

        def L(h):
            u = gf.copy()
            q.gf_evolve(u, X, h)
            return q.gf_flow_action(u, eps, steps, beta, c1=c1, c1_loss=c1)

        fd = fd4(L, 1e-4)
        assert abs(fd - ip(grad, X)) < 1e-7 * abs(fd), (k, fd, ip(grad, X))


def test_rectangle_flow_vjp_against_reference_forward(q, oracle):
    """Finite differences of the oracle's Iwasaki flow (c1 = -0.331, the
    reference algorithm) agree with the GPU adjoint."""
    ts = (3, 4, 4, 5)
    gf = setup(q, ts)
    eps, steps, beta, c1 = 0.05, 3, 2.5, -0.331
    _, grad = q.gf_flow_action_grad(gf, eps, steps, beta, c1=c1, checkpoint_every=2)
    U = np.ascontiguousarray(np.asarray(gf))
    for k in range(3):
        X = q.GaugeMomentum(gf.geo)
        X.set_rand(q.RngState(f"ref-rect-direction-{k}"), 1.0)
        Xn = np.ascontiguousarray(np.asarray(X))

        def L(h):
            u = U.copy()
            oracle.gf_evolve(u, Xn, ts, h)
            for _ in range(steps):
                oracle.gf_wilson_flow_step(u, ts, eps, c1)
            return oracle.gf_hamilton_node(u, ts, beta, 0.0)

        fd = fd4(L, 1e-4)
        assert abs(fd - ip(grad, X)) < 1e-7 * abs(fd), (k, fd, ip(grad, X))


def test_flow_vjp_against_reference_forward(q, oracle):
    """Finite differences of the oracle's flow (the reference algorithm) agree with the GPU adjoint."""
    ts = (3, 4, 4, 5)
    gf = setup(q, ts)
    eps, steps, beta = 0.05, 4, 2.5
    _, grad = q.gf_flow_action_grad(gf, eps, steps, beta, checkpoint_every=3)
    U = np.ascontiguousarray(np.asarray(gf))
    for k in range(3):
        X = q.GaugeMomentum(gf.geo)
        X.set_rand(q.RngState(f"ref-direction-{k}"), 1.0)
        Xn = np.ascontiguousarray(np.asarray(X))

        def L(h):
            u = U.copy()
            oracle.gf_evolve(u, Xn, ts, h)
            for _ in range(steps):
                oracle.gf_wilson_flow_step(u, ts, eps, 0.0)
            return oracle.gf_hamilton_node(u, ts, beta, 0.0)

        fd = fd4(L, 1e-4)
        assert abs(fd - ip(grad, X)) < 1e-7 * abs(fd)


def test_torch_autograd_function(q):
    import torch
    torch.cuda.set_device(0)
    gf = setup(q)
    V = gf.geo.total_volume
    fn = q.FlowedWilsonAction()
    gen = torch.Generator(device="cuda").manual_seed(5)
    omega = (0.05 * torch.randn((V, 4, 8), dtype=torch.float64, device="cuda", generator=gen)).requires_grad_()
    loss = fn.apply(omega, gf, 0.05, 5, 2.0)
    loss.backward()
    d = torch.randn((V, 4, 8), dtype=torch.float64, device="cuda", generator=gen)
    with torch.no_grad():
        def L(h):
            return float(fn.apply(omega + h * d, gf, 0.05, 5, 2.0))
        fd = fd4(L, 1e-4)
        an = float((omega.grad * d).sum())
    assert abs(fd - an) < 1e-7 * abs(fd), (fd, an)


def test_flowed_hmc_energy_error_scales_as_dt2(q):
    gf = setup(q, (4, 4, 4, 4), 0.2)
    rs = q.RngState("flowed-hmc")
    dh = []
    for n_step in (4, 8):
        g = gf.copy()
        _, d = q.run_flowed_hmc_pure_gauge(g, 5.8, 1, rs, flow_steps=4, n_step=n_step, md_time=0.5)
        dh.append(abs(d))
    assert dh[1] < dh[0] / 3.0, dh
