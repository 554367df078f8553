"""Discrete adjoint of upwind WENO5 + TVD-RK3 advection by a B-spline velocity.

The gradient from the reverse sweep must agree, to 1e-6 relative, with
(1) central finite differences (h = 1e-6) of the GPU forward model and
(2) central finite differences of the FP64 CPU oracle forward model (the
reference's routines in its call order), for B-spline coefficients and for
initial level-set values; the pylsmlib autograd Function must return the same
gradients; checkpointing must not change the result."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = (20, 18, 16)
LAT = 4
STEPS = 6


def problem(every=4, steps=STEPS):
    from lsmlib_b200 import adjoint, workloads
    rng = np.random.default_rng(42)
    ax, dx = workloads.axes(N, (-1, -1, -1), (1, 1, 1))
    theta = rng.normal(0.0, 0.5, size=(3, LAT, LAT, LAT))
    phi0 = workloads.union_of_spheres(ax, [(0.05, -0.1, 0.0)], [0.45])
    x, y, z = ax[0][:, None, None], ax[1][None, :, None], ax[2][None, None, :]
    target = np.asfortranarray(
        (np.sqrt((x / 0.55) ** 2 + (y / 0.45) ** 2 + (z / 0.4) ** 2) - 1.0) * 0.4)
    p = adjoint.AdvectionAdjoint(N, dx, (-1.0, -1.0, -1.0), LAT, steps, every)
    p.set_theta(theta)
    dt = p.cfl_dt(0.5)
    p.set_dt(dt)
    eps = 1.5 * dx[0]
    p.set_fields(phi0, target, eps)
    return p, theta, phi0, target, dx, dt, eps


def fd_theta(p, theta, idx, h=1e-6):
    t = theta.copy()
    t[idx] += h
    p.set_theta(t)
    lp = p.forward()
    t[idx] -= 2 * h
    p.set_theta(t)
    lm = p.forward()
    p.set_theta(theta)
    return (lp - lm) / (2 * h)


def test_gradient_matches_gpu_finite_differences():
    p, theta, phi0, target, dx, dt, eps = problem()
    loss = p.forward()
    gt, gp = p.backward()
    assert loss > 0
    rng = np.random.default_rng(0)
    flat = np.argsort(-np.abs(gt).ravel())[:6].tolist() + \
        rng.choice(gt.size, 4, replace=False).tolist()
    for q in flat:
        idx = np.unravel_index(q, gt.shape)
        fd = fd_theta(p, theta, idx)
        assert abs(fd - gt[idx]) <= 1e-6 * max(abs(fd), 1e-3 * np.max(np.abs(gt))), \
            (idx, fd, gt[idx])
    # initial level-set values near the interface
    cells = np.argwhere(np.abs(phi0[3:-3, 3:-3, 3:-3]) < 3 * dx[0])[:: 97][:5] + 3
    for c in map(tuple, cells):
        ph = phi0.copy(order="F")
        ph[c] += 1e-6
        p.set_fields(ph, target, eps)
        lp = p.forward()
        ph[c] -= 2e-6
        p.set_fields(ph, target, eps)
        lm = p.forward()
        fd = (lp - lm) / 2e-6
        assert abs(fd - gp[c]) <= 1e-6 * max(abs(fd), 1e-3 * np.max(np.abs(gp))), (c, fd, gp[c])
    p.set_fields(phi0, target, eps)


def test_gradient_matches_cpu_oracle_finite_differences():
    """The FP64 CPU path: the oracle's reference-order TVD-RK3 chain with the
    same velocity (host B-spline evaluation) and the same frozen dt."""
    import oracle
    from lsmlib_b200.adjoint import spline_velocity
    from oracle.driver import Grid, Stepper
    p, theta, phi0, target, dx, dt, eps = problem()
    p.forward()
    gt, _ = p.backward()
    g = Grid(N, dx=dx)
    st = Stepper(oracle.oracle_toolbox(), g)
    vol = dx[0] * dx[1] * dx[2]

    def cpu_loss(th):
        vel = [g.field(v) for v in spline_velocity(th, N, dx, (-1, -1, -1), LAT)]
        phi = g.field(phi0.copy(order="F"))  # the oracle steps in place
        for _ in range(STEPS):
            st.advect_step(phi, lambda c: vel, dt)
        d = oracle.heaviside(g.interior(phi), eps) - oracle.heaviside(g.interior(g.field(target)), eps)
        return float(np.sum(d * d) * vol)

    for q in np.argsort(-np.abs(gt).ravel())[:4]:
        idx = np.unravel_index(q, gt.shape)
        th = theta.copy()
        th[idx] += 1e-6
        lp = cpu_loss(th)
        th[idx] -= 2e-6
        lm = cpu_loss(th)
        fd = (lp - lm) / 2e-6
        assert abs(fd - gt[idx]) <= 1e-6 * abs(fd), (idx, fd, gt[idx])


def test_checkpoint_spacing_does_not_change_the_gradient():
    res = []
    for every in (1, 4, STEPS):
        p = problem(every=every)[0]
        p.forward()
        res.append(p.backward())
    # tile-halo contributions are accumulated with atomics, so the summation
    # order (not the arithmetic) varies between runs: compare against the
    # largest component, not cell by cell
    for gt, gp in res[1:]:
        assert np.max(np.abs(gt - res[0][0])) <= 1e-12 * np.max(np.abs(res[0][0]))
        assert np.max(np.abs(gp - res[0][1])) <= 1e-12 * np.max(np.abs(res[0][1]))


def test_torch_autograd_function():
    import torch

    from pylsmlib import advection_loss
    p, theta, phi0, target, dx, dt, eps = problem()
    p.forward()
    gt_ref, gp_ref = p.backward()
    th = torch.tensor(theta, requires_grad=True)
    ph = torch.tensor(np.ascontiguousarray(phi0), requires_grad=True)
    loss = advection_loss(th, ph, p)
    (2.0 * loss).backward()
    for got, ref in ((th.grad.numpy(), 2.0 * gt_ref), (ph.grad.numpy(), 2.0 * gp_ref)):
        assert got.shape == ref.shape
        assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
