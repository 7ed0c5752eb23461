"""Discrete adjoint of the truly linear leapfrog (no reference counterpart).

Pinned three ways: the dot-product identity <M d, l> = <d, M^T l> against
the CUDA forward step; central finite differences (eps = 1e-6) of the CPU
oracle's forward model; the checkpointed misfit gradient against the plain
adjoint sweep for several checkpoint spacings; and the torch.autograd path.
"""
import numpy as np
import pytest

from ptha_b200 import workloads
from pairs import oracle_from_kw


def _domain(nx=90, ny=60, coriolis=True, lin_fric=0.0, seed=6):
    from ptha_b200 import Domain
    kw, U = workloads.spherical_patch(nx=nx, ny=ny, seed=seed)
    kw.update(timestepping_method="linear", coriolis=coriolis, linear_friction_coeff=lin_fric)
    d = Domain(**kw)
    d.set_U(U)
    return kw, U, d


@pytest.mark.gpu
@pytest.mark.parametrize("coriolis,lin_fric", [(True, 0.0), (False, 0.0), (True, 2.0e-4)])
def test_dot_product_identity(coriolis, lin_fric):
    kw, U, d = _domain(coriolis=coriolis, lin_fric=lin_fric)
    dt = d.linear_timestep_max()
    rng = np.random.default_rng(3)
    ny, nx = U.shape[1:]
    for nsteps in (1, 7):
        delta = rng.standard_normal((3, ny, nx))
        lam = rng.standard_normal((3, ny, nx))
        Ud = U.copy()
        Ud[:3] = delta
        d.set_U(Ud)
        d.evolve_steps(nsteps, dt)
        Md = d.get_U()[:3]
        MTl = d.adjoint_linear(nsteps, dt, lambda_seed=lam)
        lhs = float(np.sum(Md * lam))
        rhs = float(np.sum(delta * MTl))
        assert lhs == pytest.approx(rhs, rel=1e-12), (nsteps, lhs, rhs)


@pytest.mark.gpu
def test_misfit_gradient_vs_oracle_finite_differences():
    kw, U, d = _domain(nx=60, ny=40)
    dt = d.linear_timestep_max()
    nsteps = 80
    m = d.metrics()
    sites = [(10, 10), (30, 20), (45, 30), (20, 30), (50, 12)]
    gauges = np.array([[m["x"][i], m["y"][j]] for i, j in sites])
    d.gauges_setup(gauges, capacity=nsteps)
    rng = np.random.default_rng(9)
    target = 0.1 * rng.standard_normal((nsteps, len(sites)))
    loss, grad = d.misfit_gradient(nsteps, dt, target, checkpoint_every=13)

    def oracle_loss(U0):
        o = oracle_from_kw(kw)
        o.U[:] = U0
        L = 0.0
        for n in range(nsteps):
            o.evolve_one_step(dt)
            y = np.array([o.U[0][j, i] for i, j in sites])
            L += 0.5 * float(np.sum((y - target[n]) ** 2))
        return L

    assert loss == pytest.approx(oracle_loss(U), rel=1e-12)
    wet = np.argwhere(U[3] < -20.0)
    pick = wet[rng.choice(len(wet), 16, replace=False)]
    eps = 1e-6
    # L is quadratic in eta0, so central differences have no truncation
    # error; their round-off floor is about eps_mach * L / eps.
    fd_floor = 10 * np.finfo(float).eps * max(loss, 1.0) / eps
    for j, i in pick:
        Up = U.copy(); Up[0, j, i] += eps
        Um = U.copy(); Um[0, j, i] -= eps
        fd = (oracle_loss(Up) - oracle_loss(Um)) / (2 * eps)
        assert grad[0, j, i] == pytest.approx(fd, rel=1e-6, abs=fd_floor), (i, j, grad[0, j, i], fd)


@pytest.mark.gpu
def test_checkpoint_spacing_does_not_change_the_gradient():
    kw, U, d = _domain()
    dt = d.linear_timestep_max()
    nsteps = 60
    m = d.metrics()
    gauges = np.array([[m["x"][i], m["y"][j]] for i, j in [(20, 20), (60, 30), (40, 45)]])
    d.gauges_setup(gauges, capacity=nsteps)
    target = np.zeros((nsteps, 3))
    ref = None
    for K in (1, 7, 60):
        loss, g = d.misfit_gradient(nsteps, dt, target, checkpoint_every=K)
        if ref is None:
            ref = (loss, g)
        assert loss == ref[0]
        assert np.array_equal(g, ref[1])
    # the same gradient from the plain adjoint sweep seeded with the residuals
    d.gauges_reset()
    d.set_U(U)
    d.evolve_steps(nsteps, dt)
    series = d.gauges_read()[:, :, 0]
    g2 = d.adjoint_linear(nsteps, dt, gauge_adjoint=series - target)
    assert np.allclose(g2, ref[1], rtol=1e-12, atol=1e-18)


@pytest.mark.gpu
def test_torch_autograd_function():
    import torch
    from ptha_b200.adjoint import GaugeWaveforms
    kw, U, d = _domain(nx=80, ny=50)
    dt = d.linear_timestep_max()
    nsteps = 40
    m = d.metrics()
    gauges = np.array([[m["x"][i], m["y"][j]] for i, j in [(15, 12), (60, 30), (40, 40)]])
    d.gauges_setup(gauges, capacity=nsteps)
    window = (slice(20, 35), slice(25, 50))
    eta = torch.tensor(U[0][window], dtype=torch.float64, device="cuda", requires_grad=True)
    target = torch.zeros((nsteps, 3), dtype=torch.float64, device="cuda")
    series = GaugeWaveforms.apply(eta, d, U, window, nsteps, dt)
    loss = 0.5 * torch.sum((series - target) ** 2)
    loss.backward()
    d.set_U(U)
    L2, g = d.misfit_gradient(nsteps, dt, target.cpu().numpy(), checkpoint_every=10)
    assert float(loss.detach()) == pytest.approx(L2, rel=1e-12)
    assert np.allclose(eta.grad.cpu().numpy(), g[0][window], rtol=1e-10, atol=1e-20)
