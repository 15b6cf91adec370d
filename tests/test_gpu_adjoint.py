"""Adjoint march (tdbem_md_march_vjp) against central differences of the forward march.

The march is linear in the prescribed values, so for any cotangent c and
direction d the central difference of <c, march(k)> along d equals <vjp(c), d>
up to the GMRES tolerance (1e-13 here); the bar for the sensor-misfit
gradient is the 1e-5 relative of central differences.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _hetero_rod(nstep=30, n=2):
    from tdbem import cases
    rng = np.random.default_rng(17)
    mats = [cases.Material(rng.uniform(15, 30), 0.25, rng.uniform(15, 25)) for _ in range(5)]
    return cases.make_case("rod5_adj", 5, n, mats, 0.6, nstep,
                           [(1.0, (0.6, 0.3, -0.2), cases.heaviside(nstep))], error=1e-13)


def test_vjp_matches_central_differences():
    from tdbem.api import MultiDomainSolver
    c = _hetero_rod()
    s = MultiDomainSolver(c)
    s.assemble()
    rng = np.random.default_rng(3)
    shape = (c.nstep + 1, c.n_elements, 3)
    c_lu, c_lt = rng.normal(size=shape), rng.normal(size=shape)
    grad, rep = s.march_vjp(c_lu, c_lt)
    assert rep.failed_step == 0 and rep.steps_solved == c.nstep
    k0 = c.known[0]
    for trial in range(3):
        d = rng.normal(size=shape)
        h = 1e-6 * np.max(np.abs(k0))
        up, ut, _ = s.march(k0 + h * d)
        dn, dt, _ = s.march(k0 - h * d)
        fd = (np.sum(c_lu * (up - dn)) + np.sum(c_lt * (ut - dt))) / (2 * h)
        ad = float(np.sum(grad * d))
        assert abs(fd - ad) <= 1e-7 * max(abs(ad), 1e-300), (trial, fd, ad)


def test_sensor_misfit_gradient():
    """J = sum_n sum_sensors |u_n - u_obs|^2 over 8 lateral-face sensors; the
    gradient with respect to single load-history entries equals central
    differences to 1e-5 relative."""
    from tdbem.api import MultiDomainSolver
    c = _hetero_rod(nstep=40)
    s = MultiDomainSolver(c)
    s.assemble()
    E = c.n_elements
    rng = np.random.default_rng(8)
    sensors = rng.choice(np.where(c.bcid == 456)[0], size=8, replace=False)
    k0 = c.known[0]
    lu0, _, _ = s.march(k0 * 1.1)                      # "observed" from another load
    obs = lu0[:, sensors, :]

    def J(k):
        lu, _, _ = s.march(k)
        return float(np.sum((lu[1:, sensors, :] - obs[1:]) ** 2)), lu

    j0, lu = J(k0)
    cot = np.zeros_like(lu)
    cot[1:, sensors, :] = 2.0 * (lu[1:, sensors, :] - obs[1:])
    grad, _ = s.march_vjp(cot, None)
    loaded = np.where(np.any(np.abs(k0) > 0, axis=(0, 2)))[0]
    for (n, e, comp) in [(1, loaded[0], 0), (7, loaded[1], 1), (20, loaded[-1], 2), (35, loaded[0], 2)]:
        h = 1e-6 * max(abs(k0[n, e, comp]), 1.0)
        kp, km = k0.copy(), k0.copy()
        kp[n, e, comp] += h
        km[n, e, comp] -= h
        fd = (J(kp)[0] - J(km)[0]) / (2 * h)
        assert abs(fd - grad[n, e, comp]) <= 1e-5 * max(abs(fd), 1e-12 * j0), (n, e, comp, fd, grad[n, e, comp])


def test_autograd_function():
    import torch
    from tdbem.api import MultiDomainSolver, march_function
    c = _hetero_rod(nstep=20)
    s = MultiDomainSolver(c)
    s.assemble()
    k = torch.tensor(c.known[0], dtype=torch.float64, requires_grad=True)
    lu, lt = march_function().apply(s, k)
    w = torch.linspace(0.5, 1.5, lu.numel(), dtype=torch.float64).reshape(lu.shape)
    loss = (w * lu).sum() + (lt ** 2).sum() * 1e-3
    loss.backward()
    grad, _ = s.march_vjp(w.numpy(), 2e-3 * lt.detach().numpy())
    assert np.allclose(k.grad.numpy(), grad, rtol=0, atol=1e-12 * np.max(np.abs(grad)))
