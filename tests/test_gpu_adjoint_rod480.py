"""Sensor-misfit gradients on the 480-element rod (5 domains, 4 x 4 elements
per face, 200 steps).

Observations U_obs come from seeded true per-domain materials (E in
[15, 30], rho in [15, 25]); the model starts from materials 10 % away. With
J = sum_n sum_sensors |U_n - U_obs,n|^2 over 8 lateral-face sensor elements,
the forward/backward pair returns dJ/d(known loads) and dJ/d(E_d, rho_d)
for the 10 material parameters, in FP64 (GMRES tolerance 1e-14), and they
are checked against central differences:
- the load history: the march is linear in it, h = 1e-6 relative, to 1e-6;
- every material parameter: h = 1e-6 relative first, to 1e-5.  The discrete
  march is piecewise smooth in the materials (a quadrature point whose r/c
  crosses a multiple of dt moves its contribution to the neighbouring
  history step), so a difference counts only when steps h and 2h agree to
  1e-6; otherwise the next smaller step is taken;
- the exact scaling identity sum_d (E_d dJ/dE_d + rho_d dJ/drho_d) =
  -<dJ/dU, U> (scaling every E and rho by one factor changes no wave
  speed), to 1e-9.
"""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem():
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    truth = cases.config_adjoint_rod(nstep=200, n=4, error=1e-14)
    truth.card = truth.materials[0]
    rng = np.random.default_rng(12)
    mats = [cases.Material(m.E * rng.uniform(0.9, 1.1), m.nu, m.rho * rng.uniform(0.9, 1.1)) for m in truth.materials]
    s = MultiDomainSolver(truth)
    s.assemble()
    obs, _, _ = s.march(truth.known[0])
    s.close()
    c = dataclasses.replace(truth, materials=mats)
    sensors = np.random.default_rng(8).choice(np.where(c.bcid == 456)[0], size=8, replace=False)
    return c, obs, sensors


def _J(c, known, obs, sensors):
    from tdbem.api import MultiDomainSolver
    s = MultiDomainSolver(c)
    s.assemble()
    lu, _, rep = s.march(known)
    s.close()
    assert rep.failed_step == 0
    return float(np.sum((lu[1:, sensors] - obs[1:, sensors]) ** 2))


def _gradients(c, obs, sensors):
    from tdbem.api import MultiDomainSolver
    s = MultiDomainSolver(c)
    s.assemble()
    lu, _, rep = s.march_forward(c.known[0])
    assert rep.steps_solved == c.nstep
    cot = np.zeros_like(lu)
    cot[1:, sensors] = 2.0 * (lu[1:, sensors] - obs[1:, sensors])
    gk, gm, _ = s.march_backward(cot, None)
    s.close()
    return lu, cot, gk, gm


def test_misfit_gradients_against_central_differences(problem):
    from tdbem import cases
    c, obs, sensors = problem
    lu, cot, gk, gm = _gradients(c, obs, sensors)
    E = np.array([m.E for m in c.materials])
    rho = np.array([m.rho for m in c.materials])
    lhs, rhs = float(np.sum(E * gm[:, 0] + rho * gm[:, 1])), -float(np.sum(cot * lu))
    assert abs(lhs - rhs) <= 1e-9 * abs(rhs), (lhs, rhs)

    k0 = c.known[0]
    rng = np.random.default_rng(3)
    for _ in range(2):
        d = rng.normal(size=k0.shape)
        h = 1e-6 * np.max(np.abs(k0))
        fd = (_J(c, k0 + h * d, obs, sensors) - _J(c, k0 - h * d, obs, sensors)) / (2 * h)
        ad = float(np.sum(gk * d))
        assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)

    def J_at(dom, which, rel):
        mm = list(c.materials)
        m = mm[dom]
        mm[dom] = cases.Material(m.E * (1 + rel), m.nu, m.rho) if which == 0 else \
            cases.Material(m.E, m.nu, m.rho * (1 + rel))
        return _J(dataclasses.replace(c, materials=mm), k0, obs, sensors)

    for dom in range(5):
        for which in (0, 1):
            theta = c.materials[dom].E if which == 0 else c.materials[dom].rho
            ad = gm[dom, which]
            fd = None
            for h in (1e-6, 1e-7, 3e-7, 3e-8):
                f1 = (J_at(dom, which, h) - J_at(dom, which, -h)) / (2 * h * theta)
                f2 = (J_at(dom, which, 2 * h) - J_at(dom, which, -2 * h)) / (4 * h * theta)
                if abs(f1 - f2) <= 1e-6 * abs(f1):
                    fd = f1
                    break
            assert fd is not None, ("no smooth step", dom, which)
            assert abs(fd - ad) <= 1e-5 * abs(fd), (dom, which, fd, ad)
