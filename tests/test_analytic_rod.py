"""Config 1 (1x1x5 rod of 5 unit-cube domains, 2x2 per face, E 20, nu 0,
rho 20, beta 0.6, 100 steps, fixed x- end, Heaviside unit axial traction on
the x+ end) against the 1-D analytic rod, the reference's own acceptance
check (tools/run_rod120_100_analytic_validation.py:165-176, 236-275, pass
marks 0.25 absolute and 0.3 relative at the worst step, :54-55):

    u(L, t) = P L / E - 2 P / (E L) sum_n cos(c k_n t) / k_n^2,
    k_n = (n + 1/2) pi / L,  c = sqrt(E / rho),

compared per step with the mean axial displacement of the loaded-end
elements.  The CPU test applies it to the reference's own output for this
case (tests/golden/rod5_n2_tight.npz, GMRES 1e-13); the GPU test to the
library's FP64 march.
"""
import math

import numpy as np
import pytest

from conftest import load_golden

ABS_TOL, REL_TOL = 0.25, 0.3


def analytic_tip(E, rho, length, t, load=1.0, terms=10000):
    """u(L, t) of a rod fixed at x = 0 under a step traction at x = L."""
    c = math.sqrt(E / rho)
    n = np.arange(terms)
    k = (n + 0.5) * math.pi / length
    return load * length / E - 2.0 * load / (E * length) * float(np.sum(np.cos(c * k * t) / (k * k)))


def worst_step(case, bd_lu, dt):
    """(max abs difference, relative difference at that step, step) of the
    loaded-end mean axial displacement against the analytic tip."""
    mesh = case.mesh
    loaded = np.flatnonzero((mesh.domain_of == mesh.domains - 1) & (mesh.face_of == 1))
    m = case.materials[0]
    u = np.asarray(bd_lu).reshape(case.nstep + 1, case.n_elements, 3)
    worst = (0.0, 0.0, 0)
    for s in range(1, case.nstep + 1):
        num = float(np.mean(u[s, loaded, 0]))
        ref = analytic_tip(m.E, m.rho, float(mesh.domains), s * dt)
        diff = abs(num - ref)
        if diff > worst[0]:
            worst = (diff, diff / max(abs(ref), 1e-12), s)
    return worst


def _config1():
    from tdbem import cases
    return cases.config_rod5(nstep=100, error=1e-13)


def test_reference_output_passes_the_analytic_check():
    c = _config1()
    g = load_golden("rod5_n2_tight")
    assert np.array_equal(g["elements"], c.mesh.elements) and np.allclose(g["points"], c.mesh.points)
    from oracle_lib import Oracle
    dt = Oracle(c).dt
    diff, rel, step = worst_step(c, g["bd_lu"], dt)
    assert diff <= ABS_TOL and rel <= REL_TOL, (diff, rel, step)


@pytest.mark.gpu
def test_march_passes_the_analytic_check():
    from tdbem.api import MultiDomainSolver
    c = _config1()
    s = MultiDomainSolver(c)
    s.assemble()
    lu, lt, rep = s.march(c.known[0])
    assert rep.failed_step == 0
    diff, rel, step = worst_step(c, lu, s.info()["dt"])
    assert diff <= ABS_TOL and rel <= REL_TOL, (diff, rel, step)
    # and the same numbers as the reference's march of this case
    g = load_golden("rod5_n2_tight")
    assert abs(diff - worst_step(c, g["bd_lu"], s.info()["dt"])[0]) <= 1e-9
    s.close()
