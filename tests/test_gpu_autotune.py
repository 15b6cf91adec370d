"""Launch-configuration autotuner (tdbem_md_autotune).

It must time at least the configuration the handle had plus alternatives,
keep one no slower than the set-up heuristic's on its own timing, leave a
valid configuration on the handle, and change the march's results by
rounding only (FP64, tight tolerance: 1e-10 of the displacement scale).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("loads,precision", [(4, "fp64"), (1, "fp64"), (8, "mixed")])
def test_autotune_keeps_results(loads, precision):
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    c = cases.config_rod5_batched(nstep=24, n=2, loads=loads, error=1e-13)
    s = MultiDomainSolver(c, precision=precision, n_loads=loads)
    s.assemble()
    lu0, lt0, rep0 = s.march(c.known)
    assert rep0.failed_step == 0
    t = s.autotune(c.known, steps=16)
    assert t.candidates >= 2 and t.steps == 16
    assert t.ms_per_step <= t.ms_per_step_default
    assert t.gmres_groups >= 1 and loads % t.gmres_groups == 0 and t.gmres_cluster >= 1
    assert t.rhs_cases_per_thread in ((4, 2) if loads >= 4 else (loads,))
    lu1, lt1, rep1 = s.march(c.known)
    assert rep1.failed_step == 0
    assert rep1.gmres_groups == t.gmres_groups and rep1.gmres_cluster == t.gmres_cluster
    tol = 1e-10 if precision == "fp64" else 1e-6
    assert np.max(np.abs(lu1 - lu0)) <= tol * np.max(np.abs(lu0))
    assert np.max(np.abs(lt1 - lt0)) <= tol * np.max(np.abs(lt0))
