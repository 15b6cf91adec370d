"""The 3,072-element, 8-domain bar (the benchmark's geometry: 8x8 per face,
E alternating 20/80, nu 0.25, rho 20, beta 0.6, seeded Ricker end traction)
against the reference solver itself, run on this host's cores through the
recording build oracle/_ref/dbem_ref_dump (B200 + host CPU).

48 time steps cover the whole history convolution (the bar's 39 non-empty
history steps are all active from step 40 on).  Both sides run GMRES at
1e-13 with restart 200, as in the reference's own card for this case.
Tolerances: per-step right-hand sides 1e-12 and solutions 1e-10 of their
largest entry over the march, boundary values 1e-10, GMRES inner iterations
within one of the reference's at every step; the 32-load FP64 batch equals
the reference on its load 0 to 1e-10; the 32-load mixed-precision march
(FP32 history blocks, GMRES tolerance 1e-9) stays within 1e-6 of the
reference at every step, relative to that step's largest displacement.
"""
import numpy as np
import pytest

import refrun

pytestmark = pytest.mark.gpu

NSTEP = 48
TIGHT = 1.0e-13


def _rel(a, b):
    b = np.asarray(b)
    a = np.asarray(a).reshape(b.shape)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _per_step_rel(u, ref):
    u = np.asarray(u).reshape(ref.shape)
    scale = np.maximum(np.max(np.abs(ref), axis=1), 1e-12 * np.max(np.abs(ref)))
    return np.max(np.abs(u - ref), axis=1) / scale


@pytest.fixture(scope="module")
def bar8():
    if not refrun.available():
        pytest.skip("the reference build oracle/_ref is absent (built where the reference sources are)")
    from tdbem import cases
    c = cases.config_bar8(nstep=NSTEP, error=TIGHT)
    d = refrun.run_case(c)
    assert int(d["solver_return"][0]) == 1, "the reference march failed"
    assert int(d["steps_recorded"][0]) == NSTEP
    return c, d


def test_bar8_fp64_matches_reference(bar8):
    from tdbem.api import MultiDomainSolver
    c, d = bar8
    s = MultiDomainSolver(c)
    s.assemble()
    assert s.info()["n_history"] == int(d["dof_counts"][2])
    s.set_record(True)
    lu, lt, rep = s.march(c.known[0])
    rhs, x, flags = s.step_record()
    assert rep.failed_step == 0 and rep.steps_solved == NSTEP
    ref_rhs = np.stack([d[f"rhs{k}"] for k in range(1, NSTEP + 1)])
    ref_x = np.stack([d[f"x{k}"] for k in range(1, NSTEP + 1)])
    ref_flags = np.stack([d[f"flag{k}"] for k in range(1, NSTEP + 1)])
    assert _rel(rhs, ref_rhs) <= 1e-12
    assert _rel(x, ref_x) <= 1e-10
    assert _rel(lu, d["bd_lu"]) <= 1e-10
    assert _rel(lt, d["bd_lt"]) <= 1e-10
    assert np.all(flags[:, 0] == 0) and np.all(ref_flags[:, 0] == 0)
    assert np.max(np.abs(flags[:, 2] - ref_flags[:, 2])) <= 1
    s.close()


def _batch_with_reference_load(c):
    from tdbem import cases
    b = cases.config_bar8_batched(nstep=NSTEP, loads=32, error=TIGHT)
    b.known[0] = c.known[0]
    return b


def test_bar8_batched_fp64_load0_matches_reference(bar8):
    from tdbem.api import MultiDomainSolver
    c, d = bar8
    b = _batch_with_reference_load(c)
    s = MultiDomainSolver(b, precision="fp64", n_loads=32)
    s.assemble()
    lu, lt, rep = s.march(b.known)
    assert rep.failed_step == 0
    assert _rel(lu[0], d["bd_lu"]) <= 1e-10
    assert _rel(lt[0], d["bd_lt"]) <= 1e-10
    s.close()


def test_bar8_batched_mixed_load0_within_1e6_of_reference(bar8):
    from tdbem.api import MultiDomainSolver
    c, d = bar8
    b = _batch_with_reference_load(c)
    s = MultiDomainSolver(b, precision="mixed", n_loads=32, tol=1e-9)
    s.assemble()
    lu, lt, rep = s.march(b.known)
    assert rep.failed_step == 0
    err = _per_step_rel(lu[0].reshape(NSTEP + 1, -1), d["bd_lu"])[1:]
    assert float(np.max(err)) <= 1e-6, float(np.max(err))
    s.close()
