"""The T-step history pass against the one-step pass and the C oracle (B200).

With two or more load cases the march lays the history blocks of steps
k >= 2T + 1 out as runs of consecutive steps and computes their part of the
right-hand sides of steps t0 .. t0 + T - 1 in one launch (bulk_steps_kernel),
beside the GMRES of steps t0 - T .. t0 - 1; the head pass covers k <= 2T.
T = 2, or 3 with TDBEM_HISTORY_STEPS=3 and at least 7 history steps;
TDBEM_RUNS=0 at assembly keeps the one-step pass
(k >= 3 of step s + 1 beside the GMRES of step s).  All compute the sums of
DBEM1/multidomain.cpp:3843-3866 in another order: FP64 agrees to 1e-12, the
mixed-precision march (GMRES to 1e-9) to 1e-8, at step counts where the last
launch's steps lie partly past the march, from the first steps (t0 < K) on,
and one load case of a batch matches the C oracle to 1e-10.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    b = np.asarray(b)
    a = np.asarray(a).reshape(b.shape)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _march(case, precision, loads, runs, tol, steps=None):
    from tdbem.api import MultiDomainSolver
    env = {"TDBEM_RUNS": runs, "TDBEM_HISTORY_STEPS": steps}
    old = {k: os.environ.get(k) for k in env}
    for k, v in env.items():
        if v is not None:
            os.environ[k] = v
    try:
        s = MultiDomainSolver(case, precision=precision, n_loads=loads, tol=tol)
        s.assemble()
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    lu, lt, rep = s.march(case.known)
    s.close()
    return lu, lt, rep


def _steps_per_pass(K, forced=None):
    return 3 if forced == "3" and K >= 7 else 2


def _pass_launches(nstep, T):
    # steps 2, 2 + T, ... launch steps e + T .. e + 2T - 1 while e + T <= nstep
    return sum(1 for e in range(2, nstep + 1, T) if e + T <= nstep)


@pytest.mark.parametrize("steps", [None, "3"])
@pytest.mark.parametrize("loads", [2, 8, 32])
@pytest.mark.parametrize("nstep", [31, 32, 33])
def test_multi_step_fp64_equals_one_step(nstep, loads, steps):
    from tdbem import cases
    c = cases.config_bar8_batched(nstep=nstep, n=2, loads=loads, error=1e-13)
    lu2, lt2, r2 = _march(c, "fp64", loads, "1", 1e-13, steps)
    lu1, lt1, r1 = _march(c, "fp64", loads, "0", 1e-13)
    assert r1.failed_step == 0 and r2.failed_step == 0
    K = r2.history_steps
    assert K >= 5
    T = _steps_per_pass(K, steps)
    assert r1.history_launches == nstep - 2
    assert r2.history_launches == _pass_launches(nstep, T)
    # the same block applications either way, split differently between the
    # head and the history passes
    assert r1.rhs_block_reads == r2.rhs_block_reads
    assert r2.history_block_steps < r1.history_block_steps
    for r in range(loads):
        assert _rel(lu2[r], lu1[r]) <= 1e-12, r
        assert _rel(lt2[r], lt1[r]) <= 1e-12, r


@pytest.mark.parametrize("steps", [None, "3"])
def test_multi_step_mixed_close_to_one_step(steps):
    from tdbem import cases
    c = cases.config_bar8_batched(nstep=40, n=2, loads=32, error=1e-9)
    lu2, _, r2 = _march(c, "mixed", 32, "1", 1e-9, steps)
    lu1, _, r1 = _march(c, "mixed", 32, "0", 1e-9)
    assert r1.failed_step == 0 and r2.failed_step == 0
    assert r2.history_launches == _pass_launches(40, _steps_per_pass(r2.history_steps, steps))
    for r in range(32):
        assert _rel(lu2[r], lu1[r]) <= 1e-8, r


def test_multi_step_load_against_oracle():
    from tdbem import cases
    from oracle_lib import Oracle
    c = cases.config_bar8_batched(nstep=30, n=2, loads=8, error=1e-13, seed=11)
    lu, lt, rep = _march(c, "fp64", 8, "1", 1e-13)
    assert rep.history_launches == _pass_launches(30, _steps_per_pass(rep.history_steps))
    ref = Oracle(c).march(c.known[5])
    assert _rel(lu[5], ref["bd_lu"]) <= 1e-10
    assert _rel(lt[5], ref["bd_lt"]) <= 1e-10


def test_short_history_keeps_one_step_pass():
    """Long time steps (beta 1.5): 4 history steps, so the one-step pass runs
    beside GMRES and no run layout is built."""
    from tdbem import cases
    nstep = 20
    c = cases.make_case("bar2_long_dt", 2, 2, [cases.Material(80.0, 0.25, 20.0)] * 2, 1.5, nstep,
                        [(1.0, (1.0, 0.0, 0.0), cases.heaviside(nstep)),
                         (0.5, (0.0, 1.0, 0.0), cases.heaviside(nstep))], error=1e-13)
    lu2, lt2, r2 = _march(c, "fp64", 2, "1", 1e-13)
    lu1, lt1, r1 = _march(c, "fp64", 2, "0", 1e-13)
    assert 3 <= r2.history_steps < 5
    assert r2.history_launches == r1.history_launches == nstep - 2
    assert np.array_equal(lu2, lu1) and np.array_equal(lt2, lt1)
