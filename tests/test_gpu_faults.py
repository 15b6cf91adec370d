"""Failures injected on the host, none of which faults, traps or hangs the
GPU: a non-finite prescribed load, a singular preconditioner leaf, and a
GMRES failure in one of several load-case groups of one launch (B200).

The reference's behaviour on the same inputs is its own: for the NaN load
the recording reference build is run on this host's cores on the same rod.
"""
import numpy as np
import pytest

import refrun
from conftest import case_from_golden, golden_hist, load_golden

pytestmark = pytest.mark.gpu

NOT_CONVERGED = 4
SINGULAR_BLOCK = 3


def _rel(a, b):
    b = np.asarray(b)
    a = np.asarray(a).reshape(b.shape)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_nan_load_stops_the_march_where_the_reference_does():
    """A NaN in the prescribed traction of step 4: GMRES cannot converge on
    that step's right-hand side, so the march stops at step 4 with the steps
    before it intact, as the reference's march stops on the first
    non-converged step (DBEM1/multidomain.cpp:3884-3885)."""
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    c = cases.config_rod5(nstep=8, error=1e-13)
    loaded = np.flatnonzero(np.any(c.known[0, 1] != 0.0, axis=1))
    c.known[0, 4, loaded[0], 0] = np.nan
    s = MultiDomainSolver(c)
    s.assemble()
    lu, lt, rep = s.march(c.known[0], raise_on_failure=False)
    assert rep.failed_step == 4 and rep.steps_solved == 3 and rep.gmres_flag != 0
    assert np.all(np.isfinite(lu[:4])) and np.all(lu[5:] == 0.0)
    clean = c.known[0].copy()
    clean[4:] = 0.0
    lu0, lt0, _ = s.march(clean)
    assert np.array_equal(lu[1:4], lu0[1:4]) and np.array_equal(lt[1:4], lt0[1:4])
    if refrun.available():
        d = refrun.run_case(c)
        assert int(d["solver_return"][0]) == -1
        assert int(d["steps_recorded"][0]) == 4 and int(d["flag4"][0]) != 0
        assert _rel(lu[1:4], d["bd_lu"][1:4]) <= 1e-10
    s.close()


def test_singular_leaf_block_is_reported():
    """The reference's matrices with one equation row's blocks zeroed: the
    preconditioner leaf holding that row has a zero row, its full-pivot
    inverse meets a pivot <= 1e-10 (inv_mat, DBEM1/lin_comp.cpp:83-117), and
    the load reports TDBEM_SINGULAR_BLOCK instead of marching."""
    from tdbem.api import MultiDomainSolver, TdbemError
    g = load_golden("rod5_n2_tight")
    c = case_from_golden(g, "rod5_singular")
    rp, col, val = g["A_row_ptr"], g["A_col"], g["A_val"].copy()
    val[rp[7]:rp[8]] = 0.0
    mts = [golden_hist(g, "MTS", i) for i in range(len(g["hist_k"]))]
    mgs = [golden_hist(g, "MGS", i) for i in range(len(g["hist_k"]))]
    s = MultiDomainSolver(c)
    with pytest.raises(TdbemError) as e:
        s.load_matrices((rp, col, val), (g["KnownM_row_ptr"], g["KnownM_col"], g["KnownM_val"]), mts, mgs)
    assert e.value.status == SINGULAR_BLOCK
    s.close()
    # the context stays usable: the intact matrices march
    s = MultiDomainSolver(c)
    s.load_matrices((rp, col, g["A_val"]), (g["KnownM_row_ptr"], g["KnownM_col"], g["KnownM_val"]), mts, mgs)
    lu, lt, rep = s.march(g["known"])
    assert rep.failed_step == 0 and _rel(lu, g["bd_lu"]) <= 1e-10
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_failure_in_one_group_of_several(monkeypatch, precision):
    """Four load cases on four GMRES clusters of one launch; two cases are
    zero (converged at once), two cannot converge: restart 2 at tolerance
    1e-18, below what the FP64 residual b - A x can resolve, so neither the
    FP64 solver nor the mixed solver's eight refinement cycles reach it.  The clusters that fail set the status word while the
    others run; the march reports TDBEM_NOT_CONVERGED at step 1 and the
    next march on a fresh handle runs normally."""
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    monkeypatch.setenv("TDBEM_GMRES_GROUPS", "4")
    c = cases.config_rod5_batched(nstep=6, loads=4, error=1e-18, iterations=2)
    c.known[0] = 0.0
    c.known[2] = 0.0
    s = MultiDomainSolver(c, precision=precision, n_loads=4)
    s.assemble()
    lu, lt, rep = s.march(c.known, raise_on_failure=False)
    assert rep.gmres_groups == 4
    assert rep.failed_step == 1 and rep.gmres_flag != 0
    assert np.all(lu[:, 2:] == 0.0)
    s.close()
    monkeypatch.delenv("TDBEM_GMRES_GROUPS")
    ok = cases.config_rod5_batched(nstep=6, loads=4, error=1e-10)
    s = MultiDomainSolver(ok, precision=precision, n_loads=4)
    s.assemble()
    _, _, rep = s.march(ok.known)
    assert rep.failed_step == 0 and rep.steps_solved == 6
    s.close()
