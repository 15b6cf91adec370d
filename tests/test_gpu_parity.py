"""CUDA path against the reference fixtures and the C oracle (B200).

Tolerances: geometry 1e-13, singular blocks and assembled matrices 1e-12
relative to the largest entry, right-hand sides 1e-12, boundary values 1e-10
(both sides run GMRES at tolerance 1e-13, so iterates agree far below that).
"""
import numpy as np
import pytest

from conftest import GOLDEN_NAMES, case_from_golden, golden_hist, load_golden

pytestmark = pytest.mark.gpu


def _rel(a, b):
    b = np.asarray(b)
    a = np.asarray(a).reshape(b.shape)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)) if b.size else 0.0


def _golden_mats(g):
    A = (g["A_row_ptr"], g["A_col"], g["A_val"])
    K = (g["KnownM_row_ptr"], g["KnownM_col"], g["KnownM_val"])
    mts = [golden_hist(g, "MTS", i) for i in range(len(g["hist_k"]))]
    mgs = [golden_hist(g, "MGS", i) for i in range(len(g["hist_k"]))]
    return A, K, mts, mgs


@pytest.fixture(scope="module", params=GOLDEN_NAMES)
def golden(request):
    return request.param, load_golden(request.param)


def test_geometry_and_singular_blocks(golden):
    from tdbem.api import MultiDomainSolver
    name, g = golden
    s = MultiDomainSolver(case_from_golden(g, name))
    geo = s.geometry()
    for k in ("coordcoef", "center", "radius", "radius_pw", "transmat"):
        assert _rel(geo[k].reshape(g[k].shape), g[k]) <= 1e-13, k
    # on_t2 cancels to rounding noise on flat elements: compare all three
    # singular blocks on the scale of the largest (the 0.5 jump term of on_t1)
    scale = max(np.max(np.abs(g["on_t1"])), np.max(np.abs(g["on_u1"])))
    for k in ("on_u1", "on_t1", "on_t2"):
        assert np.max(np.abs(geo[k] - g[k])) <= 1e-12 * scale, k
    rep, lb, lc = s.precond_layout()
    assert np.array_equal(rep, g["pre_repid"]) and np.array_equal(lc, g["pre_leaf_count"])


def test_march_on_reference_matrices(golden):
    """History RHS + GMRES + write-back fed with the reference's own matrices."""
    from tdbem.api import MultiDomainSolver
    name, g = golden
    s = MultiDomainSolver(case_from_golden(g, name))
    s.load_matrices(*_golden_mats(g))
    s.set_record(True)
    lu, lt, rep = s.march(g["known"])
    rhs, x, flags = s.step_record()
    assert rep.steps_solved == len(g["flags"])
    assert _rel(rhs, g["rhs"]) <= 1e-12
    assert _rel(x, g["x"]) <= 1e-10
    assert _rel(lu, g["bd_lu"]) <= 1e-10
    assert _rel(lt, g["bd_lt"]) <= 1e-10
    assert np.max(np.abs(flags[:, 2] - g["flags"][:, 2])) <= 1


def test_assembled_matrices(golden):
    from tdbem.api import MultiDomainSolver
    name, g = golden
    s = MultiDomainSolver(case_from_golden(g, name))
    s.assemble()
    for m in ("A", "KnownM"):
        rp, col, val = s.export_matrix(m)
        assert np.array_equal(rp, g[m + "_row_ptr"]) and np.array_equal(col, g[m + "_col"]), m
        assert _rel(val, g[m + "_val"]) <= 1e-12, m
    assert s.info()["n_history"] == g["dof_counts"][2]
    for i, k in enumerate(g["hist_k"]):
        for m in ("MTS", "MGS"):
            rp, col, val = golden_hist(g, m, i)
            rp2, col2, val2 = s.export_matrix(m, int(k))
            assert np.array_equal(rp2, rp) and np.array_equal(col2, col), (m, k)
            if len(col):
                assert _rel(val2, val) <= 1e-12, (m, k)


def test_full_path(golden):
    from tdbem.api import MultiDomainSolver
    name, g = golden
    s = MultiDomainSolver(case_from_golden(g, name))
    s.assemble()
    lu, lt, rep = s.march(g["known"])
    assert rep.failed_step == 0
    assert _rel(lu, g["bd_lu"]) <= 1e-10
    assert _rel(lt, g["bd_lt"]) <= 1e-10
    assert rep.max_interface_jump <= 1e-10 * max(np.max(np.abs(g["bd_lu"])), 1.0)


def test_card_tolerance_matches_reference():
    from tdbem.api import MultiDomainSolver
    g = load_golden("rod5_n2_card")
    c = case_from_golden(g)
    s = MultiDomainSolver(c)
    s.assemble()
    lu, lt, rep = s.march(g["known"])
    # at the card's 1e-5 GMRES tolerance the iterates differ by the solver tolerance
    assert _rel(lu, g["bd_lu"]) <= 1e-4
    assert rep.failed_step == 0


def test_against_oracle_heterogeneous_rod():
    """Seeded 5-domain rod, 3x3 per face, heterogeneous materials: CUDA vs C oracle."""
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    from oracle_lib import Oracle
    rng = np.random.default_rng(21)
    mats = [cases.Material(rng.uniform(15, 30), 0.25, rng.uniform(15, 25)) for _ in range(5)]
    c = cases.make_case("rod5_n3", 5, 3, mats, 0.6, 30, [(1.0, (0.3, 0.9, 0.3), cases.heaviside(30))],
                        error=1e-13)
    o = Oracle(c)
    ref = o.march(c.known[0])
    s = MultiDomainSolver(c)
    s.assemble()
    lu, lt, rep = s.march(c.known[0])
    assert ref["solved"] == 30 and rep.failed_step == 0
    assert _rel(lu, ref["bd_lu"]) <= 1e-10
    assert _rel(lt, ref["bd_lt"]) <= 1e-10


def test_single_domain_model_against_oracle():
    """One domain, no interfaces (the model the reference's legacy
    single-domain path solves): CUDA vs the C oracle of the same assembly."""
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    from oracle_lib import Oracle
    c = cases.make_case("cube_1dom", 1, 3, [cases.Material(20.0, 0.25, 20.0)], 0.6, 20,
                        [(1.0, (1.0, 0.0, 0.0), cases.heaviside(20))], error=1e-13)
    ref = Oracle(c).march(c.known[0])
    s = MultiDomainSolver(c)
    s.assemble()
    lu, lt, rep = s.march(c.known[0])
    assert ref["solved"] == 20 and rep.failed_step == 0
    assert _rel(lu, ref["bd_lu"]) <= 1e-10
    assert _rel(lt, ref["bd_lt"]) <= 1e-10


def test_mixed_precision_close_to_fp64():
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    c = cases.config_rod5(nstep=60, error=1e-8)
    s64 = MultiDomainSolver(c, precision="fp64")
    s64.assemble()
    u64, t64, _ = s64.march(c.known[0])
    s32 = MultiDomainSolver(c, precision="mixed")
    s32.assemble()
    u32, t32, rep = s32.march(c.known[0])
    assert rep.failed_step == 0
    assert _rel(u32, u64) <= 1e-6


def test_gmres_failure_reported():
    """A restart too small to converge: the march stops at step 1 like the reference."""
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    c = cases.config_rod5(nstep=5, error=1e-15, iterations=2)
    s = MultiDomainSolver(c)
    s.assemble()
    lu, lt, rep = s.march(c.known[0], raise_on_failure=False)
    assert rep.failed_step == 1 and rep.gmres_flag != 0
    assert np.all(lu[2:] == 0.0)


def test_batched_loads_match_single_runs():
    """R = 4 load cases marched together equal four single-case marches."""
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    c = cases.config_rod5_batched(nstep=40, loads=4, error=1e-13)
    sb = MultiDomainSolver(c, n_loads=4)
    sb.assemble()
    lu, lt, rep = sb.march(c.known)
    assert rep.failed_step == 0 and lu.shape == c.known.shape
    s1 = MultiDomainSolver(c)
    s1.assemble()
    for r in range(4):
        u1, t1, rep1 = s1.march(c.known[r])
        assert _rel(lu[r], u1) <= 1e-10, r
        assert _rel(lt[r], t1) <= 1e-10, r


def test_batched_32_fp64_matches_single_runs():
    """32 load cases take the source-major history pass; sampled cases equal
    single-case marches (which take the row pass)."""
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    c = cases.config_rod5_batched(nstep=40, loads=32, error=1e-13)
    sb = MultiDomainSolver(c, n_loads=32)
    sb.assemble()
    lu, lt, rep = sb.march(c.known)
    assert rep.failed_step == 0
    s1 = MultiDomainSolver(c)
    s1.assemble()
    for r in (0, 13, 31):
        u1, t1, _ = s1.march(c.known[r])
        assert _rel(lu[r], u1) <= 1e-10, r
        assert _rel(lt[r], t1) <= 1e-10, r


def test_batched_mixed_32_loads_close_to_fp64():
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    c = cases.config_rod5_batched(nstep=60, loads=32, error=1e-8)
    s64 = MultiDomainSolver(c, n_loads=32)
    s64.assemble()
    u64, _, _ = s64.march(c.known)
    s32 = MultiDomainSolver(c, precision="mixed", n_loads=32)
    s32.assemble()
    u32, _, rep = s32.march(c.known)
    assert rep.failed_step == 0
    for r in range(32):
        assert _rel(u32[r], u64[r]) <= 1e-6, r


def test_batched_case_against_oracle():
    """One case of an R = 8 batch against the C oracle."""
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    from oracle_lib import Oracle
    c = cases.config_rod5_batched(nstep=30, loads=8, error=1e-13, seed=9)
    s = MultiDomainSolver(c, n_loads=8)
    s.assemble()
    lu, lt, rep = s.march(c.known)
    ref = Oracle(c).march(c.known[5])
    assert _rel(lu[5], ref["bd_lu"]) <= 1e-10
    assert _rel(lt[5], ref["bd_lt"]) <= 1e-10


def test_history_length_on_domain_contrast_bar():
    """A short stiff and a long soft domain (history lengths 6 and 30): the
    library stops its history assembly at the skip-rule bound and keeps the
    same steps and blocks as the oracle assembled to NStep without a stop."""
    import numpy as np
    from test_history_bound import _contrast_case
    from tdbem.api import MultiDomainSolver
    from oracle_lib import Oracle
    c = _contrast_case()
    o = Oracle(c)
    o.assemble(kmax=c.nstep)
    last = max(k for k in range(1, c.nstep + 1)
               if len(o.matrix("MTS", k)[1]) or len(o.matrix("MGS", k)[1]))
    s = MultiDomainSolver(c)
    s.assemble()
    _, _, rep = s.march(c.known[0])
    assert rep.history_steps == last
    for k in range(1, last + 1):
        for m in ("MTS", "MGS"):
            rp, col, val = o.matrix(m, k)
            rp2, col2, val2 = s.export_matrix(m, k)
            assert np.array_equal(rp2, rp) and np.array_equal(col2, col), (m, k)
            if len(col):
                assert _rel(val2, val) <= 1e-12, (m, k)
