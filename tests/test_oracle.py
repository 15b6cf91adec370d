"""The C restatement oracle against fixtures recorded from the reference
solver itself (tests/golden/make_golden.py): every stage must agree to
rounding, and in practice agrees bit for bit."""
import numpy as np
import pytest

from conftest import GOLDEN_NAMES, case_from_golden, golden_hist, load_golden
from oracle_lib import Oracle

GEOM = ["coordcoef", "center", "radius", "radius_pw", "rcen_pw", "transmat", "on_u1", "on_t1", "on_t2"]


@pytest.fixture(scope="module", params=GOLDEN_NAMES)
def pinned(request):
    g = load_golden(request.param)
    o = Oracle(case_from_golden(g, request.param))
    o.assemble()
    return g, o


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)) if b.size else 0.0


def test_geometry_and_singular_blocks(pinned):
    g, o = pinned
    geo = o.geometry()
    for k in GEOM:
        assert _rel(geo[k].reshape(g[k].shape), g[k]) <= 1e-14, k


def test_dof_counts(pinned):
    g, o = pinned
    assert list(o.dof_counts()) == list(g["dof_counts"][:3])


def test_step0_matrices(pinned):
    g, o = pinned
    for m in ("A", "KnownM"):
        rp, col, val = o.matrix(m)
        assert np.array_equal(rp, g[m + "_row_ptr"]) and np.array_equal(col, g[m + "_col"]), m
        assert _rel(val, g[m + "_val"]) <= 1e-13, m


def test_history_matrices(pinned):
    g, o = pinned
    for i, k in enumerate(g["hist_k"]):
        for m in ("MTS", "MGS"):
            rp, col, val = golden_hist(g, m, i)
            rp2, col2, val2 = o.matrix(m, int(k))
            assert np.array_equal(rp2, rp) and np.array_equal(col2, col), (m, k)
            if len(col):
                assert _rel(val2, val) <= 1e-13, (m, k)


def test_preconditioner_layout(pinned):
    g, o = pinned
    rep, lb, lc = o.precond_layout()
    assert np.array_equal(rep, g["pre_repid"])
    assert np.array_equal(lb, g["pre_leaf_begin"]) and np.array_equal(lc, g["pre_leaf_count"])


def test_march(pinned):
    g, o = pinned
    r = o.march(g["known"])
    n = r["solved"]
    assert n == len(g["flags"])
    assert np.array_equal(r["flags"], g["flags"])
    assert _rel(r["rhs"], g["rhs"]) <= 1e-12
    assert _rel(r["x"], g["x"]) <= 1e-10
    assert _rel(r["bd_lu"], g["bd_lu"]) <= 1e-10
    assert _rel(r["bd_lt"], g["bd_lt"]) <= 1e-10


def test_card_tolerance_march():
    """The shipped card tolerance (1e-5): same iteration counts as the reference."""
    g = load_golden("rod5_n2_card")
    o = Oracle(case_from_golden(g))
    r = o.march(g["known"])
    assert np.array_equal(r["flags"], g["flags"])
    assert _rel(r["bd_lu"], g["bd_lu"]) <= 1e-10


def test_invalid_bcid_rejected():
    g = load_golden("rod5_n2_tight")
    c = case_from_golden(g)
    c.bcid = c.bcid.copy()
    c.bcid[5] = 126
    with pytest.raises(ValueError, match="BCID"):
        Oracle(c)


def test_nonconforming_interface_rejected():
    g = load_golden("rod5_n2_tight")
    c = case_from_golden(g)
    itf = c.mesh.interfaces.copy()
    itf[0, 3] = itf[1, 3]          # two pairs share one B element
    c.mesh.interfaces = itf
    with pytest.raises(ValueError, match="interface"):
        Oracle(c)
