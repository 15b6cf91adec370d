"""The reference's diagnostic files (tests/golden/diagnostics_rod5_10.npz,
from tests/golden/make_golden_validation.py --diagnostics) on the CPU:

- they agree exactly with the reference's validation file of the same case
  (tests/golden/validation_rod5_10.npz): interface displacements and
  tractions per step, element and component;
- they are consistent in themselves: the KnownM, history G and history T
  parts add up to the right-hand side, and the residual probe's norms are
  those of the breakdown's rows;
- the C oracle reproduces the reference's per-step right-hand side and
  solution column (x in unknown order read at the row's index) to 1e-10 of
  their scale.
"""
import dataclasses
import os

import numpy as np

from conftest import case_from_golden, load_golden

HERE = os.path.dirname(os.path.abspath(__file__))


def _load():
    v = np.load(os.path.join(HERE, "golden", "validation_rod5_10.npz"))
    d = np.load(os.path.join(HERE, "golden", "diagnostics_rod5_10.npz"))
    st = v["state"]
    E = int(st[:, 1].max()) + 1
    state = st.reshape(-1, E, st.shape[1])  # [step][element][column]
    cols = {name: {c: i for i, c in enumerate(d[name + "_cols"])} for name in
            ("rhs_breakdown", "residual_probe", "interface_transfer_audit")}
    return state, d, cols


def test_audit_equals_validation_state():
    state, d, cols = _load()
    a, ci = d["interface_transfer_audit"], cols["interface_transfer_audit"]
    for k, row in enumerate(a):
        step, ea, eb, comp = int(row[ci["step"]]), int(row[ci["eleA"]]), int(row[ci["eleB"]]), k % 3
        assert row[ci["uA"]] == state[step, ea, 10 + comp]
        assert row[ci["uB"]] == state[step, eb, 10 + comp]
        assert row[ci["tA"]] == state[step, ea, 13 + comp]
        assert row[ci["tB"]] == state[step, eb, 13 + comp]
        assert row[ci["uJump"]] == row[ci["uA"]] - row[ci["uB"]]


def test_breakdown_and_probe_are_consistent():
    _, d, cols = _load()
    rb, rc = d["rhs_breakdown"], cols["rhs_breakdown"]
    scale = np.max(np.abs(rb[:, rc["totalRhs"]]))
    parts = rb[:, rc["knownRhs"]] + rb[:, rc["historyG"]] + rb[:, rc["historyT"]]
    assert np.max(np.abs(parts - rb[:, rc["totalRhs"]])) <= 1e-14 * scale
    rp, pc = d["residual_probe"], cols["residual_probe"]
    for row in rp:
        m = rb[:, rc["step"]] == row[pc["step"]]
        res = rb[m, rc["residual"]]
        assert abs(np.sqrt(np.sum(rb[m, rc["totalRhs"]] ** 2)) - row[pc["l2Rhs"]]) <= 1e-12 * row[pc["l2Rhs"]]
        assert abs(np.max(np.abs(res)) - row[pc["maxAbsResidual"]]) <= 1e-12 * max(row[pc["maxAbsResidual"]], 1e-300)
        assert abs(np.sqrt(np.sum(res ** 2)) - row[pc["l2Residual"]]) <= 1e-12 * max(row[pc["l2Residual"]], 1e-300)


def test_oracle_reproduces_reference_rhs_and_solution():
    from oracle_lib import Oracle
    _, d, cols = _load()
    g = load_golden("rod5_n2_tight")
    c = case_from_golden(g, "rod5_n2_tight")
    c = dataclasses.replace(c, nstep=10, known=c.known[:, :11])
    out = Oracle(c).march(c.known[0])
    rb, rc = d["rhs_breakdown"], cols["rhs_breakdown"]
    E = c.n_elements
    ref_rhs = rb[:, rc["totalRhs"]].reshape(c.nstep, E * 3)
    ref_x = rb[:, rc["solution"]].reshape(c.nstep, E * 3)
    assert np.max(np.abs(out["rhs"] - ref_rhs)) <= 1e-10 * np.max(np.abs(ref_rhs))
    assert np.max(np.abs(out["x"] - ref_x)) <= 1e-10 * np.max(np.abs(ref_x))
