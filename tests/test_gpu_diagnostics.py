"""Diagnostic CSV files against the ones the reference itself wrote.

tests/golden/diagnostics_rod5_10.npz holds the numeric columns of
rhs_breakdown.csv, residual_probe.csv and interface_transfer_audit.csv from
the reference run with DBEM_RHS_DIAGNOSTIC=1 on the 5-domain rod (10 steps,
GMRES tolerance 1e-13; made by tests/golden/make_golden_validation.py
--diagnostics).  The library's files must have the same headers and rows;
identifiers equal, values within the FP64 parity bar (1e-10 relative to the
column's largest magnitude).  The residual columns are rounding noise on
both sides and are held to 1e-10 of the right-hand side's scale.
"""
import dataclasses
import os

import numpy as np
import pytest

from conftest import case_from_golden, load_golden

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))

HEADERS = {
    "rhs_breakdown": "solver,step,rowNode,rowElement,localNode,domain,surfaceType,bcid,cx,cy,cz,component,"
                     "knownRhs,historyG,historyT,totalRhs,Ax,residual,solution",
    "residual_probe": "solver,step,maxAbsResidual,l2Residual,l2Rhs,relativeResidual",
    "interface_transfer_audit": "solver,step,interfaceId,domainA,domainB,normalSign,localNode,nodeA,nodeB,eleA,"
                                "eleB,component,uA,uB,uJump,tA,tB,tResidual",
}
TEXT = {"rhs_breakdown": {0, 11}, "residual_probe": {0}, "interface_transfer_audit": {0, 11}}


def _read(path, skip):
    lines = open(path).read().splitlines()
    head = lines[0].split(",")
    text = [[v for i, v in enumerate(ln.split(",")) if i in skip] for ln in lines[1:]]
    num = np.array([[float(v) for i, v in enumerate(ln.split(",")) if i not in skip] for ln in lines[1:]])
    return lines[0], [head[i] for i in range(len(head)) if i not in skip], text, num


def _solver():
    from tdbem.api import MultiDomainSolver
    g = load_golden("rod5_n2_tight")
    c = case_from_golden(g, "rod5_n2_tight")
    c = dataclasses.replace(c, nstep=10, known=c.known[:, :11])
    s = MultiDomainSolver(c)
    s.assemble()
    return c, s


def _close(mine, ref, scale, tol=1e-10):
    return np.max(np.abs(mine - ref)) <= tol * max(scale, 1e-300)


def test_diagnostic_files_match_reference(tmp_path):
    ref = np.load(os.path.join(HERE, "golden", "diagnostics_rod5_10.npz"))
    c, s = _solver()
    s.set_record(True)
    lu, lt, rep = s.march(c.known[0])
    assert rep.steps_solved == c.nstep
    s.write_validation(str(tmp_path), lu, lt, rep)
    s.write_rhs_diagnostics(str(tmp_path), rep)
    got = {}
    for name, skip in TEXT.items():
        header, cols, text, num = _read(tmp_path / (name + ".csv"), skip)
        assert header == HEADERS[name]
        assert cols == list(ref[name + "_cols"])
        assert num.shape == ref[name].shape, (name, num.shape, ref[name].shape)
        assert all(t[0] == "multidomain" for t in text)
        if len(skip) == 2:
            assert [t[1] for t in text] == ["x", "y", "z"] * (len(text) // 3)
        got[name] = dict(zip(cols, num.T))
    rb = dict(zip(ref["rhs_breakdown_cols"], ref["rhs_breakdown"].T))
    mb = got["rhs_breakdown"]
    for k in ("step", "rowNode", "rowElement", "localNode", "domain", "surfaceType", "bcid"):
        assert np.array_equal(mb[k], rb[k]), k
    for k in ("cx", "cy", "cz", "knownRhs", "historyG", "historyT", "totalRhs", "Ax", "solution"):
        assert _close(mb[k], rb[k], np.max(np.abs(rb[k]))), k
    rhs_scale = np.max(np.abs(rb["totalRhs"]))
    assert _close(mb["residual"], rb["residual"], rhs_scale)
    # the parts add up to the right-hand side the solver used
    assert _close(mb["knownRhs"] + mb["historyG"] + mb["historyT"], mb["totalRhs"], rhs_scale, 1e-13)

    rp = dict(zip(ref["residual_probe_cols"], ref["residual_probe"].T))
    mp = got["residual_probe"]
    assert np.array_equal(mp["step"], rp["step"])
    assert _close(mp["l2Rhs"], rp["l2Rhs"], np.max(rp["l2Rhs"]))
    for k in ("maxAbsResidual", "l2Residual"):
        assert _close(mp[k], rp[k], np.max(rp["l2Rhs"])), k
    assert np.max(np.abs(mp["relativeResidual"] - rp["relativeResidual"])) <= 1e-10

    ra = dict(zip(ref["interface_transfer_audit_cols"], ref["interface_transfer_audit"].T))
    ma = got["interface_transfer_audit"]
    for k in ("step", "interfaceId", "domainA", "domainB", "normalSign", "localNode", "nodeA", "nodeB", "eleA", "eleB"):
        assert np.array_equal(ma[k], ra[k]), k
    for k, scale_k in (("uA", "uA"), ("uB", "uB"), ("uJump", "uA"), ("tA", "tA"), ("tB", "tB"), ("tResidual", "tA")):
        assert _close(ma[k], ra[k], np.max(np.abs(ra[scale_k]))), k


def test_rhs_diagnostics_need_a_recorded_march(tmp_path):
    from tdbem.api import TdbemError
    c, s = _solver()
    s.set_record(False)
    _, _, rep = s.march(c.known[0])
    with pytest.raises(TdbemError):
        s.write_rhs_diagnostics(str(tmp_path), rep)
