"""Validation output (tdbem_md_write_validation) against the reference's own files.

tests/golden/validation_rod5_10.npz holds validation_state.csv and
validation_metrics.txt as the reference wrote them for the 5-domain rod
(10 steps, GMRES tolerance 1e-13).  The library's files for the same case
must have the same columns and keys; identifiers and counts equal, values
within the FP64 parity bar (1e-10 relative), GMRES inner iterations within
one per step; the two timing keys are not compared.
"""
import dataclasses
import os

import numpy as np
import pytest

from conftest import case_from_golden, load_golden

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _metrics(path):
    keys, vals = [], []
    for ln in open(path).read().splitlines():
        k, v = ln.split("=", 1)
        keys.append(k)
        vals.append(v)
    return keys, vals


def test_validation_files_match_reference(tmp_path):
    from tdbem.api import MultiDomainSolver
    ref = np.load(os.path.join(HERE, "golden", "validation_rod5_10.npz"))
    g = load_golden("rod5_n2_tight")
    c = case_from_golden(g, "rod5_n2_tight")
    c = dataclasses.replace(c, nstep=10, known=c.known[:, :11])
    s = MultiDomainSolver(c)
    s.assemble()
    lu, lt, rep = s.march(c.known[0])
    s.write_validation(str(tmp_path), lu, lt, rep)

    mine = np.loadtxt(tmp_path / "validation_state.csv", delimiter=",", skiprows=1)
    assert open(tmp_path / "validation_state.csv").readline().strip() == \
        "step,element,localNode,nodeId,domain,surfaceType,bcid,x,y,z,ux,uy,uz,tx,ty,tz"
    want = ref["state"]
    assert mine.shape == want.shape
    assert np.array_equal(mine[:, :7], want[:, :7])
    assert np.max(np.abs(mine[:, 7:10] - want[:, 7:10])) <= 1e-13
    for cols in (slice(10, 13), slice(13, 16)):
        scale = np.max(np.abs(want[:, cols]))
        assert np.max(np.abs(mine[:, cols] - want[:, cols])) <= 1e-10 * scale

    keys, vals = _metrics(tmp_path / "validation_metrics.txt")
    rkeys, rvals = list(ref["keys"]), list(ref["values"])
    assert keys == rkeys
    mv, rv = dict(zip(keys, vals)), dict(zip(rkeys, rvals))
    skip = {"MultiDomainMatrixAssemblyTime", "MultiDomainGMRESTime"}
    approx = {"MultiDomainTotalInnerIterations", "MultiDomainAverageInnerIterations"}
    steps = int(rv["MultiDomainSolvedSteps"])
    for k in keys:
        if k in skip:
            continue
        if k in approx:
            tol = steps if k == "MultiDomainTotalInnerIterations" else 1.0
            assert abs(float(mv[k]) - float(rv[k])) <= tol, k
        elif k.startswith("InterfaceStep") or k.startswith("InterfaceOverall"):
            assert abs(float(mv[k]) - float(rv[k])) <= 1e-10 * max(1.0, abs(float(rv[k]))), k
        elif k == "Dt":
            assert abs(float(mv[k]) - float(rv[k])) <= 1e-15 * float(rv[k])
        elif k.startswith("DomainMaterial"):
            a = [float(x) for x in mv[k].split()[1::2]]
            b = [float(x) for x in rv[k].split()[1::2]]
            assert np.allclose(a, b, rtol=1e-14, atol=0), k
        else:
            assert mv[k] == rv[k], (k, mv[k], rv[k])
