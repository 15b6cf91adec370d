import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "parallel3.0_omp_multidomin_1node_b200")
for p in (PKG, os.path.join(REPO, "tests"), os.path.join(REPO, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def case_from_golden(g, name="golden"):
    from tdbem import cases
    sc = g["scalars"]
    mesh = cases.BarMesh(points=g["points"], elements=g["elements"], domain_of=g["domain_of"],
                         face_of=np.full(len(g["elements"]), -1, np.int64), interfaces=g["interfaces"],
                         domains=len(g["materials"]))
    mats = [cases.Material(*m) for m in g["materials"]]
    return cases.Case(name=name, mesh=mesh, materials=mats, bcid=g["bcid"], known=g["known"][None],
                      beta=float(sc[0]), nstep=int(sc[1]), gap=float(sc[2]), iterations=int(sc[3]),
                      error=float(sc[4]), max_leaf=int(sc[5]))


def golden_hist(g, which, i):
    """(row_ptr, col, val) of history matrix number i (k = g['hist_k'][i])."""
    rp = g[which + "_row_ptr"]
    start = int(sum(int(rp[j][-1]) for j in range(i)))
    n = int(rp[i][-1])
    return rp[i], g[which + "_col"][start:start + n], g[which + "_val"][start:start + n]


GOLDEN_NAMES = ["rod5_n2_tight", "bar2_mixed_tight", "fixture_rod120", "cube1_tight"]
