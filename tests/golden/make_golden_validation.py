"""Golden validation outputs of the reference solver (development container only).

Runs the unchanged reference (oracle/_ref/dbem_ref, built by `make -C oracle
ref`) with DBEM_VALIDATION_OUTPUT=1 and stores what it writes,
validation_state.csv as a numeric table and validation_metrics.txt as keys
and values, next to this script:

  validation_rod5_10.npz   the 5-domain rod of rod5_n2_tight (its inputs,
                           first 10 steps): the multi-domain path
  diagnostics_rod5_10.npz  the same run with DBEM_RHS_DIAGNOSTIC=1: the
                           numeric columns of rhs_breakdown.csv,
                           residual_probe.csv and interface_transfer_audit.csv

    python tests/golden/make_golden_validation.py [--diagnostics]
"""
import dataclasses
import glob
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "parallel3.0_omp_multidomin_1node_b200"))
sys.path.insert(0, os.path.dirname(HERE))

from tdbem import cases  # noqa: E402


def run(case):
    d = tempfile.mkdtemp(prefix="tdbem_val_")
    try:
        cases.write_reference_inputs(case, d, threads=4)
        for t in ("gaussposition", "gaussweight"):
            shutil.copy(os.path.join(REPO, "oracle", "_ref", t), d)
        env = dict(os.environ, DBEM_VALIDATION_OUTPUT="1", OMP_NUM_THREADS="4")
        # the reference driver exits with status 1 after a completed run
        subprocess.run([os.path.join(REPO, "oracle", "_ref", "dbem_ref")], cwd=d, env=env,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        state = [p for p in glob.glob(os.path.join(d, "*validation_state.csv"))]
        metrics = [p for p in glob.glob(os.path.join(d, "*validation_metrics.txt"))]
        assert len(state) == 1 and len(metrics) == 1, os.listdir(d)
        table = np.loadtxt(state[0], delimiter=",", skiprows=1)
        keys, vals = [], []
        for ln in open(metrics[0]).read().splitlines():
            k, v = ln.split("=", 1)
            keys.append(k)
            vals.append(v)
        return table, np.array(keys), np.array(vals)
    finally:
        shutil.rmtree(d, ignore_errors=True)


def _numeric_csv(path, skip):
    """Rows of a CSV with the text columns (indices in skip) left out."""
    lines = open(path).read().splitlines()
    head = lines[0].split(",")
    keep = [i for i in range(len(head)) if i not in skip]
    rows = [[float(v) for i, v in enumerate(ln.split(",")) if i not in skip] for ln in lines[1:]]
    return np.array([head[i] for i in keep]), np.array(rows)


def run_diagnostics(case):
    d = tempfile.mkdtemp(prefix="tdbem_diag_")
    try:
        cases.write_reference_inputs(case, d, threads=4)
        for t in ("gaussposition", "gaussweight"):
            shutil.copy(os.path.join(REPO, "oracle", "_ref", t), d)
        env = dict(os.environ, DBEM_VALIDATION_OUTPUT="1", DBEM_RHS_DIAGNOSTIC="1", OMP_NUM_THREADS="4")
        subprocess.run([os.path.join(REPO, "oracle", "_ref", "dbem_ref")], cwd=d, env=env,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        out = {}
        # text columns: solver (0) and component (11) of rhs_breakdown and the
        # audit; solver of residual_probe
        for name, skip in (("rhs_breakdown", {0, 11}), ("residual_probe", {0}),
                           ("interface_transfer_audit", {0, 11})):
            found = glob.glob(os.path.join(d, "*" + name + ".csv"))
            assert len(found) == 1, os.listdir(d)
            cols, rows = _numeric_csv(found[0], skip)
            out[name + "_cols"] = cols
            out[name] = rows
        return out
    finally:
        shutil.rmtree(d, ignore_errors=True)


def main():
    from conftest import case_from_golden, load_golden
    g = load_golden("rod5_n2_tight")
    c = case_from_golden(g, "rod5_n2_tight")
    c = dataclasses.replace(c, nstep=10, known=c.known[:, :11])
    if "--diagnostics" in sys.argv:
        np.savez_compressed(os.path.join(HERE, "diagnostics_rod5_10.npz"), **run_diagnostics(c))
        return
    table, keys, vals = run(c)
    np.savez_compressed(os.path.join(HERE, "validation_rod5_10.npz"), state=table, keys=keys, values=vals,
                        known=c.known[0], scalars=np.array([c.beta, c.nstep, c.gap, c.iterations, c.error,
                                                            c.max_leaf]))


if __name__ == "__main__":
    main()
