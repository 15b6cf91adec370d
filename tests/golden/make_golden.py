"""Regenerate the golden fixtures in this directory from the reference solver.

Runs in the development container only (it needs the reference sources to
build oracle/_ref and, for one fixture, reads the reference's own shipped
rod120_100 case).  For each case it writes the reference's input files,
runs oracle/_ref/dbem_ref_dump (the unchanged reference with a recording
wrapper, see oracle/ref_dump.cpp) and stores inputs and recorded outputs as a
compressed .npz next to this script:

  inputs      points, elements, interfaces, materials, bcid, known, scalars
  geometry    the reference's per-element geometry and singular blocks
  matrices    A, KnownM, MTS_k, MGS_k (block-CCSR, (row, col) order)
  march       per-step rhs, x, gmres flag/iterations, final bd lu/lt

    python tests/golden/make_golden.py
"""
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "parallel3.0_omp_multidomin_1node_b200"))
sys.path.insert(0, HERE)

from tdbem import cases  # noqa: E402
from refdump import read_dump  # noqa: E402

# the reference checkout (TDBEM_REFERENCE overrides the default location)
REFERENCE = os.environ.get("TDBEM_REFERENCE", "/root/reference")
REF_FIXTURE = os.path.join(REFERENCE, "DBEM1_val", "rod120_100_analytic", "20260711_152215")


def run_reference(case_dir, threads=8):
    ref = os.path.join(REPO, "oracle", "_ref")
    for t in ("gaussposition", "gaussweight"):
        shutil.copy(os.path.join(ref, t), case_dir)
    dump = os.path.join(case_dir, "dump.bin")
    env = dict(os.environ, TDBEM_DUMP=dump, DBEM_VALIDATION_OUTPUT="0", OMP_NUM_THREADS=str(threads))
    with open(os.path.join(case_dir, "run.log"), "w") as log:
        subprocess.run([os.path.join(ref, "dbem_ref_dump")], cwd=case_dir, env=env, stdout=log,
                       stderr=subprocess.STDOUT, check=False)
    return read_dump(dump)


def pack(case, d, out, keep_matrices=True):
    E = case.n_elements
    n = int(d["meta"][3])
    arrays = dict(
        points=case.mesh.points, elements=case.mesh.elements, interfaces=case.mesh.interfaces,
        domain_of=case.mesh.domain_of,
        materials=np.array([[m.E, m.nu, m.rho] for m in case.materials]),
        bcid=case.bcid, known=case.known[0],
        scalars=np.array([case.beta, case.nstep, case.gap, case.iterations, float(d["error"][0]),
                          case.max_leaf]),
        ref_mats=np.stack([d[f"mat{i}"] for i in range(len(case.materials))]),
        coordcoef=d["coordcoef"], center=d["center"], radius=d["radius"], radius_pw=d["radius_pw"],
        rcen_pw=d["rcen_pw"], node=d["node"], transmat=d["transmat"], on_u1=d["on_u1"],
        on_t1=d["on_t1"], on_t2=d["on_t2"], dof_counts=d["dof_counts"],
        bd_lu=d["bd_lu"], bd_lt=d["bd_lt"], solver_return=d["solver_return"],
    )
    steps = int(d["steps_recorded"][0])
    arrays["rhs"] = np.stack([d[f"rhs{s}"] for s in range(1, steps + 1)])
    arrays["x"] = np.stack([d[f"x{s}"] for s in range(1, steps + 1)])
    arrays["flags"] = np.stack([d[f"flag{s}"] for s in range(1, steps + 1)])
    for k in ("pre.repid", "pre.outpid", "pre.leaf_begin", "pre.leaf_count", "pre.inverse"):
        arrays[k.replace(".", "_")] = d[k]
    if keep_matrices:
        for m in ("A", "KnownM"):
            arrays[m + "_row_ptr"] = d[m + ".row_ptr"]
            arrays[m + "_col"] = d[m + ".col"]
            arrays[m + "_val"] = d[m + ".val"]
        ks = sorted(int(k[3:-8]) for k in d if k.startswith("MTS") and k.endswith(".row_ptr"))
        arrays["hist_k"] = np.array(ks, dtype=np.int64)
        for m in ("MTS", "MGS"):
            arrays[m + "_row_ptr"] = np.stack([d[f"{m}{k}.row_ptr"] for k in ks]) if ks else np.zeros((0, E + 1))
            arrays[m + "_col"] = np.concatenate([d[f"{m}{k}.col"] for k in ks]) if ks else np.zeros(0)
            arrays[m + "_val"] = np.concatenate([d[f"{m}{k}.val"] for k in ks]) if ks else np.zeros((0, 9))
    assert n == case.nstep
    np.savez_compressed(out, **arrays)
    print(f"{os.path.basename(out)}: E={E} steps={steps} flags(last)={arrays['flags'][-1]} "
          f"size={os.path.getsize(out) / 1e6:.2f} MB")


def golden_cases():
    tight = 1.0e-13
    rod = cases.config_rod5(nstep=100)
    yield "rod5_n2_tight", rod, tight, True
    yield "rod5_n2_card", rod, 1.0e-5, False
    rng_mats = [cases.Material(20.0, 0.25, 20.0), cases.Material(80.0, 0.25, 20.0)]
    rng = np.random.default_rng(11)
    v = rng.normal(size=3)
    v /= np.linalg.norm(v)
    mesh = cases.build_bar(2, 2.0, 1.0, 1.0, 2, 2, 2)
    c1, _ = cases.wave_speeds(rng_mats[0])
    dt = 0.6 * cases.mean_element_size(mesh) / c1
    prof = cases.ricker(np.arange(41) * dt, 0.5 * c1)
    bar2 = cases._finish_case("bar2_mixed", mesh, rng_mats, 0.6, 40, [(1.0, v, prof)])
    yield "bar2_mixed_tight", bar2, tight, True
    # one domain without interfaces through the reference's multi-domain path
    # (DomainCount = 1; the reference then also runs its own check that the
    # one-domain builder equals its legacy assembly, DBEM1/multidomain.cpp:2932-3045)
    cube = cases.make_case("cube1", 1, 3, [cases.Material(20.0, 0.25, 20.0)], 0.6, 20,
                           [(1.0, (1.0, 0.0, 0.0), cases.heaviside(20))])
    yield "cube1_tight", cube, tight, True
    if os.path.isdir(REF_FIXTURE):
        yield "fixture_rod120", cases.read_reference_inputs(REF_FIXTURE), None, True


def main():
    subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), f"TDBEM_REFERENCE={REFERENCE}", "dump"], check=True,
                   stdout=subprocess.DEVNULL)
    only = set(sys.argv[1:])
    for name, case, err, keep in golden_cases():
        if only and name not in only:
            continue
        with tempfile.TemporaryDirectory() as tmp:
            if name == "fixture_rod120":
                for item in os.listdir(REF_FIXTURE):
                    src = os.path.join(REF_FIXTURE, item)
                    (shutil.copytree if os.path.isdir(src) else shutil.copy)(src, os.path.join(tmp, item))
            else:
                cases.write_reference_inputs(case, tmp, error=err)
            d = run_reference(tmp)
            pack(case, d, os.path.join(HERE, name + ".npz"), keep_matrices=keep)


if __name__ == "__main__":
    main()
