"""The reference's own driver with its solver call served by the B200 library.

oracle/_ref/dbem_ref_b200 is the unchanged reference program (datacard,
model and bd readers, element set-up, singular integrals) linked with the
legacy-signature shim (shim/tdbem_legacy_shim.cpp): its call to
DynaGMRESSolverMultiDomainCCSR goes to tdbem_md_create / assemble / march.
The bd it ends with must equal the reference's own (golden fixtures) to
1e-10 relative, the FP64 parity bar of the direct ABI path.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import case_from_golden, load_golden

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(REPO, "oracle", "_ref")
EXE = os.path.join(REF, "dbem_ref_b200")


def _read_bd(path):
    with open(path, "rb") as f:
        n, nodes = (int(v) for v in np.frombuffer(f.read(16), np.int64))
        rc = int(np.frombuffer(f.read(4), np.int32)[0])
        data = np.frombuffer(f.read(), np.float64).reshape(n + 1, 2, 3 * nodes)
    return rc, data[:, 0], data[:, 1]


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", ["rod5_n2_tight", "bar2_mixed_tight"])
def test_reference_driver_through_shim(name, tmp_path):
    if not os.path.exists(EXE):
        pytest.skip("reference driver with the shim is not built (make -C oracle b200)")
    from tdbem import cases
    g = load_golden(name)
    case = case_from_golden(g, name)
    cases.write_reference_inputs(case, str(tmp_path), threads=4)
    for t in ("gaussposition", "gaussweight"):
        shutil.copy(os.path.join(REF, t), tmp_path)
    out = tmp_path / "bd.bin"
    env = dict(os.environ, TDBEM_BD_OUT=str(out), DBEM_VALIDATION_OUTPUT="0", OMP_NUM_THREADS="4")
    r = subprocess.run([EXE], cwd=tmp_path, env=env, capture_output=True, text=True, timeout=600)
    assert out.exists(), r.stdout[-2000:] + r.stderr[-2000:]
    rc, lu, lt = _read_bd(out)
    assert rc == 1 == int(g["solver_return"][0])
    assert _rel(lu, g["bd_lu"].reshape(lu.shape)) <= 1e-10
    assert _rel(lt, g["bd_lt"].reshape(lt.shape)) <= 1e-10
