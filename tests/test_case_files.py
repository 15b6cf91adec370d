"""Reference input files read by the library's input layer (tdbem_case_read).

The case directories are written from the golden fixtures in the reference's
formats: the text datacard / .model / .bd, the DBEMBIN binary forms selected
by the card's input mode, and the batch boundary modes whose files become
load cases.  Everything read must equal the fixture's inputs exactly.
"""
import os
import struct

import numpy as np
import pytest

from conftest import case_from_golden, load_golden


def _write_case(tmp, name="rod5_n2_tight"):
    from tdbem import cases
    g = load_golden(name)
    c = case_from_golden(g, name)
    cases.write_reference_inputs(c, str(tmp), threads=4)
    return g, c


def _check_inputs(f, g, c, loads=None):
    a = f.arrays()
    assert f.title == c.name
    assert np.array_equal(a["points"], g["points"])
    assert np.array_equal(a["elements"], g["elements"])
    assert np.array_equal(a["bcid"], g["bcid"])
    assert np.array_equal(a["materials"], g["materials"])
    assert np.array_equal(a["interfaces"], g["interfaces"])
    p = f.problem
    sc = g["scalars"]
    assert (p.beta, p.n_steps, p.gap, p.restart, p.tol, p.max_leaf) == (sc[0], int(sc[1]), sc[2], int(sc[3]),
                                                                           sc[4], int(sc[5]))
    m0 = c.card_material()
    assert (p.card_E, p.card_nu, p.card_rho) == (m0.E, m0.nu, m0.rho)
    want = g["known"][None] if loads is None else loads
    assert np.array_equal(f.known, want)


def test_text_case(tmp_path):
    from tdbem.api import CaseFiles
    g, c = _write_case(tmp_path)
    f = CaseFiles(str(tmp_path))
    assert f.n_loads == 1
    _check_inputs(f, g, c)


def _dbembin(kind):
    return b"DBEMBIN\0" + struct.pack("<4I", 1, kind, 0x01020304, 0)


def test_binary_case(tmp_path):
    """Input mode 1: input/<title>.model.bin and .bd.bin (DBEM1/DBEM.cpp:89-293)."""
    from tdbem.api import CaseFiles
    g, c = _write_case(tmp_path)
    card = open(tmp_path / "BEM_DATACARD.DAT").read().split("\n")
    # the input-mode line follows premaxleafpointnum: "0" -> "1"
    i = card.index(str(c.max_leaf))
    assert card[i + 1] == "0"
    card[i + 1] = "1"
    open(tmp_path / "BEM_DATACARD.DAT", "w").write("\n".join(card))
    base = tmp_path / "input" / c.name
    os.remove(str(base) + ".model")
    os.remove(str(base) + ".bd")
    with open(str(base) + ".model.bin", "wb") as fh:
        fh.write(_dbembin(1))
        fh.write(struct.pack("<q", len(g["points"])))
        fh.write(np.ascontiguousarray(g["points"], "<f8").tobytes())
        fh.write(struct.pack("<q", len(g["elements"])))
        fh.write(np.ascontiguousarray(g["elements"], "<i8").tobytes())
        fh.write(struct.pack("<q", 0))
    with open(str(base) + ".bd.bin", "wb") as fh:
        fh.write(_dbembin(2))
        fh.write(struct.pack("<qq", len(g["elements"]), c.nstep))
        fh.write(np.ascontiguousarray(g["bcid"], "<i4").tobytes())
        fh.write(np.ascontiguousarray(g["known"], "<f8").tobytes())
    f = CaseFiles(str(tmp_path))
    _check_inputs(f, g, c)


def test_batch_boundary_files_become_load_cases(tmp_path):
    """Batch mode 1 (a list of boundary files): one load case per file."""
    from tdbem import cases
    from tdbem.api import CaseFiles
    g, c = _write_case(tmp_path)
    rng = np.random.default_rng(3)
    loads = np.stack([g["known"], g["known"] * rng.uniform(0.5, 2.0)])
    names = []
    for r in range(2):
        nm = f"load{r}.bd"
        with open(tmp_path / nm, "w") as fh:
            fh.write("\n".join(str(int(b)) for b in g["bcid"]) + "\n")
            for s in range(c.nstep + 1):
                fh.write("\n".join("\t".join(cases._fmt(x) for x in row) for row in loads[r][s]) + "\n")
        names.append(nm)
    card = open(tmp_path / "BEM_DATACARD.DAT").read().split("\n")
    i = card.index(str(c.max_leaf))
    card[i + 2] = "1\n2\n" + "\n".join(names)   # batch mode 1, two files
    open(tmp_path / "BEM_DATACARD.DAT", "w").write("\n".join(card))
    f = CaseFiles(str(tmp_path))
    assert f.n_loads == 2
    _check_inputs(f, g, c, loads=loads)


def test_bad_cards_rejected(tmp_path):
    from tdbem.api import CaseFiles, TdbemError
    with pytest.raises(TdbemError, match="BEM_DATACARD"):
        CaseFiles(str(tmp_path))
    g, c = _write_case(tmp_path)
    card = open(tmp_path / "BEM_DATACARD.DAT").read().split("\n")
    card[10] = "1"    # solvers = 1 (Gauss): not the multi-domain march
    open(tmp_path / "BEM_DATACARD.DAT", "w").write("\n".join(card))
    with pytest.raises(TdbemError, match="solvers = 2"):
        CaseFiles(str(tmp_path))


@pytest.mark.gpu
def test_march_from_case_files(tmp_path):
    """Files -> tdbem_case_read -> create / assemble / march equals the reference's bd."""
    from tdbem.api import CaseFiles, MultiDomainSolver
    g, c = _write_case(tmp_path)
    f = CaseFiles(str(tmp_path))
    s = MultiDomainSolver.from_case_files(f)
    s.assemble()
    lu, lt, rep = s.march(f.known)
    assert rep.failed_step == 0
    scale = np.max(np.abs(g["bd_lu"]))
    assert np.max(np.abs(lu[0].reshape(g["bd_lu"].shape) - g["bd_lu"])) <= 1e-10 * scale
    scale = np.max(np.abs(g["bd_lt"]))
    assert np.max(np.abs(lt[0].reshape(g["bd_lt"].shape) - g["bd_lt"])) <= 1e-10 * scale
