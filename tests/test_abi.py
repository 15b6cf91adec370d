"""C ABI checks that need no GPU: the library loads, exports every entry
point declared in include/tdbem.h, and rejects invalid models before any
device work."""
import os
import re

import numpy as np
import pytest

from conftest import REPO


def test_header_symbols_exported():
    from tdbem import api
    L = api.load_library()
    hdr = open(os.path.join(REPO, "include", "tdbem.h")).read()
    names = set(re.findall(r"\b(tdbem_[a-z_]+)\s*\(", hdr))
    assert names, "no entry points parsed"
    for n in sorted(names):
        assert hasattr(L, n), n
    assert set(api.SIGNATURES) == names


def test_abi_version():
    from tdbem import api
    assert api.load_library().tdbem_abi_version() == 3


def test_invalid_bcid_rejected_before_device_work():
    from tdbem import api, cases
    c = cases.config_rod5(nstep=2)
    c.bcid = c.bcid.copy()
    c.bcid[7] = 153
    with pytest.raises(api.TdbemError, match="BCID"):
        api.MultiDomainSolver(c)


def test_bad_interface_rejected():
    from tdbem import api, cases
    c = cases.config_rod5(nstep=2)
    itf = c.mesh.interfaces.copy()
    itf[3, 1] = itf[3, 3]      # eleA in the wrong domain
    c.mesh.interfaces = itf
    with pytest.raises(api.TdbemError, match="interface"):
        api.MultiDomainSolver(c)


def test_status_strings():
    from tdbem import api
    L = api.load_library()
    for code in range(9):
        assert L.tdbem_status_string(code)


@pytest.mark.parametrize("field,value,match", [
    ("n_loads", 3, "n_loads"),
    ("tol", 0.0, "tol"),
    ("gap", 1.5, "gap"),
])
def test_invalid_parameters_rejected(field, value, match):
    import dataclasses
    from tdbem import api, cases
    c = cases.config_rod5(nstep=2)
    kw = {}
    if field == "n_loads":
        kw["n_loads"] = value
    elif field == "tol":
        kw["tol"] = value
    else:
        c = dataclasses.replace(c, gap=value)
    with pytest.raises(api.TdbemError, match=match):
        api.MultiDomainSolver(c, **kw)


def test_point_out_of_range_rejected():
    from tdbem import api, cases
    c = cases.config_rod5(nstep=2)
    el = c.mesh.elements.copy()
    el[5, 2] = len(c.mesh.points) + 7
    c.mesh.elements = el
    with pytest.raises(api.TdbemError, match="point out of range"):
        api.MultiDomainSolver(c)


def test_invalid_materials_rejected():
    from tdbem import api, cases
    c = cases.config_rod5(nstep=2)
    c.materials = list(c.materials)
    c.card = c.materials[0]
    c.materials[2] = cases.Material(-1.0, 0.25, 20.0)
    with pytest.raises(api.TdbemError, match="material"):
        api.MultiDomainSolver(c)
    c.materials[2] = c.materials[0]
    c.card = cases.Material(0.0, 0.25, 20.0)
    with pytest.raises(api.TdbemError, match="wave speed"):
        api.MultiDomainSolver(c)


def test_null_handles_rejected():
    import ctypes
    from tdbem import api
    L = api.load_library()
    buf = (ctypes.c_double * 8)()
    rep = api.Report()
    assert L.tdbem_md_march_forward(None, buf, buf, buf, ctypes.byref(rep), None) == 1
    assert L.tdbem_md_march_backward(None, None, None, buf, None, ctypes.byref(rep), None) == 1
    assert L.tdbem_md_march_vjp(None, None, None, buf, ctypes.byref(rep), None) == 1
    assert L.tdbem_md_autotune(None, buf, 4, None, None) == 1
    assert L.tdbem_md_write_rhs_diagnostics(None, b".", ctypes.byref(rep)) == 1
    assert L.tdbem_md_march_many(None, 0, None, None, None, None, None) == 1
    assert L.tdbem_last_error()
