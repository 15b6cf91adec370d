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
    assert api.load_library().tdbem_abi_version() == 1


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
