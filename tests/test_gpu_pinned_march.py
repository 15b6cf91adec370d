"""tdbem_md_march from pinned host buffers streams its copies beside the
march by chunks of steps; the results must equal the march from pageable
buffers (whole copies before and after) bit for bit, for one and for
several load cases, and when the step count is not a multiple of the
chunk count."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("loads,nstep", [(1, 30), (8, 13)])
def test_pinned_march_equals_pageable(loads, nstep):
    import torch
    from tdbem import cases
    from tdbem.api import MultiDomainSolver, Report, load_library
    c = cases.config_rod5_batched(nstep=nstep, n=2, loads=loads, error=1e-12)
    s = MultiDomainSolver(c, precision="mixed" if loads > 1 else "fp64", n_loads=loads)
    s.assemble()
    lu0, lt0, rep0 = s.march(c.known)
    kh = torch.from_numpy(np.ascontiguousarray(c.known)).pin_memory()
    lu = torch.zeros_like(kh).pin_memory()
    lt = torch.zeros_like(kh).pin_memory()
    rep = Report()
    L = load_library()
    for _ in range(2):  # twice: the copies of one call must not disturb the next
        assert L.tdbem_md_march(s.h, ctypes.c_void_p(kh.data_ptr()), ctypes.c_void_p(lu.data_ptr()),
                                ctypes.c_void_p(lt.data_ptr()), ctypes.byref(rep), None) == 0
        assert rep.steps_solved == nstep
        assert np.array_equal(lu.numpy(), lu0)
        assert np.array_equal(lt.numpy(), lt0)
