"""No-allocation solve (tdbem_md_solve_noalloc) against the march's own GMRES.

The file name sorts last, so in a full run the entry point is exercised after
every other GPU test has used the library in the same process.  Tolerance:
the unknowns within 1e-10 relative of the solution the march recorded for
the same right-hand side (both are the FP64 GMRES at tolerance 1e-13).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    b = np.asarray(b)
    a = np.asarray(a).reshape(b.shape)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_noalloc_solve_matches_march():
    import torch
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    c = cases.config_rod5(nstep=6, error=1e-13)
    s = MultiDomainSolver(c)
    s.assemble()
    s.set_record(True)
    _, _, rep = s.march(c.known[0])
    assert rep.failed_step == 0
    rhs, x, flags = s.step_record()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    # two calls in a row on the one static scratch, different right-hand sides
    for step in (3, 4):
        b = torch.from_numpy(rhs[step - 1].copy()).to(dev)
        out = torch.full_like(b, float("nan"))
        f = s.solve_noalloc(b.data_ptr(), out.data_ptr(), stream=stream)
        assert f[0] == 0
        assert abs(f[2] - int(flags[step - 1][2])) <= 1
        assert _rel(out.cpu().numpy(), x[step - 1]) <= 1e-10, step


def test_noalloc_solve_rejects_oversize():
    """1080 elements at restart 480 need more than the 32 MiB static scratch."""
    import torch
    from tdbem import cases
    from tdbem.api import MultiDomainSolver, TdbemError
    c = cases.config_rod5(nstep=3, n=6, error=1e-13, iterations=480)
    s = MultiDomainSolver(c)
    s.assemble()
    b = torch.zeros(3 * c.mesh.elements.shape[0], dtype=torch.float64, device="cuda:0")
    out = torch.zeros_like(b)
    with pytest.raises(TdbemError, match="static scratch"):
        s.solve_noalloc(b.data_ptr(), out.data_ptr())
