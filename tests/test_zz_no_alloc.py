"""No-allocation solve (tdbem_md_solve_noalloc) against the march's own GMRES.

The file name sorts last, so in a full run the entry point is exercised after
every other GPU test has used the library in the same process.  Tolerance:
the unknowns within 1e-10 relative of the solution the march recorded for
the same right-hand side (both are the FP64 GMRES at tolerance 1e-13).  The
calls after the first leave the device's free memory unchanged.
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
    bs = [torch.from_numpy(rhs[step - 1].copy()).to(dev) for step in (3, 4, 5)]
    outs = [torch.full_like(b, float("nan")) for b in bs]
    torch.cuda.synchronize()
    # the first call sets up (the scratch array's address, kernel loading);
    # the two calls after it, on the one static scratch with different
    # right-hand sides, must leave the device's free memory where it was
    s.solve_noalloc(bs[0].data_ptr(), outs[0].data_ptr(), stream=stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    for i, step in enumerate((4, 5), start=1):
        f = s.solve_noalloc(bs[i].data_ptr(), outs[i].data_ptr())  # torch's current stream by default
        assert f[0] == 0
        assert abs(f[2] - int(flags[step - 1][2])) <= 1
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0, (free0, free1)
    for i, step in enumerate((3, 4, 5)):
        assert _rel(outs[i].cpu().numpy(), x[step - 1]) <= 1e-10, step


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
