"""Several models marched together (tdbem_md_march_many) equal their own marches."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_uneven_models_together_equal_separate_marches():
    import torch
    from tdbem import cases
    from tdbem.api import MultiDomainSolver, march_many
    rods = cases.config_uneven_rods(count=4, nstep=30, n_min=2, n_max=4, error=1e-12)
    rods[1] = cases.config_uneven_rods(count=2, nstep=17, n_min=3, n_max=3, seed=9, error=1e-12)[1]  # other length
    dev = torch.device("cuda:0")
    solvers, known, lu, lt = [], [], [], []
    for c in rods:
        s = MultiDomainSolver(c)
        s.assemble()
        solvers.append(s)
        k = torch.from_numpy(np.ascontiguousarray(c.known[:1])).to(dev)
        known.append(k)
        lu.append(torch.zeros_like(k))
        lt.append(torch.zeros_like(k))
    stream = torch.cuda.current_stream(dev).cuda_stream
    reps = march_many(solvers, [k.data_ptr() for k in known], [x.data_ptr() for x in lu],
                      [x.data_ptr() for x in lt], stream)
    torch.cuda.synchronize()
    for i, (s, c) in enumerate(zip(solvers, rods)):
        assert reps[i].failed_step == 0 and reps[i].steps_solved == c.nstep
        u1, t1, _ = s.march(c.known[0])
        assert np.array_equal(lu[i][0].cpu().numpy(), u1), i
        assert np.array_equal(lt[i][0].cpu().numpy(), t1), i
