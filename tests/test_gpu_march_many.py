"""Several models marched together (tdbem_md_march_many) equal their own marches.

By default each model's steps go to its own streams and run the
single-march kernels: equal bit for bit.  With TDBEM_MARCH_MANY=grouped,
models of one device, load-case count and precision are marched grouped: each
time step is one launch of every model's head right-hand side, one GMRES
launch with one cluster per model and one bulk right-hand-side launch beside
it.  The models then run with a common cluster size, so results equal the
models' own marches to rounding: 1e-10 of the scale in FP64 (GMRES
tolerance 1e-12), 1e-7 in mixed precision.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rods(loads):
    from tdbem import cases
    rods = cases.config_uneven_rods(count=4, nstep=30, n_min=2, n_max=4, error=1e-12)
    rods[1] = cases.config_uneven_rods(count=2, nstep=17, n_min=3, n_max=3, seed=9, error=1e-12)[1]  # other length
    if loads > 1:
        rng = np.random.default_rng(11)
        for c in rods:
            c.known = np.concatenate([c.known * rng.uniform(0.5, 2.0) for _ in range(loads)])
    return rods


def _march_together(loads, precision):
    import torch
    from tdbem.api import MultiDomainSolver, march_many
    rods = _rods(loads)
    dev = torch.device("cuda:0")
    solvers, known, lu, lt = [], [], [], []
    for c in rods:
        s = MultiDomainSolver(c, precision=precision, n_loads=loads)
        s.assemble()
        solvers.append(s)
        k = torch.from_numpy(np.ascontiguousarray(c.known)).to(dev)
        known.append(k)
        lu.append(torch.zeros_like(k))
        lt.append(torch.zeros_like(k))
    stream = torch.cuda.current_stream(dev).cuda_stream
    reps = march_many(solvers, [k.data_ptr() for k in known], [x.data_ptr() for x in lu],
                      [x.data_ptr() for x in lt], stream)
    torch.cuda.synchronize()
    return rods, solvers, reps, lu, lt


@pytest.mark.parametrize("loads,precision,tol", [(1, "fp64", 1e-10), (4, "mixed", 1e-7)])
def test_grouped_models_equal_separate_marches(loads, precision, tol, monkeypatch):
    monkeypatch.setenv("TDBEM_MARCH_MANY", "grouped")
    rods, solvers, reps, lu, lt = _march_together(loads, precision)
    for i, (s, c) in enumerate(zip(solvers, rods)):
        assert reps[i].failed_step == 0 and reps[i].steps_solved == c.nstep
        u1, t1, _ = s.march(c.known)
        assert np.max(np.abs(lu[i].cpu().numpy() - u1)) <= tol * np.max(np.abs(u1)), i
        assert np.max(np.abs(lt[i].cpu().numpy() - t1)) <= tol * np.max(np.abs(t1)), i


def test_streams_path_equals_separate_marches_bit_for_bit(monkeypatch):
    monkeypatch.delenv("TDBEM_MARCH_MANY", raising=False)
    rods, solvers, reps, lu, lt = _march_together(1, "fp64")
    for i, (s, c) in enumerate(zip(solvers, rods)):
        assert reps[i].failed_step == 0 and reps[i].steps_solved == c.nstep
        u1, t1, _ = s.march(c.known[0])
        assert np.array_equal(lu[i][0].cpu().numpy(), u1), i
        assert np.array_equal(lt[i][0].cpu().numpy(), t1), i
