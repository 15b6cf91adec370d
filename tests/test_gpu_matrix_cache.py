"""Matrix cache file (tdbem_md_save_matrices / tdbem_md_load_matrix_cache).

A handle loaded from the cache must march exactly like the handle that
assembled the matrices; a cache is refused by a different model or NStep.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_cache_round_trip_and_refusals(tmp_path):
    import dataclasses
    from tdbem import cases
    from tdbem.api import MultiDomainSolver, TdbemError
    c = cases.config_rod5(nstep=40, error=1e-13)
    s1 = MultiDomainSolver(c)
    s1.assemble()
    lu1, lt1, r1 = s1.march(c.known[0])
    path = str(tmp_path / "rod5.tdbemcache")
    s1.save_matrices(path)

    s2 = MultiDomainSolver(c)
    s2.load_matrix_cache(path)
    lu2, lt2, r2 = s2.march(c.known[0])
    assert r2.failed_step == 0 and r2.history_blocks == r1.history_blocks and r2.a_blocks == r1.a_blocks
    assert np.array_equal(lu1, lu2) and np.array_equal(lt1, lt2)

    other = dataclasses.replace(c, materials=[cases.Material(21.0, 0.0, 20.0)] + list(c.materials[1:]))
    with pytest.raises(TdbemError, match="fingerprint"):
        MultiDomainSolver(other).load_matrix_cache(path)
    shorter = dataclasses.replace(c, nstep=30, known=c.known[:, :31])
    with pytest.raises(TdbemError, match="NStep"):
        MultiDomainSolver(shorter).load_matrix_cache(path)
