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


def test_cache_sections_are_the_references_layout(tmp_path):
    """Every matrix of a saved cache (A, KnownM, each MTS_k and MGS_k) is read
    by the reference's own CCSRMat::ReadBinary at its offset and written back
    byte for byte by CCSRMat::WriteBinary (the reference's binary layout on
    this platform: 64-bit counts, int32 row pointers and columns, 9 doubles
    per block); the file's own header and index come before them."""
    import os
    import struct
    from test_builder import REF_CCSR, reference_rewrite
    if not os.path.exists(REF_CCSR):
        pytest.skip("reference CCSR harness not built (needs the reference sources)")
    from tdbem import cases
    from tdbem.api import MultiDomainSolver
    c = cases.config_rod5(nstep=20, error=1e-13)
    s = MultiDomainSolver(c)
    s.assemble()
    path = str(tmp_path / "rod5.tdbemcache")
    s.save_matrices(path)
    data = open(path, "rb").read()
    magic, version, count = struct.unpack_from("<16s2i", data, 0)
    assert magic.rstrip(b"\0") == b"TDBEMMDCACHE" and version == 1
    E = struct.unpack_from("<q", data, 24)[0]
    head = 16 + 8 + 6 * 8 + 2 * 8 + 8
    seen = set()
    for i in range(count):
        typ, step, off, nbytes = struct.unpack_from("<2i2q", data, head + 24 * i)
        again, n, nnz = reference_rewrite(path, off)
        assert n == E
        assert again == data[off:off + nbytes], (typ, step)
        seen.add(typ)
    assert seen == {1, 2, 3, 4}
