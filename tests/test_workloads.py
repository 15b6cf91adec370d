"""The synthetic workloads the measurements are quoted on have the sizes
stated for them: element counts, domains, interface pairs, load cases and
steps (generators in tdbem/cases.py)."""
import numpy as np


def test_bar_rod_box_sizes():
    from tdbem import cases
    bar = cases.config_bar8(nstep=4)
    assert bar.n_elements == 3072 and len(bar.materials) == 8 and len(bar.mesh.interfaces) == 7 * 64
    assert [m.E for m in bar.materials] == [20.0, 80.0] * 4
    rod = cases.config_rod5(nstep=4)
    assert rod.n_elements == 120 and len(rod.mesh.interfaces) == 16
    batch = cases.config_rod5_batched(nstep=4, loads=32)
    assert batch.n_elements == 120 and batch.known.shape == (32, 5, 120, 3)
    box = cases.config_layered_box(nstep=2)
    assert box.n_elements == 6912 and len(box.materials) == 4 and box.known.shape[0] == 8
    adj = cases.config_adjoint_rod(nstep=2)
    assert adj.n_elements == 480
    assert all(15 <= m.E <= 30 and 15 <= m.rho <= 25 for m in adj.materials)


def test_uneven_rods():
    from tdbem import cases
    rods = cases.config_uneven_rods(count=16, nstep=2)
    sizes = sorted(c.n_elements for c in rods)
    assert len(rods) == 16 and sizes[0] >= 30 * 16 and sizes[-1] <= 30 * 144
    assert all(10 <= m.E <= 100 for c in rods for m in c.materials)
    # every rod: fixed x- end (BCID 123), loaded x+ end
    assert all(np.any(c.bcid == 123) and np.any(c.known != 0.0) for c in rods)
