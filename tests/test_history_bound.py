"""The history length bound against an untruncated assembly (C oracle, CPU).

The reference assembles every history step up to MaxN
(DBEM1/multidomain.cpp:3718-3740).  The library and the oracle stop at the
last step any block can be nonzero: NeedCal skips every kernel of step k of
field element e at source s once (k - 1) dt >= (|c_e - s| + radius_e) / C2
(DBEM1/dsquareelement.cpp:1156-1190), so steps k >= 1 + D / (C2 dt) of a
domain are empty, D the largest |c_e - s| + radius_e over its pairs.  Here
a bar of a short stiff and a long soft domain (history lengths about 4x
apart) is assembled to NStep without any stop and compared with that bound,
per domain and overall.
"""
import numpy as np

from oracle_lib import Oracle


def _contrast_case(nstep=40):
    from tdbem import cases
    mats = [cases.Material(80.0, 0.25, 20.0), cases.Material(20.0, 0.25, 20.0)]
    return cases.make_case("bar2_contrast", 2, 2, mats, 0.6, nstep,
                           [(1.0, (1.0, 0.0, 0.0), cases.heaviside(nstep))], lengths=[0.5, 3.0], error=1e-13)


def _last_nonempty(o, rows, kmax):
    last = 0
    for k in range(1, kmax + 1):
        for which in ("MTS", "MGS"):
            rp, col, val = o.matrix(which, k)
            if np.any(np.diff(rp)[rows] > 0):
                last = k
    return last


def _domain_bounds(c, geo, dt):
    """1 + D / (C2 dt) per domain (the restated skip rule)."""
    from tdbem import cases
    E = c.n_elements
    per = E // len(c.materials)
    out = []
    for d, m in enumerate(c.materials):
        sl = slice(d * per, (d + 1) * per)
        ctr, rad = geo["center"][sl], geo["radius"][sl]
        # collocation node: local (0, 0) of the 8-node element, the mean of
        # its corners when the mid-side points sit at the edge midpoints
        node = c.mesh.points[c.mesh.elements[sl, :4]].mean(axis=1)
        dmax = np.max(np.linalg.norm(ctr[:, None, :] - node[None, :, :], axis=2) + rad[:, None])
        _, c2 = cases.wave_speeds(m)
        out.append(1.0 + dmax / (c2 * dt))
    return out


def test_bound_covers_every_nonzero_history_step():
    c = _contrast_case()
    o = Oracle(c)
    kb = o.history_step_bound()
    n = o.assemble(kmax=c.nstep)          # every step to NStep, no stop
    assert n == c.nstep
    geo = o.geometry()
    bounds = _domain_bounds(c, geo, o.dt)
    assert max(bounds) <= kb - 1 and kb - 1 <= np.ceil(max(bounds))
    E = c.n_elements
    per = E // 2
    lasts = [_last_nonempty(o, np.arange(d * per, (d + 1) * per), c.nstep) for d in range(2)]
    for d in range(2):
        # steps k >= 1 + D / (C2 dt) of a domain hold no block ...
        assert lasts[d] < bounds[d], (d, lasts[d], bounds[d])
        # ... and the bound is tight to a step or two
        assert lasts[d] >= bounds[d] - 3.0, (d, lasts[d], bounds[d])
    assert lasts[1] >= 3 * lasts[0]       # a large contrast between the domains
    # the default assembly stops at the bound and keeps the same steps
    o2 = Oracle(c)
    assert o2.assemble() == max(lasts)
    for k in range(1, max(lasts) + 1):
        for which in ("MTS", "MGS"):
            a, b = o.matrix(which, k), o2.matrix(which, k)
            assert all(np.array_equal(x, y) for x, y in zip(a, b)), (which, k)
