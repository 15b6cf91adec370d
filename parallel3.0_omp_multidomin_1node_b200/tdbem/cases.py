"""Synthetic multi-domain TDBEM cases: bar geometries, boundary codes and load
histories, plus writers for the reference solver's own input formats.

A case is a bar of ``domains`` box-shaped sub-domains stacked along x.  Every
box face is meshed into flat 8-node quadrilaterals (corners then edge
midpoints, outward normal = (p1-p0) x (p3-p0)).  Elements are numbered
domain-major, and inside a domain face by face: x-, x+, y-, y+, z-, z+, which
gives the contiguous equal element ranges the reference's domain split assumes
(DBEM1/multidomain.cpp:1413-1436).  The x+ face of domain d and the x- face of
domain d+1 are paired element by element as conforming interfaces with
normalSign -1 (DBEM1/multidomain.h:30-50).

Boundary codes follow the reference's constant-element multi-domain path:
elements on the x- end of the first domain are BCID 123 (displacement given,
zero), all others BCID 456 (traction given).  Prescribed values are element
local components (t1, t2, n) of a global vector, the frame the reference uses
for ``BoundaryValue::lu`` (DBEM1/dsquareelement.h:82-125).

The time step follows DBEM1/DBEM.cpp:909-914: dt = beta * mean|P0-P1| / c1 of
the card (first-domain) material.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

__all__ = [
    "Material",
    "BarMesh",
    "Case",
    "build_bar",
    "local_frames",
    "mean_element_size",
    "wave_speeds",
    "ricker",
    "make_case",
    "config_rod5",
    "config_bar8",
    "config_rod5_batched",
    "config_adjoint_rod",
    "config_layered_box",
    "write_reference_inputs",
]


@dataclasses.dataclass(frozen=True)
class Material:
    E: float
    nu: float
    rho: float

    @property
    def G(self) -> float:
        return self.E / 2.0 / (1.0 + self.nu)


def wave_speeds(m: Material) -> Tuple[float, float]:
    """(c1, c2) as DBEM1/dsquareelement.cpp:63-70 defines them."""
    G = m.G
    c1 = math.sqrt((2.0 - 2.0 * m.nu) / (1.0 - 2.0 * m.nu) * G / m.rho)
    c2 = math.sqrt(G / m.rho)
    return c1, c2


@dataclasses.dataclass
class BarMesh:
    points: np.ndarray          # (P, 3) float64
    elements: np.ndarray        # (E, 8) int64, 0-based point ids
    domain_of: np.ndarray       # (E,) int64
    face_of: np.ndarray         # (E,) int64: 0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+
    interfaces: np.ndarray      # (I, 5) int64: domainA, eleA, domainB, eleB, normalSign (0-based)
    domains: int

    @property
    def n_elements(self) -> int:
        return int(self.elements.shape[0])


class _PointTable:
    def __init__(self) -> None:
        self.points: List[Tuple[float, float, float]] = []
        self.index = {}

    def add(self, p) -> int:
        key = (round(float(p[0]), 12), round(float(p[1]), 12), round(float(p[2]), 12))
        i = self.index.get(key)
        if i is None:
            i = len(self.points)
            self.index[key] = i
            self.points.append(key)
        return i


def _quad(table: _PointTable, c0, c1, c2, c3) -> List[int]:
    corners = [np.asarray(c, dtype=np.float64) for c in (c0, c1, c2, c3)]
    mids = [0.5 * (corners[i] + corners[(i + 1) % 4]) for i in range(4)]
    return [table.add(p) for p in corners + mids]


def build_bar(domains: int, length: float, width: float, height: float,
              nx: int, ny: int, nz: int, lengths: Optional[Sequence[float]] = None) -> BarMesh:
    """Bar of ``domains`` boxes along x, centred on the origin; ``lengths``
    gives each box's length along x (default: ``length / domains`` each).
    Every box has the same element count, as the reference's contiguous
    equal domain ranges require."""
    if domains < 1 or min(nx, ny, nz) < 1:
        raise ValueError("domains and face divisions must be >= 1")
    table = _PointTable()
    elems: List[List[int]] = []
    dom: List[int] = []
    face: List[int] = []
    first_of_face: List[dict] = []
    y0, y1 = -0.5 * width, 0.5 * width
    z0, z1 = -0.5 * height, 0.5 * height
    if lengths is None:
        lengths = [length / domains] * domains
    if len(lengths) != domains or min(lengths) <= 0.0:
        raise ValueError("lengths: one positive length per domain")
    length = float(sum(lengths))
    starts = np.concatenate([[0.0], np.cumsum(lengths)])
    ys = np.linspace(y0, y1, ny + 1)
    zs = np.linspace(z0, z1, nz + 1)
    for d in range(domains):
        xa = -0.5 * length + starts[d]
        xb = xa + lengths[d]
        xs = np.linspace(xa, xb, nx + 1)
        faces = {}
        # x- face: outward -x.  (p1-p0) along +z, (p3-p0) along +y -> z x y = -x
        faces[0] = len(elems)
        for iy in range(ny):
            for iz in range(nz):
                elems.append(_quad(table, (xa, ys[iy], zs[iz]), (xa, ys[iy], zs[iz + 1]),
                                   (xa, ys[iy + 1], zs[iz + 1]), (xa, ys[iy + 1], zs[iz])))
                dom.append(d); face.append(0)
        # x+ face: outward +x.  y x z = +x
        faces[1] = len(elems)
        for iy in range(ny):
            for iz in range(nz):
                elems.append(_quad(table, (xb, ys[iy], zs[iz]), (xb, ys[iy + 1], zs[iz]),
                                   (xb, ys[iy + 1], zs[iz + 1]), (xb, ys[iy], zs[iz + 1])))
                dom.append(d); face.append(1)
        # y- face: outward -y.  x x z = -y
        for ix in range(nx):
            for iz in range(nz):
                elems.append(_quad(table, (xs[ix], y0, zs[iz]), (xs[ix + 1], y0, zs[iz]),
                                   (xs[ix + 1], y0, zs[iz + 1]), (xs[ix], y0, zs[iz + 1])))
                dom.append(d); face.append(2)
        # y+ face: outward +y.  z x x = +y
        for ix in range(nx):
            for iz in range(nz):
                elems.append(_quad(table, (xs[ix], y1, zs[iz]), (xs[ix], y1, zs[iz + 1]),
                                   (xs[ix + 1], y1, zs[iz + 1]), (xs[ix + 1], y1, zs[iz])))
                dom.append(d); face.append(3)
        # z- face: outward -z.  y x x = -z
        for ix in range(nx):
            for iy in range(ny):
                elems.append(_quad(table, (xs[ix], ys[iy], z0), (xs[ix], ys[iy + 1], z0),
                                   (xs[ix + 1], ys[iy + 1], z0), (xs[ix + 1], ys[iy], z0)))
                dom.append(d); face.append(4)
        # z+ face: outward +z.  x x y = +z
        for ix in range(nx):
            for iy in range(ny):
                elems.append(_quad(table, (xs[ix], ys[iy], z1), (xs[ix + 1], ys[iy], z1),
                                   (xs[ix + 1], ys[iy + 1], z1), (xs[ix], ys[iy + 1], z1)))
                dom.append(d); face.append(5)
        first_of_face.append(faces)
    itf = []
    nyz = ny * nz
    for d in range(domains - 1):
        a0 = first_of_face[d][1]
        b0 = first_of_face[d + 1][0]
        for j in range(nyz):
            itf.append((d, a0 + j, d + 1, b0 + j, -1))
    mesh = BarMesh(points=np.asarray(table.points, dtype=np.float64),
                   elements=np.asarray(elems, dtype=np.int64),
                   domain_of=np.asarray(dom, dtype=np.int64),
                   face_of=np.asarray(face, dtype=np.int64),
                   interfaces=np.asarray(itf, dtype=np.int64).reshape(-1, 5),
                   domains=domains)
    _check_pairs(mesh)
    return mesh


def _check_pairs(mesh: BarMesh) -> None:
    for dA, eA, dB, eB, _ in mesh.interfaces:
        ca = mesh.points[mesh.elements[eA, :4]].mean(axis=0)
        cb = mesh.points[mesh.elements[eB, :4]].mean(axis=0)
        if np.max(np.abs(ca - cb)) > 1e-9:
            raise RuntimeError(f"non-conforming interface pair {eA} <-> {eB}")


def local_frames(mesh: BarMesh) -> np.ndarray:
    """(E, 3, 3) rows t1, t2, n of each flat element's local frame."""
    p = mesh.points[mesh.elements]
    t1 = p[:, 1] - p[:, 0]
    t1 /= np.linalg.norm(t1, axis=1, keepdims=True)
    r2 = p[:, 3] - p[:, 0]
    n = np.cross(t1, r2)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    t2 = np.cross(n, t1)
    return np.stack([t1, t2, n], axis=1)


def mean_element_size(mesh: BarMesh) -> float:
    """Mean corner-0 to corner-1 distance (DBEM1/DBEM.cpp:2383-2396)."""
    p = mesh.points[mesh.elements]
    return float(np.mean(np.linalg.norm(p[:, 1] - p[:, 0], axis=1)))


def ricker(t: np.ndarray, f0: float, t0: Optional[float] = None) -> np.ndarray:
    """Ricker wavelet (1 - 2 pi^2 f0^2 tau^2) exp(-pi^2 f0^2 tau^2), tau = t - t0."""
    if t0 is None:
        t0 = 1.0 / f0
    a = (math.pi * f0 * (np.asarray(t, dtype=np.float64) - t0)) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


@dataclasses.dataclass
class Case:
    """One multi-domain problem with R load cases (R = known.shape[0])."""
    name: str
    mesh: BarMesh
    materials: List[Material]
    bcid: np.ndarray            # (E,) int64, 123 or 456
    known: np.ndarray           # (R, NStep+1, E, 3) element-local prescribed values
    beta: float
    nstep: int
    gap: float = 0.4
    iterations: int = 200
    error: float = 1.0e-5
    max_leaf: int = 10
    dt: float = 0.0
    card: Optional[Material] = None  # the datacard material that sets dt (None: the first domain's)

    @property
    def n_elements(self) -> int:
        return self.mesh.n_elements

    @property
    def n_loads(self) -> int:
        return int(self.known.shape[0])

    def card_material(self) -> Material:
        return self.card if self.card is not None else self.materials[0]


def _finish_case(name, mesh, materials, beta, nstep, loads, **kw) -> Case:
    """loads: list of (amplitude, unit_direction(3,), profile(NStep+1,)) for the x+ end."""
    E = mesh.n_elements
    bcid = np.full(E, 456, dtype=np.int64)
    fixed = (mesh.domain_of == 0) & (mesh.face_of == 0)
    bcid[fixed] = 123
    loaded = (mesh.domain_of == mesh.domains - 1) & (mesh.face_of == 1)
    frames = local_frames(mesh)
    known = np.zeros((len(loads), nstep + 1, E, 3), dtype=np.float64)
    for r, (amp, direction, profile) in enumerate(loads):
        g = np.asarray(direction, dtype=np.float64)
        loc = np.einsum("eij,j->ei", frames[loaded], g)          # (nl, 3)
        known[r][:, loaded, :] = amp * np.asarray(profile)[:, None, None] * loc[None]
    c1, _ = wave_speeds(materials[0])
    dt = beta * mean_element_size(mesh) / c1
    return Case(name=name, mesh=mesh, materials=list(materials), bcid=bcid, known=known,
                beta=beta, nstep=nstep, dt=dt, **kw)


def heaviside(nstep: int) -> np.ndarray:
    h = np.ones(nstep + 1)
    h[0] = 0.0
    return h


def make_case(name: str, domains: int, n: int, materials: Sequence[Material], beta: float, nstep: int,
              loads, length: Optional[float] = None, width: float = 1.0, height: float = 1.0,
              nx: Optional[int] = None, lengths: Optional[Sequence[float]] = None, **kw) -> Case:
    if length is None:
        length = float(domains)
    mesh = build_bar(domains, length, width, height, nx if nx else n, n, n, lengths=lengths)
    return _finish_case(name, mesh, materials, beta, nstep, loads, **kw)


def config_rod5(nstep: int = 100, n: int = 2, **kw) -> Case:
    """1x1x5 bar of 5 unit-cube domains, n x n per face, E=20 nu=0 rho=20,
    beta 0.6, Heaviside unit axial traction on the x+ end."""
    mats = [Material(20.0, 0.0, 20.0)] * 5
    return make_case(f"rod5_n{n}", 5, n, mats, 0.6, nstep,
                     [(1.0, (1.0, 0.0, 0.0), heaviside(nstep))], **kw)


def config_bar8(nstep: int = 400, n: int = 8, seed: int = 2, **kw) -> Case:
    """1x1x8 bar of 8 unit-cube domains, n x n per face, E alternating 20/80,
    nu 0.25, rho 20, beta 0.6; end traction shaped as a Ricker pulse with peak
    frequency 0.5 c1/L (L = 1) along a seeded unit direction."""
    mats = [Material(20.0 if d % 2 == 0 else 80.0, 0.25, 20.0) for d in range(8)]
    rng = np.random.default_rng(seed)
    v = rng.normal(size=3)
    v /= np.linalg.norm(v)
    c1, _ = wave_speeds(mats[0])
    mesh = build_bar(8, 8.0, 1.0, 1.0, n, n, n)
    dt = 0.6 * mean_element_size(mesh) / c1
    prof = ricker(np.arange(nstep + 1) * dt, 0.5 * c1)
    return _finish_case(f"bar8_n{n}", mesh, mats, 0.6, nstep, [(1.0, v, prof)], **kw)


def config_rod5_batched(nstep: int = 200, n: int = 2, loads: int = 32, seed: int = 3, **kw) -> Case:
    """Config-1 geometry with R seeded load cases: amplitude U(0.5, 2), random
    unit direction, Heaviside or Ricker profile."""
    mats = [Material(20.0, 0.0, 20.0)] * 5
    mesh = build_bar(5, 5.0, 1.0, 1.0, n, n, n)
    c1, _ = wave_speeds(mats[0])
    dt = 0.6 * mean_element_size(mesh) / c1
    rng = np.random.default_rng(seed)
    L = []
    for _ in range(loads):
        amp = rng.uniform(0.5, 2.0)
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        if rng.uniform() < 0.5:
            prof = heaviside(nstep)
        else:
            prof = ricker(np.arange(nstep + 1) * dt, 0.5 * c1)
        L.append((amp, v, prof))
    return _finish_case(f"rod5_n{n}_R{loads}", mesh, mats, 0.6, nstep, L, **kw)


def config_uneven_rods(count: int = 16, nstep: int = 200, n_min: int = 4, n_max: int = 12, seed: int = 6,
                       **kw) -> list:
    """Independent 5-domain rods (config-1 geometry) with n x n elements per
    face, n seeded in [n_min, n_max], per-domain E log-uniform in [10, 100],
    nu 0.25, rho 20, each with one seeded end load (amplitude U(0.5, 2),
    random direction, Heaviside or Ricker)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(n_min, n_max + 1))
        mats = [Material(float(np.exp(rng.uniform(np.log(10.0), np.log(100.0)))), 0.25, 20.0) for _ in range(5)]
        mesh = build_bar(5, 5.0, 1.0, 1.0, n, n, n)
        c1, _ = wave_speeds(mats[0])
        dt = 0.6 * mean_element_size(mesh) / c1
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        prof = heaviside(nstep) if rng.uniform() < 0.5 else ricker(np.arange(nstep + 1) * dt, 0.5 * c1)
        out.append(_finish_case(f"rod5_n{n}_u{i}", mesh, mats, 0.6, nstep, [(rng.uniform(0.5, 2.0), v, prof)], **kw))
    return out


def config_adjoint_rod(nstep: int = 200, n: int = 4, seed: int = 5, **kw) -> Case:
    """5-domain rod, 4 x 4 per face, seeded per-domain E in [15, 30] and rho in
    [15, 25]; Heaviside axial end traction."""
    rng = np.random.default_rng(seed)
    mats = [Material(rng.uniform(15, 30), 0.25, rng.uniform(15, 25)) for _ in range(5)]
    return make_case(f"adj_rod5_n{n}", 5, n, mats, 0.6, nstep,
                     [(1.0, (1.0, 0.0, 0.0), heaviside(nstep))], **kw)


def config_layered_box(nstep: int = 1000, n: int = 24, nx: int = 6, loads: int = 8, seed: int = 7, **kw) -> Case:
    """4x4x4 box in 4 layers along x (n x n on the layer faces, nx divisions
    through each layer), per-layer E log-uniform [10, 100], nu 0.25, rho U(1, 3);
    x- face fixed, R seeded Ricker tractions on the x+ face."""
    rng = np.random.default_rng(seed)
    mats = [Material(float(np.exp(rng.uniform(np.log(10), np.log(100)))), 0.25, rng.uniform(1, 3))
            for _ in range(4)]
    mesh = build_bar(4, 4.0, 4.0, 4.0, nx, n, n)
    c1, _ = wave_speeds(mats[0])
    dt = 0.6 * mean_element_size(mesh) / c1
    L = []
    for _ in range(loads):
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        L.append((rng.uniform(0.5, 2.0), v, ricker(np.arange(nstep + 1) * dt, 0.5 * c1 / 4.0)))
    return _finish_case(f"box4_n{n}", mesh, mats, 0.6, nstep, L, **kw)


def _fmt(v: float) -> str:
    if abs(v) < 1.0e-300:
        v = 0.0
    return repr(float(v))


def write_reference_inputs(case: Case, directory: str, load: int = 0, threads: int = 8,
                           error: Optional[float] = None) -> str:
    """Write BEM_DATACARD.DAT and input/<name>.model|.bd for the reference
    solver (DBEM1/DBEM.cpp:637-791, 826-1085; DBEM1/multidomain.cpp:1305-1362).
    Returns the case title.  Values are written with 17 significant digits so
    the reference reads back exactly the doubles held here."""
    os.makedirs(os.path.join(directory, "input"), exist_ok=True)
    title = case.name
    mesh = case.mesh
    with open(os.path.join(directory, "input", title + ".model"), "w") as f:
        f.write(f"{len(mesh.points)}\n")
        for p in mesh.points:
            f.write(f"{_fmt(p[0])}\t{_fmt(p[1])}\t{_fmt(p[2])}\n")
        f.write(f"{mesh.n_elements}\n")
        for e in mesh.elements:
            f.write("\t".join(str(int(i) + 1) for i in e) + "\n")
        f.write("0\n")
    with open(os.path.join(directory, "input", title + ".bd"), "w") as f:
        f.write("\n".join(str(int(b)) for b in case.bcid) + "\n")
        vals = case.known[load]
        for s in range(case.nstep + 1):
            f.write("\n".join("\t".join(_fmt(x) for x in row) for row in vals[s]) + "\n")
    m0 = case.card_material()
    err = case.error if error is None else error
    with open(os.path.join(directory, "BEM_DATACARD.DAT"), "w") as f:
        f.write(f"{title}\n{threads}\n2\n{_fmt(case.beta)}\n{case.nstep}\n{_fmt(case.gap)}\n")
        f.write(f"{_fmt(m0.E)}\n{_fmt(m0.nu)}\n{_fmt(m0.rho)}\n1\n2\n")
        f.write(f"{case.iterations}\n{_fmt(err)}\n{case.max_leaf}\n0\n0\n")
        f.write(f"{mesh.domains}\n")
        for d, m in enumerate(case.materials):
            f.write(f"{d + 1} {_fmt(m.E)} {_fmt(m.nu)} {_fmt(m.rho)}\n")
        f.write(f"{len(mesh.interfaces)}\n")
        for dA, eA, dB, eB, s in mesh.interfaces:
            f.write(f"{dA + 1} {eA + 1} {dB + 1} {eB + 1} {s}\n")
    return title


def read_reference_inputs(directory: str) -> Case:
    """Read a reference case directory (BEM_DATACARD.DAT + input/<title>.model
    and .bd, text form) into a Case with one load case.  Follows the card
    layout of DBEM1/DBEM.cpp:637-791 for solver 2 with the optional
    multi-domain tail of DBEM1/multidomain.cpp:1305-1362; element and
    domain ids in the interface lines may be 0- or 1-based as the reference
    accepts (DBEM1/multidomain.cpp:1439-1460)."""
    tok = open(os.path.join(directory, "BEM_DATACARD.DAT")).read().split()
    pos = 0

    def nxt():
        nonlocal pos
        pos += 1
        return tok[pos - 1]

    title = nxt()
    _threads = int(nxt()); _flag = int(nxt())
    beta = float(nxt()); nstep = int(nxt()); gap = float(nxt())
    E = float(nxt()); nu = float(nxt()); rho = float(nxt()); _amp = float(nxt())
    solver = int(nxt())
    if solver != 2:
        raise ValueError("only the GMRES solver card (solvers = 2) is supported")
    iterations = int(nxt()); error = float(nxt()); max_leaf = int(nxt())
    _inmode = int(nxt()); _batch = int(nxt())
    ndom = int(nxt())
    mats = [None] * ndom
    raw = [(int(nxt()), float(nxt()), float(nxt()), float(nxt())) for _ in range(ndom)]
    zero_based = any(r[0] == 0 for r in raw)
    for i, e, v, r in raw:
        mats[i if zero_based else i - 1] = Material(e, v, r)
    nitf = int(nxt()) if pos < len(tok) else 0
    itf_raw = [tuple(int(nxt()) for _ in range(5)) for _ in range(nitf)]
    ele_zero = any(t[1] == 0 or t[3] == 0 for t in itf_raw)
    dom_zero = any(t[0] == 0 or t[2] == 0 for t in itf_raw)
    itf = [(a - (0 if dom_zero else 1), ea - (0 if ele_zero else 1), b - (0 if dom_zero else 1),
            eb - (0 if ele_zero else 1), -1 if s == 0 else s) for a, ea, b, eb, s in itf_raw]

    mt = open(os.path.join(directory, "input", title + ".model")).read().split()
    p = 0
    npts = int(mt[p]); p += 1
    pts = np.array(mt[p:p + 3 * npts], dtype=np.float64).reshape(npts, 3); p += 3 * npts
    ne = int(mt[p]); p += 1
    ele = np.array(mt[p:p + 8 * ne], dtype=np.int64).reshape(ne, 8) - 1
    bt = open(os.path.join(directory, "input", title + ".bd")).read().split()
    bcid = np.array(bt[:ne], dtype=np.int64)
    vals = np.array(bt[ne:ne + (nstep + 1) * ne * 3], dtype=np.float64).reshape(1, nstep + 1, ne, 3)
    per = ne // ndom
    extra = ne % ndom
    dom = np.zeros(ne, dtype=np.int64)
    b = 0
    for d in range(ndom):
        c = per + (1 if d < extra else 0)
        dom[b:b + c] = d
        b += c
    mesh = BarMesh(points=pts, elements=ele, domain_of=dom, face_of=np.full(ne, -1, dtype=np.int64),
                   interfaces=np.asarray(itf, dtype=np.int64).reshape(-1, 5), domains=ndom)
    c1, _ = wave_speeds(Material(E, nu, rho))
    dt = beta * mean_element_size(mesh) / c1
    return Case(name=title, mesh=mesh, materials=mats, bcid=bcid, known=vals, beta=beta, nstep=nstep,
                gap=gap, iterations=iterations, error=error, max_leaf=max_leaf, dt=dt)


def config_bar8_batched(nstep: int = 400, n: int = 8, loads: int = 32, seed: int = 4, **kw) -> Case:
    """The 8-domain bar with R seeded load cases on the x+ end: amplitude
    U(0.5, 2), random unit direction, Heaviside or Ricker (peak frequency
    0.5 c1/L) time profile."""
    mats = [Material(20.0 if d % 2 == 0 else 80.0, 0.25, 20.0) for d in range(8)]
    mesh = build_bar(8, 8.0, 1.0, 1.0, n, n, n)
    c1, _ = wave_speeds(mats[0])
    dt = 0.6 * mean_element_size(mesh) / c1
    rng = np.random.default_rng(seed)
    L = []
    for _ in range(loads):
        amp = rng.uniform(0.5, 2.0)
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        prof = heaviside(nstep) if rng.uniform() < 0.5 else ricker(np.arange(nstep + 1) * dt, 0.5 * c1)
        L.append((amp, v, prof))
    return _finish_case(f"bar8_n{n}_R{loads}", mesh, mats, 0.6, nstep, L, **kw)
