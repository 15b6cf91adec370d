"""ctypes binding of the C restatement oracle (oracle/tdbem_oracle.c).

Test infrastructure: used only by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, always as the checker.
"""
import ctypes
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(REPO, "oracle", "_build", "libtdbem_oracle.so")

_lib = None


class _CCSR(ctypes.Structure):
    _fields_ = [("n_rows", ctypes.c_int64), ("nnz", ctypes.c_int64),
                ("row_ptr", ctypes.POINTER(ctypes.c_int32)), ("col", ctypes.POINTER(ctypes.c_int32)),
                ("val", ctypes.POINTER(ctypes.c_double))]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "port"], check=True,
                           stdout=subprocess.DEVNULL)
        L = ctypes.CDLL(LIB_PATH)
        P, D, I64, I32 = ctypes.c_void_p, ctypes.c_double, ctypes.c_int64, ctypes.c_int32
        L.orc_create.restype = P
        L.orc_create.argtypes = [I64, P, I64, P, P, I32, P, I64, P, D, D, D, D, D, I32, I32, D, I32, D]
        L.orc_destroy.argtypes = [P]
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_dt.restype = D
        L.orc_dt.argtypes = [P]
        L.orc_dof_counts.argtypes = [P, P]
        L.orc_geometry.argtypes = [P] + [P] * 9
        L.orc_assemble.restype = I32
        L.orc_assemble.argtypes = [P, I32]
        L.orc_history_step_bound.restype = I32
        L.orc_history_step_bound.argtypes = [P]
        L.orc_matrix.restype = I32
        L.orc_matrix.argtypes = [P, I32, I32, ctypes.POINTER(_CCSR)]
        L.orc_precond_layout.restype = I64
        L.orc_precond_layout.argtypes = [P, P, P, P]
        L.orc_march.restype = I32
        L.orc_march.argtypes = [P, P, P, P, P, P, P]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    """One oracle problem built from a tdbem.cases.Case (load case ``load``)."""

    def __init__(self, case, tol=None, restart=None, max_length=1000.0):
        L = lib()
        m = case.mesh
        self.case = case
        self._keep = [np.ascontiguousarray(m.points, dtype=np.float64),
                      np.ascontiguousarray(m.elements, dtype=np.int64),
                      np.ascontiguousarray(case.bcid, dtype=np.int32),
                      np.ascontiguousarray([[x.E, x.nu, x.rho] for x in case.materials], dtype=np.float64),
                      np.ascontiguousarray(m.interfaces, dtype=np.int64)]
        pts, ele, bc, mats, itf = self._keep
        c = case.card_material()
        self.h = L.orc_create(len(pts), _ptr(pts), len(ele), _ptr(ele), _ptr(bc), len(mats), _ptr(mats),
                              len(itf), _ptr(itf), c.E, c.nu, c.rho, case.beta, case.gap, case.nstep,
                              restart or case.iterations, case.error if tol is None else tol, case.max_leaf,
                              max_length)
        if not self.h:
            raise ValueError(L.orc_last_error().decode())
        self.E = case.n_elements

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    @property
    def dt(self):
        return lib().orc_dt(self.h)

    def dof_counts(self):
        out = np.zeros(3, dtype=np.int64)
        lib().orc_dof_counts(self.h, _ptr(out))
        return out

    def geometry(self):
        E = self.E
        g = dict(coordcoef=np.zeros((E, 3, 8)), center=np.zeros((E, 3)), radius=np.zeros(E),
                 radius_pw=np.zeros(E), rcen_pw=np.zeros((E, 36, 3)), transmat=np.zeros((E, 9)),
                 on_u1=np.zeros((E, 9)), on_t1=np.zeros((E, 9)), on_t2=np.zeros((E, 9)))
        lib().orc_geometry(self.h, *(_ptr(g[k]) for k in ("coordcoef", "center", "radius", "radius_pw",
                                                           "rcen_pw", "transmat", "on_u1", "on_t1", "on_t2")))
        return g

    def assemble(self, kmax=0):
        return lib().orc_assemble(self.h, kmax)

    def history_step_bound(self):
        return lib().orc_history_step_bound(self.h)

    def matrix(self, which, k=0):
        """which: 'A', 'KnownM', 'MTS', 'MGS' -> (row_ptr, col, val[nnz, 9]) copies."""
        code = {"A": 0, "KnownM": 1, "MTS": 2, "MGS": 3}[which]
        m = _CCSR()
        if not lib().orc_matrix(self.h, code, k, ctypes.byref(m)):
            raise KeyError((which, k))
        rp = np.ctypeslib.as_array(m.row_ptr, shape=(m.n_rows + 1,)).copy()
        if m.nnz:
            col = np.ctypeslib.as_array(m.col, shape=(m.nnz,)).copy()
            val = np.ctypeslib.as_array(m.val, shape=(m.nnz * 9,)).copy().reshape(m.nnz, 9)
        else:
            col = np.zeros(0, np.int32)
            val = np.zeros((0, 9))
        return rp, col, val

    def precond_layout(self):
        E = self.E
        rep = np.zeros(E, np.int64)
        lb = np.zeros(E, np.int64)
        lc = np.zeros(E, np.int64)
        n = lib().orc_precond_layout(self.h, _ptr(rep), _ptr(lb), _ptr(lc))
        return rep, lb[:n], lc[:n]

    def march(self, known):
        """known: (NStep+1, E, 3) -> dict(bd_lu, bd_lt, rhs, x, flags, solved)."""
        N = self.case.nstep
        E = self.E
        known = np.ascontiguousarray(known, dtype=np.float64)
        lu = np.zeros((N + 1, 3 * E))
        lt = np.zeros((N + 1, 3 * E))
        rhs = np.zeros((N, 3 * E))
        x = np.zeros((N, 3 * E))
        flags = np.zeros((N, 3), np.int32)
        solved = lib().orc_march(self.h, _ptr(known), _ptr(lu), _ptr(lt), _ptr(rhs), _ptr(x), _ptr(flags))
        return dict(bd_lu=lu, bd_lt=lt, rhs=rhs, x=x, flags=flags, solved=solved)
