"""Python binding of the B200 multi-domain TDBEM library (include/tdbem.h).

``DynaGMRESSolverMultiDomainCCSR`` mirrors the reference entry point of the
same name (DBEM1/multidomain.h:214-223): it takes the model, the boundary
values bd[0..NStep] (element-local prescribed values in ``lu``) and the
datacard's iterations / error / premaxleafpointnum / NStep / MaxLength, and
returns 1 when every step converged, -1 otherwise, with bd overwritten by the
global-frame displacement and traction histories.  ``MultiDomainSolver`` is
the handle-level API (create, assemble, march, exports).

There is no CPU path: loading fails loudly when the CUDA library is absent.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

from . import build as _build

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "libtdbem_b200.so")

PRECISION = {"fp64": 0, "mixed": 1}
STATUS = {0: "OK", 1: "INVALID_INPUT", 2: "DOFMAP_INVALID", 3: "SINGULAR_BLOCK", 4: "NOT_CONVERGED",
          5: "CUDA_ERROR", 6: "OUT_OF_MEMORY", 7: "NOT_ASSEMBLED"}


class TdbemError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class _Problem(ctypes.Structure):
    _fields_ = [("n_points", ctypes.c_int64), ("points", ctypes.c_void_p), ("n_elements", ctypes.c_int64),
                ("elements", ctypes.c_void_p), ("bcid", ctypes.c_void_p), ("n_domains", ctypes.c_int32),
                ("materials", ctypes.c_void_p), ("n_interfaces", ctypes.c_int64), ("interfaces", ctypes.c_void_p),
                ("card_E", ctypes.c_double), ("card_nu", ctypes.c_double), ("card_rho", ctypes.c_double),
                ("beta", ctypes.c_double), ("gap", ctypes.c_double), ("n_steps", ctypes.c_int32),
                ("restart", ctypes.c_int32), ("tol", ctypes.c_double), ("max_leaf", ctypes.c_int32),
                ("max_length", ctypes.c_double), ("precision", ctypes.c_int32), ("n_loads", ctypes.c_int32),
                ("dt", ctypes.c_double)]


class Report(ctypes.Structure):
    _fields_ = [("steps_solved", ctypes.c_int32), ("failed_step", ctypes.c_int32), ("gmres_flag", ctypes.c_int32),
                ("total_inner", ctypes.c_int64), ("max_refinements", ctypes.c_int32),
                ("history_steps", ctypes.c_int32), ("history_blocks", ctypes.c_int64),
                ("a_blocks", ctypes.c_int64), ("max_interface_jump", ctypes.c_double),
                ("max_interface_balance", ctypes.c_double), ("rhs_bytes", ctypes.c_double),
                ("ms_rhs", ctypes.c_double),
                ("ms_gmres", ctypes.c_double), ("ms_total", ctypes.c_double), ("gmres_cluster", ctypes.c_int32),
                ("gmres_groups", ctypes.c_int32), ("rhs_block_reads", ctypes.c_double),
                ("history_launches", ctypes.c_int32), ("ms_history", ctypes.c_double),
                ("history_bytes", ctypes.c_double), ("history_block_steps", ctypes.c_double),
                ("history_vector_loads", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None

class Tuning(ctypes.Structure):
    _fields_ = [("gmres_groups", ctypes.c_int32), ("gmres_cluster", ctypes.c_int32),
                ("rhs_cases_per_thread", ctypes.c_int32), ("candidates", ctypes.c_int32),
                ("steps", ctypes.c_int32), ("ms_per_step", ctypes.c_double),
                ("ms_per_step_default", ctypes.c_double)]


# every entry point of include/tdbem.h with (restype, argtypes)
_P, _I32, _I64, _D = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
SIGNATURES = {
    "tdbem_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "tdbem_last_error": (ctypes.c_char_p, []),
    "tdbem_abi_version": (_I32, []),
    "tdbem_md_create": (ctypes.c_int, [ctypes.POINTER(_Problem), _I32, ctypes.POINTER(_P)]),
    "tdbem_md_destroy": (None, [_P]),
    "tdbem_md_assemble": (ctypes.c_int, [_P, _P]),
    "tdbem_md_load_matrices": (ctypes.c_int, [_P] + [_P] * 6 + [_I32] + [_P] * 6 + [_P]),
    "tdbem_md_march": (ctypes.c_int, [_P, _P, _P, _P, ctypes.POINTER(Report), _P]),
    "tdbem_md_march_device": (ctypes.c_int, [_P, _P, _P, _P, ctypes.POINTER(Report), _P]),
    "tdbem_md_march_many": (ctypes.c_int, [_P, _I32, _P, _P, _P, _P, _P]),
    "tdbem_md_march_vjp": (ctypes.c_int, [_P, _P, _P, _P, ctypes.POINTER(Report), _P]),
    "tdbem_md_march_forward": (ctypes.c_int, [_P, _P, _P, _P, ctypes.POINTER(Report), _P]),
    "tdbem_md_march_backward": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.POINTER(Report), _P]),
    "tdbem_md_autotune": (ctypes.c_int, [_P, _P, _I32, ctypes.POINTER(Tuning), _P]),
    "tdbem_md_set_record": (ctypes.c_int, [_P, _I32]),
    "tdbem_md_step_record": (ctypes.c_int, [_P, _P, _P, _P]),
    "tdbem_md_export_matrix": (ctypes.c_int, [_P, _I32, _I32, ctypes.POINTER(_I64), ctypes.POINTER(_I64), _P, _P, _P]),
    "tdbem_md_geometry": (ctypes.c_int, [_P] + [_P] * 8),
    "tdbem_md_info": (ctypes.c_int, [_P, ctypes.POINTER(_D)] + [ctypes.POINTER(_I64)] * 4),
    "tdbem_md_precond_layout": (ctypes.c_int, [_P, _P, _P, _P]),
    "tdbem_md_solve_noalloc": (ctypes.c_int, [_P, _P, _P, _P, _P]),
    "tdbem_md_write_validation": (ctypes.c_int, [_P, ctypes.c_char_p, _I32, _P, _P, ctypes.POINTER(Report)]),
    "tdbem_md_write_rhs_diagnostics": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.POINTER(Report)]),
    "tdbem_md_save_matrices": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "tdbem_md_load_matrix_cache": (ctypes.c_int, [_P, ctypes.c_char_p, _P]),
    "tdbem_case_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_P)]),
    "tdbem_case_problem": (ctypes.c_int, [_P, ctypes.POINTER(_Problem)]),
    "tdbem_case_known": (ctypes.c_int, [_P, _P]),
    "tdbem_case_title": (ctypes.c_char_p, [_P]),
    "tdbem_case_destroy": (None, [_P]),
}


def load_library(build_if_missing: bool = True):
    """Load (building first if needed) the in-tree CUDA library."""
    global _lib
    if _lib is None:
        if build_if_missing:
            _build.build()
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA library {LIB_PATH} is missing; run tdbem/build.py (no CPU fallback exists)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _check(status):
    if status != 0:
        raise TdbemError(status, load_library().tdbem_last_error().decode())


class CaseFiles:
    """A reference case directory read by the library's input layer
    (tdbem_case_read): the problem description and the prescribed values
    of every load case, shape (n_loads, n_steps + 1, n_elements, 3)."""

    def __init__(self, directory: str):
        L = load_library()
        self.c = ctypes.c_void_p()
        _check(L.tdbem_case_read(os.fsencode(directory), ctypes.byref(self.c)))
        self.problem = _Problem()
        _check(L.tdbem_case_problem(self.c, ctypes.byref(self.problem)))
        p = self.problem
        self.title = L.tdbem_case_title(self.c).decode()
        self.n_elements, self.n_steps, self.n_loads = p.n_elements, p.n_steps, p.n_loads
        self.known = np.zeros((p.n_loads, p.n_steps + 1, p.n_elements, 3))
        _check(L.tdbem_case_known(self.c, _ptr(self.known)))

    def arrays(self):
        """Copies of the problem arrays: points, elements, bcid, materials, interfaces."""
        p = self.problem

        def arr(ptr, n, ct):
            return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), shape=(n,)).copy()
        return dict(points=arr(p.points, 3 * p.n_points, ctypes.c_double).reshape(-1, 3),
                    elements=arr(p.elements, 8 * p.n_elements, ctypes.c_int64).reshape(-1, 8),
                    bcid=arr(p.bcid, p.n_elements, ctypes.c_int32),
                    materials=arr(p.materials, 3 * p.n_domains, ctypes.c_double).reshape(-1, 3),
                    interfaces=arr(p.interfaces, 5 * p.n_interfaces, ctypes.c_int64).reshape(-1, 5))

    def close(self):
        if getattr(self, "c", None):
            load_library().tdbem_case_destroy(self.c)
            self.c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MultiDomainSolver:
    """One multi-domain model resident on one GPU."""

    @classmethod
    def from_case_files(cls, files: "CaseFiles", precision: str = "fp64", device: int = 0):
        """A solver for a case read from reference input files."""
        self = cls.__new__(cls)
        self.case = None
        self.E, self.nstep, self.n_loads = files.n_elements, files.n_steps, files.n_loads
        pr = _Problem.from_buffer_copy(files.problem)
        pr.precision = PRECISION[precision]
        self._files = files
        h = ctypes.c_void_p()
        _check(load_library().tdbem_md_create(ctypes.byref(pr), device, ctypes.byref(h)))
        self.h = h
        self.device = device
        return self

    def __init__(self, case, precision: str = "fp64", tol: Optional[float] = None, restart: Optional[int] = None,
                 max_leaf: Optional[int] = None, max_length: float = 1000.0, n_loads: int = 1, device: int = 0):
        L = load_library()
        m = case.mesh
        self.case = case
        self.E = case.n_elements
        self.nstep = case.nstep
        self.n_loads = n_loads
        self._arrays = [np.ascontiguousarray(m.points, dtype=np.float64),
                        np.ascontiguousarray(m.elements, dtype=np.int64),
                        np.ascontiguousarray(case.bcid, dtype=np.int32),
                        np.ascontiguousarray([[x.E, x.nu, x.rho] for x in case.materials], dtype=np.float64),
                        np.ascontiguousarray(m.interfaces, dtype=np.int64).reshape(-1, 5)]
        pts, ele, bc, mats, itf = self._arrays
        c = case.card_material()
        pr = _Problem(len(pts), _ptr(pts), len(ele), _ptr(ele), _ptr(bc), len(mats), _ptr(mats), len(itf),
                      _ptr(itf), c.E, c.nu, c.rho, case.beta, case.gap, case.nstep,
                      restart or case.iterations, case.error if tol is None else tol,
                      max_leaf or case.max_leaf, max_length, PRECISION[precision], n_loads)
        h = ctypes.c_void_p()
        _check(L.tdbem_md_create(ctypes.byref(pr), device, ctypes.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            load_library().tdbem_md_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def assemble(self, stream: int = 0):
        _check(load_library().tdbem_md_assemble(self.h, stream or None))

    def load_matrices(self, A, KnownM, mts, mgs, stream: int = 0):
        """A, KnownM: (row_ptr, col, val[nnz, 9]); mts, mgs: lists of the same for k = 1..K."""
        def c32(a):
            return np.ascontiguousarray(a, dtype=np.int32)

        def f64(a):
            return np.ascontiguousarray(a, dtype=np.float64)

        K = len(mts)
        ar, ac, av = c32(A[0]), c32(A[1]), f64(A[2])
        kr, kc, kv = c32(KnownM[0]), c32(KnownM[1]), f64(KnownM[2])
        if K:
            tr = c32(np.concatenate([m[0] for m in mts])); tc = c32(np.concatenate([m[1] for m in mts]))
            tv = f64(np.concatenate([np.reshape(m[2], (-1, 9)) for m in mts]))
            gr = c32(np.concatenate([m[0] for m in mgs])); gc = c32(np.concatenate([m[1] for m in mgs]))
            gv = f64(np.concatenate([np.reshape(m[2], (-1, 9)) for m in mgs]))
        else:
            tr = tc = gr = gc = np.zeros(1, np.int32)
            tv = gv = np.zeros((1, 9))
        self._keep_loaded = (ar, ac, av, kr, kc, kv, tr, tc, tv, gr, gc, gv)
        _check(load_library().tdbem_md_load_matrices(self.h, _ptr(ar), _ptr(ac), _ptr(av), _ptr(kr), _ptr(kc),
                                                     _ptr(kv), K, _ptr(tr), _ptr(tc), _ptr(tv), _ptr(gr),
                                                     _ptr(gc), _ptr(gv), stream or None))

    def set_record(self, on: bool = True):
        _check(load_library().tdbem_md_set_record(self.h, 1 if on else 0))

    def march(self, known, raise_on_failure: bool = True):
        """known: (R, NStep+1, E, 3) or (NStep+1, E, 3) -> (bd_lu, bd_lt, report) of the same shape."""
        known = np.asarray(known, dtype=np.float64)
        squeeze = known.ndim == 3
        k4 = np.ascontiguousarray(known[None] if squeeze else known)
        lu = np.zeros_like(k4)
        lt = np.zeros_like(k4)
        rep = Report()
        st = load_library().tdbem_md_march(self.h, _ptr(k4), _ptr(lu), _ptr(lt), ctypes.byref(rep), None)
        if st != 0 and (raise_on_failure or st != 4):
            _check(st)
        if squeeze:
            lu, lt = lu[0], lt[0]
        return lu, lt, rep

    def autotune(self, known, steps: int = 32) -> Tuning:
        """Time launch configurations on the first `steps` steps of `known`
        ((R, NStep+1, E, 3) or (NStep+1, E, 3)) and keep the fastest."""
        k = np.asarray(known, dtype=np.float64)
        k4 = np.ascontiguousarray(k[None] if k.ndim == 3 else k)
        t = Tuning()
        _check(load_library().tdbem_md_autotune(self.h, _ptr(k4), int(steps), ctypes.byref(t), None))
        return t

    def march_device(self, known_ptr: int, out_lu_ptr: int, out_lt_ptr: int, stream: int = 0) -> Report:
        """Device-resident march: raw device pointers (e.g. torch tensor data_ptr())."""
        rep = Report()
        _check(load_library().tdbem_md_march_device(self.h, ctypes.c_void_p(known_ptr), ctypes.c_void_p(out_lu_ptr),
                                                    ctypes.c_void_p(out_lt_ptr), ctypes.byref(rep),
                                                    ctypes.c_void_p(stream) if stream else None))
        return rep

    def solve_noalloc(self, rhs_ptr: int, x_ptr: int, stream: Optional[int] = None, wait: bool = True):
        """One FP64 solve A x = rhs (device pointers, 3E doubles each; rhs in
        equation-row order, x in unknown order) on the library's static
        scratch, without device allocation.  The work runs on `stream`
        (a cudaStream_t as an int); by default on torch's current stream of
        the handle's device, so it is ordered with the torch work that wrote
        rhs and will read x.  With `wait`, returns the (flag, refinements,
        inner iterations) triple and raises on a nonzero flag; otherwise
        returns None once the work is enqueued (a solve that does not
        converge is then not reported)."""
        if stream is None:
            import torch
            stream = torch.cuda.current_stream(self.device).cuda_stream
        flags = np.zeros(3, np.int32) if wait else None
        _check(load_library().tdbem_md_solve_noalloc(self.h, ctypes.c_void_p(rhs_ptr), ctypes.c_void_p(x_ptr),
                                                     _ptr(flags), ctypes.c_void_p(stream) if stream else None))
        return None if flags is None else tuple(int(v) for v in flags)

    def march_vjp(self, cot_lu=None, cot_lt=None):
        """Gradient of <cot_lu, out_lu> + <cot_lt, out_lt> with respect to the
        prescribed values (one-load FP64 handles); shapes (NStep+1, E, 3)."""
        shape = (self.nstep + 1, self.E, 3)
        cl = None if cot_lu is None else np.ascontiguousarray(np.reshape(cot_lu, shape), dtype=np.float64)
        ct = None if cot_lt is None else np.ascontiguousarray(np.reshape(cot_lt, shape), dtype=np.float64)
        grad = np.zeros(shape)
        rep = Report()
        _check(load_library().tdbem_md_march_vjp(self.h, _ptr(cl), _ptr(ct), _ptr(grad), ctypes.byref(rep), None))
        return grad, rep

    def march_forward(self, known):
        """One-load march, (NStep+1, E, 3) -> (bd_lu, bd_lt, report), keeping
        on the device the state march_backward needs."""
        k = np.ascontiguousarray(np.reshape(known, (self.nstep + 1, self.E, 3)), dtype=np.float64)
        lu, lt = np.zeros_like(k), np.zeros_like(k)
        rep = Report()
        _check(load_library().tdbem_md_march_forward(self.h, _ptr(k), _ptr(lu), _ptr(lt), ctypes.byref(rep), None))
        return lu, lt, rep

    def march_backward(self, cot_lu=None, cot_lt=None, materials: bool = True):
        """After march_forward: gradients of <cot_lu, out_lu> + <cot_lt, out_lt>
        with respect to the prescribed values, shape (NStep+1, E, 3), and (with
        `materials`) with respect to each domain's (E, rho), shape (D, 2)."""
        shape = (self.nstep + 1, self.E, 3)
        cl = None if cot_lu is None else np.ascontiguousarray(np.reshape(cot_lu, shape), dtype=np.float64)
        ct = None if cot_lt is None else np.ascontiguousarray(np.reshape(cot_lt, shape), dtype=np.float64)
        grad = np.zeros(shape)
        gm = np.zeros((len(self.case.materials), 2)) if materials else None
        rep = Report()
        _check(load_library().tdbem_md_march_backward(self.h, _ptr(cl), _ptr(ct), _ptr(grad), _ptr(gm),
                                                      ctypes.byref(rep), None))
        return grad, gm, rep

    def save_matrices(self, path: str):
        """Write the assembled matrices to a cache file."""
        _check(load_library().tdbem_md_save_matrices(self.h, os.fsencode(path)))

    def load_matrix_cache(self, path: str, stream: int = 0):
        """Load matrices saved by save_matrices for the same model instead of assembling."""
        _check(load_library().tdbem_md_load_matrix_cache(self.h, os.fsencode(path), stream or None))

    def write_validation(self, directory: str, lu, lt, report: Report, load: int = 0):
        """validation_state.csv and validation_metrics.txt of one load case of
        a march (lu, lt as march() returned them), in the reference's formats."""
        lu4 = np.ascontiguousarray(lu[None] if np.ndim(lu) == 3 else lu, dtype=np.float64)
        lt4 = np.ascontiguousarray(lt[None] if np.ndim(lt) == 3 else lt, dtype=np.float64)
        _check(load_library().tdbem_md_write_validation(self.h, os.fsencode(directory), load, _ptr(lu4), _ptr(lt4),
                                                         ctypes.byref(report)))

    def write_rhs_diagnostics(self, directory: str, report: Report):
        """rhs_breakdown.csv and residual_probe.csv of the last march (load
        case 0), which must have been recorded (set_record(True) before
        march(), or march_forward())."""
        _check(load_library().tdbem_md_write_rhs_diagnostics(self.h, os.fsencode(directory), ctypes.byref(report)))

    def step_record(self):
        n = self.nstep
        rhs = np.zeros((n, 3 * self.E))
        x = np.zeros((n, 3 * self.E))
        flags = np.zeros((n, 3), np.int32)
        _check(load_library().tdbem_md_step_record(self.h, _ptr(rhs), _ptr(x), _ptr(flags)))
        return rhs, x, flags

    def export_matrix(self, which: str, k: int = 0):
        code = {"A": 0, "KnownM": 1, "MTS": 2, "MGS": 3}[which]
        L = load_library()
        nr, nnz = ctypes.c_int64(), ctypes.c_int64()
        _check(L.tdbem_md_export_matrix(self.h, code, k, ctypes.byref(nr), ctypes.byref(nnz), None, None, None))
        rp = np.zeros(nr.value + 1, np.int32)
        col = np.zeros(max(nnz.value, 1), np.int32)
        val = np.zeros((max(nnz.value, 1), 9))
        _check(L.tdbem_md_export_matrix(self.h, code, k, ctypes.byref(nr), ctypes.byref(nnz), _ptr(rp), _ptr(col),
                                        _ptr(val)))
        return rp, col[:nnz.value], val[:nnz.value]

    def geometry(self):
        E = self.E
        g = dict(coordcoef=np.zeros((E, 3, 8)), center=np.zeros((E, 3)), radius=np.zeros(E), radius_pw=np.zeros(E),
                 transmat=np.zeros((E, 9)), on_u1=np.zeros((E, 9)), on_t1=np.zeros((E, 9)), on_t2=np.zeros((E, 9)))
        _check(load_library().tdbem_md_geometry(self.h, *(_ptr(g[k]) for k in ("coordcoef", "center", "radius",
                                                                             "radius_pw", "transmat", "on_u1",
                                                                             "on_t1", "on_t2"))))
        return g

    def info(self):
        dt = ctypes.c_double()
        v = [ctypes.c_int64() for _ in range(4)]
        _check(load_library().tdbem_md_info(self.h, ctypes.byref(dt), *(ctypes.byref(x) for x in v)))
        return dict(dt=dt.value, n_unknown=v[0].value, n_known=v[1].value, n_history=v[2].value,
                    n_leaves=v[3].value)

    def precond_layout(self):
        inf = self.info()
        rep = np.zeros(self.E, np.int64)
        lb = np.zeros(inf["n_leaves"], np.int64)
        lc = np.zeros(inf["n_leaves"], np.int64)
        _check(load_library().tdbem_md_precond_layout(self.h, _ptr(rep), _ptr(lb), _ptr(lc)))
        return rep, lb, lc


def DynaGMRESSolverMultiDomainCCSR(case, bd_lu, iterations: int, error: float, maxleafpointnum: int, NStep: int,
                                   MaxLength: float = 1000.0, precision: str = "fp64", device: int = 0):
    """Mirror of the reference solver call.

    bd_lu: (NStep+1, E, 3) element-local prescribed values (bd[n].lu).
    Returns (ret, bd_lu_out, bd_lt_out, report): ret is 1 when every step
    converged and -1 on the first non-converged step (the march stops there,
    later steps stay zero) or on invalid input, as the reference returns.
    """
    import dataclasses
    c = dataclasses.replace(case, nstep=NStep, iterations=iterations, error=error, max_leaf=maxleafpointnum)
    try:
        s = MultiDomainSolver(c, precision=precision, max_length=MaxLength, device=device)
        s.assemble()
        lu, lt, rep = s.march(np.asarray(bd_lu)[: NStep + 1], raise_on_failure=False)
        s.close()
    except TdbemError:
        return -1, None, None, None
    return (1 if rep.failed_step == 0 else -1), lu, lt, rep


def march_many(solvers, known_ptrs, out_lu_ptrs, out_lt_ptrs, stream: int = 0):
    """March several solvers' models together (tdbem_md_march_many) on device
    buffers (raw pointers, one per solver); returns the reports."""
    n = len(solvers)
    hs = (ctypes.c_void_p * n)(*[s.h.value for s in solvers])
    kp = (ctypes.c_void_p * n)(*known_ptrs)
    up = (ctypes.c_void_p * n)(*out_lu_ptrs)
    tp = (ctypes.c_void_p * n)(*out_lt_ptrs)
    reps = (Report * n)()
    _check(load_library().tdbem_md_march_many(hs, n, kp, up, tp, reps, ctypes.c_void_p(stream) if stream else None))
    return list(reps)


def march_function():
    """A torch.autograd.Function over the FP64 one-load march:
    apply(solver, known[, materials]) -> (out_lu, out_lt) as torch float64
    tensors on known's device (CPU, or CUDA without host copies).  Its
    backward is the adjoint march (the forward/backward pair of the C ABI).
    materials, if given, is a (D, 2) tensor of each domain's (E, rho), which
    must equal the solver's; it receives dJ/dE and dJ/drho."""
    import torch

    def ptr(t):
        return None if t is None else ctypes.c_void_p(t.data_ptr())

    class TdbemMarch(torch.autograd.Function):
        @staticmethod
        def forward(ctx, solver, known, *rest):
            ctx.solver = solver
            ctx.n_rest = len(rest)
            materials = rest[0] if rest else None
            ctx.with_materials = materials is not None
            ctx.mat_device = materials.device if materials is not None else None
            if materials is not None:
                want = np.array([[m.E, m.rho] for m in solver.case.materials])
                if not np.array_equal(materials.detach().cpu().numpy(), want):
                    raise ValueError("materials differ from the solver's; build a solver for them")
            ctx.cuda = known.is_cuda
            if known.is_cuda:
                # device buffers go to the C ABI as they are, on torch's stream
                k = known.detach().to(torch.float64).contiguous()
                lu, lt = torch.zeros_like(k), torch.zeros_like(k)
                rep = Report()
                ctx.stream = torch.cuda.current_stream(k.device).cuda_stream
                _check(load_library().tdbem_md_march_forward(solver.h, ptr(k), ptr(lu), ptr(lt), ctypes.byref(rep),
                                                              ctypes.c_void_p(ctx.stream)))
                return lu, lt
            lu, lt, _ = solver.march_forward(known.detach().cpu().numpy())
            return torch.from_numpy(lu), torch.from_numpy(lt)

        @staticmethod
        def backward(ctx, g_lu, g_lt):
            s = ctx.solver
            if ctx.cuda:
                gl = None if g_lu is None else g_lu.detach().to(torch.float64).contiguous()
                gt = None if g_lt is None else g_lt.detach().to(torch.float64).contiguous()
                ref = gl if gl is not None else gt
                grad = torch.zeros((s.nstep + 1, s.E, 3), dtype=torch.float64, device=ref.device)
                gm = np.zeros((len(s.case.materials), 2)) if ctx.with_materials else None
                rep = Report()
                _check(load_library().tdbem_md_march_backward(s.h, ptr(gl), ptr(gt), ptr(grad), _ptr(gm),
                                                              ctypes.byref(rep), ctypes.c_void_p(ctx.stream)))
            else:
                g, gm, _ = s.march_backward(None if g_lu is None else g_lu.detach().cpu().numpy(),
                                            None if g_lt is None else g_lt.detach().cpu().numpy(),
                                            materials=ctx.with_materials)
                grad = torch.from_numpy(g)
            tail = [torch.from_numpy(gm).to(ctx.mat_device) if gm is not None else None] if ctx.n_rest else []
            return (None, grad, *tail)

    return TdbemMarch
