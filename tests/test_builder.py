"""Block builder rules: the C oracle's restatement against the reference's own
MultiDomainCCSRBuilder (oracle/_ref/dbem_ref_builder, the unchanged
reference objects), CPU.

AddBlock (DBEM1/multidomain.cpp:1120-1144) skips a block whose sign is 0,
that is all zero, whose largest entry is at most 1e-14, or that holds a
non-finite value (:1126-1133, with a message); it adds sign * block^T
(column-major in, row-major stored) to the (row, column) entry in call order
and erases the entry when the sum falls to at most 1e-14.  Build emits rows
in order, columns ascending.  The call list below plants every case among
seeded random blocks; both builders must store the same structure and the
same bits.
"""
import ctypes
import os
import shutil
import struct
import subprocess
import tempfile

import numpy as np
import pytest

from oracle_lib import _ptr, lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BUILDER = os.path.join(REPO, "oracle", "_ref", "dbem_ref_builder")


def _calls(seed=7, rows=12, cols=9, n=400):
    rng = np.random.default_rng(seed)
    r = rng.integers(0, rows, n)
    c = rng.integers(0, cols, n)
    sg = rng.choice([-1.0, 1.0, 0.5], n)
    b = rng.normal(size=(n, 9)) * 10.0 ** rng.uniform(-3, 1, (n, 1))
    planted = {}
    # non-finite values: skipped (the reference prints a message)
    b[5, 3] = np.nan
    b[17, 0] = np.inf
    b[29, 8] = -np.inf
    # all zero, and largest entry 1e-15: skipped
    b[41] = 0.0
    b[53] = 1e-15
    # sign 0: skipped
    sg[65] = 0.0
    # out of range: skipped
    r[77] = rows
    c[89] = -1
    # a block added and then taken away again (sum <= 1e-14): erased
    r[101], c[101], sg[101] = 3, 4, 1.0
    r[102], c[102], sg[102] = 3, 4, -1.0
    b[102] = b[101]
    # a lone NaN block at an otherwise empty (row, column)
    r[113], c[113] = rows - 1, cols - 1
    b[113, 4] = np.nan
    mask = (r == rows - 1) & (c == cols - 1)
    mask[113] = False
    r[mask] = 0
    planted.update(nan_cell=(rows - 1, cols - 1), cancel_cell=(3, 4))
    cancel = (r == 3) & (c == 4)
    cancel[[101, 102]] = False
    r[cancel] = 2
    return rows, cols, r.astype(np.int64), c.astype(np.int64), sg, b, planted


def _oracle(rows, cols, r, c, sg, b):
    L = lib()
    L.orc_builder_replay.restype = ctypes.c_int64
    L.orc_builder_replay.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64] + [ctypes.c_void_p] * 7
    b = np.ascontiguousarray(b)
    nnz = L.orc_builder_replay(rows, cols, len(r), _ptr(r), _ptr(c), _ptr(sg), _ptr(b), None, None, None)
    rp = np.zeros(rows + 1, np.int32)
    col = np.zeros(max(nnz, 1), np.int32)
    val = np.zeros((max(nnz, 1), 9))
    L.orc_builder_replay(rows, cols, len(r), _ptr(r), _ptr(c), _ptr(sg), _ptr(b), _ptr(rp), _ptr(col), _ptr(val))
    return rp, col[:nnz], val[:nnz]


def _reference(rows, cols, r, c, sg, b):
    with tempfile.TemporaryDirectory() as tmp:
        # the reference reads its Gauss tables from the working directory
        # while its objects are initialised
        for t in ("gaussposition", "gaussweight"):
            shutil.copy(os.path.join(REPO, "oracle", "_ref", t), tmp)
        inp, out = os.path.join(tmp, "calls.bin"), os.path.join(tmp, "out.bin")
        with open(inp, "wb") as f:
            f.write(struct.pack("<3q", rows, cols, len(r)))
            for i in range(len(r)):
                f.write(struct.pack("<2q", int(r[i]), int(c[i])))
                f.write(struct.pack("<d", float(sg[i])))
                f.write(np.ascontiguousarray(b[i], dtype="<f8").tobytes())
        res = subprocess.run([REF_BUILDER, inp, out], cwd=tmp, capture_output=True, text=True, timeout=60)
        assert res.returncode == 0, res.stderr
        data = open(out, "rb").read()
    n_rows, nnz = struct.unpack_from("<2q", data, 0)
    o = 16
    rp = np.frombuffer(data, "<i4", n_rows + 1, o)
    o += 4 * (n_rows + 1)
    col = np.frombuffer(data, "<i4", nnz, o)
    o += 4 * nnz
    val = np.frombuffer(data, "<f8", 9 * nnz, o).reshape(nnz, 9)
    return rp, col, val, res.stdout


def test_oracle_builder_rules():
    rows, cols, r, c, sg, b, planted = _calls()
    rp, col, val = _oracle(rows, cols, r, c, sg, b)
    assert np.all(np.isfinite(val))
    cells = {(i, int(col[j])) for i in range(rows) for j in range(rp[i], rp[i + 1])}
    assert planted["nan_cell"] not in cells and planted["cancel_cell"] not in cells
    for i in range(rows):
        assert np.all(np.diff(col[rp[i]:rp[i + 1]]) > 0)
    assert np.all(np.max(np.abs(val), axis=1) > 1e-14)
    # one kept entry recomputed by hand: sum of sign * block^T over its calls
    i0, c0 = 0, int(col[rp[0]])
    acc = np.zeros((3, 3))
    for k in range(len(r)):
        if r[k] == i0 and c[k] == c0 and sg[k] != 0.0 and np.all(np.isfinite(b[k])) and np.max(np.abs(b[k])) > 1e-14:
            acc += sg[k] * b[k].reshape(3, 3).T  # column-major in, row-major stored
    assert np.array_equal(val[rp[0]].reshape(3, 3), acc)


@pytest.mark.skipif(not os.path.exists(REF_BUILDER), reason="reference builder harness not built (needs the "
                    "reference sources)")
def test_oracle_builder_equals_reference_builder():
    rows, cols, r, c, sg, b, _ = _calls()
    rp, col, val = _oracle(rows, cols, r, c, sg, b)
    rp2, col2, val2, out = _reference(rows, cols, r, c, sg, b)
    assert np.array_equal(rp, rp2) and np.array_equal(col, col2)
    assert np.array_equal(val, val2)  # same bits: same accumulation order
    # the reference reports each non-finite block it skips: the NaN, +inf and
    # -inf planted among the random calls and the lone NaN cell
    assert out.count("skipped non-finite block") == 4


REF_CCSR = os.path.join(REPO, "oracle", "_ref", "dbem_ref_ccsr")


def ccsr_section(rp, col, val):
    """One matrix in the cache file's layout: int64 n, int64 nnz, int32
    row_ptr[n + 1], int32 col[nnz], double val[nnz][9]."""
    rp = np.asarray(rp, "<i4")
    return (struct.pack("<2q", len(rp) - 1, len(col)) + rp.tobytes() + np.asarray(col, "<i4").tobytes()
            + np.ascontiguousarray(val, "<f8").tobytes())


def reference_rewrite(path, offset):
    """The matrix at `offset` of `path` read by the reference's
    CCSRMat::ReadBinary and written back by CCSRMat::WriteBinary
    (DBEM1/mat_vec.cpp:1690-1730); returns (bytes, n, nnz)."""
    with tempfile.TemporaryDirectory() as tmp:
        for t in ("gaussposition", "gaussweight"):
            shutil.copy(os.path.join(REPO, "oracle", "_ref", t), tmp)
        out = os.path.join(tmp, "out.bin")
        res = subprocess.run([REF_CCSR, path, str(offset), out], cwd=tmp, capture_output=True, text=True,
                             timeout=60)
        assert res.returncode == 0, (res.returncode, res.stderr)
        n, nnz = map(int, res.stdout.split())
        return open(out, "rb").read(), n, nnz


@pytest.mark.skipif(not os.path.exists(REF_CCSR), reason="reference CCSR harness not built (needs the reference "
                    "sources)")
def test_cache_matrix_layout_is_the_references(tmp_path):
    """A matrix section laid out as the library's cache writes it (after a
    leading pad, as a section sits inside the file) is read and written back
    unchanged by the reference's own CCSRMat binary routines."""
    rows, cols, r, c, sg, b, _ = _calls()
    rp, col, val = _oracle(rows, cols, r, c, sg, b)
    sec = ccsr_section(rp, col, val)
    path = str(tmp_path / "section.bin")
    with open(path, "wb") as f:
        f.write(b"\0" * 40 + sec)
    again, n, nnz = reference_rewrite(path, 40)
    assert (n, nnz) == (rows, len(col))
    assert again == sec
