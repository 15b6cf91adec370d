"""Build the CUDA library (csrc/*.cu -> libtdbem_b200.so, in-tree) for sm_100a.

Each translation unit is compiled to its own object under csrc/_build/ (in
parallel, and only when the unit or a header it may include is newer than
its object), then the objects are linked into the shared library.
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(CSRC, "_build")
LIB = os.path.join(PKG, "libtdbem_b200.so")
HDR = os.path.join(os.path.dirname(PKG), "include", "tdbem.h")
SOURCES = ["capi.cu", "assemble.cu", "march.cu", "runs.cu", "inputs.cu", "adjoint.cu", "diag.cu"]
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
         "--expt-relaxed-constexpr"]


def nvcc_path():
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if p and os.path.exists(p):
            return p
    raise RuntimeError("nvcc not found")


def _sources():
    return [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def _headers_mtime():
    t = os.path.getmtime(HDR) if os.path.exists(HDR) else 0.0
    for f in os.listdir(CSRC):
        if f.endswith((".cuh", ".h")):
            t = max(t, os.path.getmtime(os.path.join(CSRC, f)))
    return t


def _obj(src):
    return os.path.join(OBJ, src[:-3] + ".o")


def _stale(src, hdr_t):
    o = _obj(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    return os.path.getmtime(os.path.join(CSRC, src)) > t or hdr_t > t


def needs_build():
    if not os.path.exists(LIB):
        return True
    hdr_t = _headers_mtime()
    t = os.path.getmtime(LIB)
    return any(_stale(s, hdr_t) or os.path.getmtime(_obj(s)) > t for s in _sources())


def _compile(src, verbose):
    cmd = [nvcc_path()] + FLAGS + (["-Xptxas", "-v"] if verbose else []) + \
        ["-c", os.path.join(CSRC, src), "-o", _obj(src) + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n" + r.stdout + r.stderr)
    os.replace(_obj(src) + ".tmp", _obj(src))
    return r.stdout + r.stderr


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    hdr_t = _headers_mtime()
    todo = [s for s in _sources() if force or verbose or _stale(s, hdr_t)]
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        logs = list(ex.map(lambda s: _compile(s, verbose), todo))
    if verbose:
        sys.stderr.write("".join(logs))
    cmd = [nvcc_path()] + FLAGS + ["-shared", "-o", LIB + ".tmp"] + [_obj(s) for s in _sources()]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
