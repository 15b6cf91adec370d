"""Run the reference solver build (oracle/_ref/dbem_ref_dump) on a case and
read its records (test infrastructure, the checker only).

The executable is the reference compiled unchanged from its sources by
oracle/Makefile, linked with the recording wrapper oracle/ref_dump.cpp.  It
needs the two Gauss-table data files that the Makefile copies next to it.
"""
import os
import shutil
import subprocess
import tempfile

from refdump import read_dump

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(REPO, "oracle", "_ref")
DUMP_EXE = os.path.join(REF, "dbem_ref_dump")


def available():
    return all(os.path.exists(os.path.join(REF, f)) for f in ("dbem_ref_dump", "gaussposition", "gaussweight"))


def run_case(case, error=None, threads=None, matrices=False, timeout=1800):
    """Write the case's reference inputs (load case 0), run the recording
    reference build and return its records (see oracle/ref_dump.cpp):
    per-step rhs{s}, x{s}, flag{s}, bd_lu / bd_lt [NStep+1][3E], meta, ...
    With matrices=False the serial re-assembly of the matrices is skipped."""
    from tdbem import cases
    threads = threads or os.cpu_count() or 1
    with tempfile.TemporaryDirectory(prefix="tdbem_ref_") as tmp:
        cases.write_reference_inputs(case, tmp, threads=threads, error=error)
        for t in ("gaussposition", "gaussweight"):
            shutil.copy(os.path.join(REF, t), tmp)
        dump = os.path.join(tmp, "dump.bin")
        env = dict(os.environ, TDBEM_DUMP=dump, DBEM_VALIDATION_OUTPUT="0", OMP_NUM_THREADS=str(threads),
                   TDBEM_DUMP_MATRICES="1" if matrices else "0")
        with open(os.path.join(tmp, "run.log"), "w") as log:
            rc = subprocess.run([DUMP_EXE], cwd=tmp, env=env, stdout=log, stderr=subprocess.STDOUT,
                                timeout=timeout).returncode
        if not os.path.exists(dump):
            tail = open(os.path.join(tmp, "run.log"), errors="replace").read()[-2000:]
            raise RuntimeError(f"reference run wrote no records (rc={rc}):\n{tail}")
        return read_dump(dump)
