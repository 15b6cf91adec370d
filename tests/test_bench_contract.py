"""bench.py's CPU-side pieces: the committed ncu summary it reads the
DRAM-to-algorithmic traffic ratio from, the measured-peak fallback, and
the default workload of its command line."""
import importlib.util
import os

from conftest import REPO


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_traffic_ratio_from_committed_profile():
    b = _bench()
    r = b.profile_traffic_ratio()
    assert r is not None and 0.9 < r < 2.0


def test_peak_fallback_is_labelled():
    b = _bench()
    peak, kind = b.measured_hbm_peak()
    assert peak > 1000.0 and kind in ("measured", "fallback")


def test_default_arguments():
    b = _bench()
    a = b.parse_args([])
    assert a.gpus == 1 and a.warmup >= 3 and a.steps >= 1
