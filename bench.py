#!/usr/bin/env python
"""Benchmark of the multi-domain TDBEM time march on B200.

Workload: the heterogeneous 8-domain bar (1x1x8, 8x8 elements per face,
3072 constant elements, E alternating 20/80, nu 0.25, rho 20, beta 0.6,
400 time steps, seeded Ricker end traction), synthetic inputs generated by
tdbem.cases.config_bar8.  A bench step is one full march of the 400 time
steps for the load cases of one model (history right-hand side, GMRES and
write-back every time step), with the matrices assembled once beforehand.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm reports, as `value`, the FP32-history / FP64-refined solver's
time steps per second (load-case time steps / s, whole job), next to the
plain FP64 GPU path, the roofline of the history right-hand-side kernel, an
end-to-end figure through the C ABI with host buffers, and a bounded sample
of the reference CPU solver.  Multi-GPU runs are independent replicas (one
model per GPU, no collective on the data path): scaling "weak".

The reference arm (--impl reference) times the unchanged reference solver
(oracle/_ref/dbem_ref, built from the reference sources) on the same bar,
with all host cores, on the first W+K time steps.
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "parallel3.0_omp_multidomin_1node_b200")
sys.path.insert(0, PKG)

METRIC = "timesteps/s mixed-prec+batched vs FP64 GPU at ≤1e-6 rel err; history SpMV GB/s"


def workload(args):
    if args.workload == "box":
        return (f"box: 4x4x4 block in 4 layers along x, 24x24 elements on the layer faces, 6 through each layer, "
                f"6912 elements, {args.nstep} steps, {args.loads} seeded Ricker loads on the x+ face")
    n = args.n
    return (f"bar8: 1x1x8 bar, 8 unit-cube domains, {n}x{n} per face, {48 * n * n} elements, {args.nstep} steps, "
            f"{args.loads} seeded end-load cases (Heaviside / Ricker)")


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nstep", type=int, default=400, help="time steps per march")
    ap.add_argument("--n", type=int, default=8, help="elements per face edge")
    ap.add_argument("--loads", type=int, default=32, help="load cases marched together (headline mode)")
    ap.add_argument("--tol", type=float, default=1e-9, help="GMRES relative tolerance")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["bar8", "box"], default="bar8",
                    help="bar8: the headline 3072-element bar; box: the layered block (6912 elements, 1000 steps, "
                         "8 loads; use --nstep 1000 --loads 8 --no-cpu-baseline)")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------
# reference CPU solver (oracle/_ref/dbem_ref): run and time march steps
# history steps of the bar that carry blocks (about 39 at 8x8 per face):
# reference steps after this many apply the full convolution
REF_STEADY = 40


def run_reference(nstep, n, threads, tol):
    """Run the reference on the bar with nstep steps at GMRES tolerance tol;
    return per-step start times (seconds, monotonic), the end time of the
    march and the process start time."""
    from tdbem import cases
    exe = os.path.join(REPO, "oracle", "_ref", "dbem_ref")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    case = cases.config_bar8(nstep=nstep, n=n, error=tol)
    tmp = tempfile.mkdtemp(prefix="tdbem_ref_")
    try:
        cdir = os.path.join(tmp, "case")
        os.makedirs(cdir)
        cases.write_reference_inputs(case, cdir, threads=threads)
        for t in ("gaussposition", "gaussweight"):
            shutil.copy(os.path.join(REPO, "oracle", "_ref", t), cdir)
        env = dict(os.environ, DBEM_VALIDATION_OUTPUT="0", OMP_NUM_THREADS=str(threads))
        cmd = ["stdbuf", "-oL", exe] if shutil.which("stdbuf") else [exe]
        t_start = time.monotonic()
        p = subprocess.Popen(cmd, cwd=cdir, env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                             errors="replace")
        step_t = {}
        t_end = None
        for line in p.stdout:
            now = time.monotonic()
            if line.startswith("MultiDomain GMRES Solver: Step "):
                step_t[int(line.split("Step ")[1].split(".")[0])] = now
            elif line.startswith("MultiDomain performance:"):
                t_end = now
        p.wait()
        if t_end is None or len(step_t) < nstep:
            raise RuntimeError(f"reference run ended early (rc={p.returncode}, steps={len(step_t)})")
        return step_t, t_end, t_start
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def reference_rate(first, last, nstep, n, threads, tol):
    """(time steps/s over steps first..last, their seconds, the reference's
    set-up seconds: process start to its first step, i.e. input reading,
    geometry, Step0 and history assembly and the preconditioner)."""
    step_t, t_end, t_start = run_reference(nstep, n, threads, tol)
    t1 = step_t[first]
    t2 = step_t[last + 1] if last + 1 in step_t else t_end
    return (last - first + 1) / (t2 - t1), t2 - t1, step_t[1] - t_start


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    # the first REF_STEADY steps (>= warmup) fill the history; the timed
    # steps after them apply every non-empty history step, like the bulk of
    # the 400-step march
    timed = max(1, args.steps)
    first = max(REF_STEADY, args.warmup) + 1
    nstep = first + timed - 1
    sample = (f"reference solver on the same bar, one load case, GMRES tolerance {args.tol:g} (as the GPU arm), "
              f"time steps {first}..{nstep} of a {nstep}-step run (every non-empty history step active), "
              f"assembly excluded")
    try:
        rate, secs, setup = reference_rate(first, nstep, nstep, args.n, threads, args.tol)
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": f"reference run failed: {e}"}))
        return 0
    line = {"metric": METRIC, "value": rate, "unit": "timesteps/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": timed, "warmup": args.warmup, "ms_per_step": 1e3 * secs / max(timed, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": workload(args), "load_cases": 1, "threads": threads,
                                            "gmres_tol": args.tol},
            "assembly_s": setup,
            "cpu_baseline": {"value": rate, "unit": "timesteps/s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": rate, "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during timing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_hbm_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


def profile_traffic_ratio():
    """DRAM bytes per algorithmic byte of the 32-load two-step history pass,
    from the committed ncu summary (line 'dram_to_algorithmic=' in
    profiles/bulk_steps_kernel_bar8_32loads_mixed.txt); None when absent."""
    p = os.path.join(REPO, "profiles", "bulk_steps_kernel_bar8_32loads_mixed.txt")
    try:
        for ln in open(p):
            if ln.startswith("dram_to_algorithmic="):
                return float(ln.split("=")[1])
    except OSError:
        pass
    return None


# L2 read peak of the B200s here: ncu's sustained peak of L2 sector
# throughput from tex requests (lts__t_sectors_srcunit_tex, 2 sectors of 32 B
# per clock and slice; 722.5 G sectors/s at the 1.96 GHz L2 clock) in a
# capture of the history kernel.  Copies and reductions through torch reach
# only 3.7-6.7 TB/s, less than the history pass's own gather, so they are not
# a ceiling.
L2_PEAK_GBS = 722.5 * 32


def replica_seeds(rank):
    """Load seeds of one replica: every rank marches its own load cases."""
    return 2 + rank, 4 + rank


def reduce_max(v, dist, device):
    """Max of a per-rank value over the process group (the timed region's
    duration is the slowest rank's)."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def ours_arm(args):
    import ctypes

    import numpy as np
    import torch
    from tdbem import api, cases

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        return reduce_max(v, dist, "cuda")

    R = args.loads
    N = args.nstep
    # GMRES tolerance tight enough that the FP64 and mixed paths can be
    # compared at the 1e-6 level (the card's 1e-5 bounds both only to ~1e-5)
    seed_single, seed_batch = replica_seeds(rank)
    if args.workload == "box":
        import dataclasses
        batch = cases.config_layered_box(nstep=N, loads=R, seed=7 + rank, error=args.tol)
        single = dataclasses.replace(batch, known=np.ascontiguousarray(batch.known[:1]))
    else:
        single = cases.config_bar8(nstep=N, n=args.n, seed=seed_single, error=args.tol)
        batch = cases.config_bar8_batched(nstep=N, n=args.n, loads=R, seed=seed_batch, error=args.tol)
    stream = torch.cuda.current_stream()
    modes = [("fp64", 1, single), ("mixed", 1, single), ("fp64", R, batch), ("mixed", R, batch)]
    results = {}
    for prec, r, case in modes:
        s = api.MultiDomainSolver(case, precision=prec, n_loads=r, device=local)
        t0 = time.perf_counter()
        s.assemble()
        torch.cuda.synchronize()
        asm = time.perf_counter() - t0
        known_d = torch.from_numpy(np.ascontiguousarray(case.known[:r])).to("cuda")
        out_lu = torch.zeros_like(known_d)
        out_lt = torch.zeros_like(known_d)
        for _ in range(args.warmup):
            s.march_device(known_d.data_ptr(), out_lu.data_ptr(), out_lt.data_ptr(), stream.cuda_stream)
        headline = (prec, r) == ("mixed", R)
        sampler = ClockSampler(local) if headline else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        reps = []
        for _ in range(args.steps):
            reps.append(s.march_device(known_d.data_ptr(), out_lu.data_ptr(), out_lt.data_ptr(), stream.cuda_stream))
        ev1.record(stream)
        barrier()
        ms = max_over_ranks(ev0.elapsed_time(ev1))
        clocks = sampler.stop() if sampler else None
        results[(prec, r)] = dict(solver=s, ms=ms, asm=asm, rep=reps[-1], loads=r, case=case,
                                  rhs_bytes=sum(x.rhs_bytes for x in reps), ms_rhs=sum(x.ms_rhs for x in reps),
                                  ms_gmres=sum(x.ms_gmres for x in reps), clocks=clocks,
                                  lu=out_lu.cpu().numpy() if prec == "fp64" and r == R or headline else None)
        if not headline:
            s.close()
        del known_d, out_lu, out_lt
        torch.cuda.empty_cache()

    def rate(key):
        res = results[key]
        return world * args.steps * N * res["loads"] / (res["ms"] / 1e3)

    hd = results[("mixed", R)]
    ref = results[("fp64", R)]
    # per-step max relative displacement error of the mixed path vs FP64 (all loads)
    rel = 0.0
    for r in range(R):
        u64 = ref["lu"][r].reshape(N + 1, -1)
        u32 = hd["lu"][r].reshape(N + 1, -1)
        scale = np.maximum(np.max(np.abs(u64), axis=1), 1e-300)
        rel = max(rel, float(np.max(np.max(np.abs(u32 - u64), axis=1)[1:] / scale[1:])))

    # end to end through the C ABI with pinned host buffers (inputs in, all
    # boundary values out, every march)
    L = api.load_library()
    s = hd["solver"]
    kh = torch.from_numpy(np.ascontiguousarray(batch.known[:R])).pin_memory()
    lu_h = torch.zeros_like(kh).pin_memory()
    lt_h = torch.zeros_like(kh).pin_memory()
    rep = api.Report()

    def call():
        st = L.tdbem_md_march(s.h, ctypes.c_void_p(kh.data_ptr()), ctypes.c_void_p(lu_h.data_ptr()),
                              ctypes.c_void_p(lt_h.data_ptr()), ctypes.byref(rep), ctypes.c_void_p(stream.cuda_stream))
        if st != 0:
            raise RuntimeError(L.tdbem_last_error().decode())

    for _ in range(max(1, args.warmup // 2)):
        call()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        call()
    e1.record(stream)
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1))

    # The history pass timed alone, for the roofline: one more march of the
    # same handle with the history passes run after each step's GMRES instead
    # of beside it (TDBEM_OVERLAP=0), so the events around them bracket those
    # kernels only.  Outside the timed region; same results.
    os.environ["TDBEM_OVERLAP"] = "0"
    try:
        call()
    finally:
        del os.environ["TDBEM_OVERLAP"]
    serial = {"ms": rep.ms_history, "launches": rep.history_launches, "bytes": rep.history_bytes,
              "block_steps": rep.history_block_steps, "vector_loads": rep.history_vector_loads}
    # history passes of one time step launch N - 2 times, of T steps about (N - 2) / T
    steps_per_pass = max(1, round((N - 2) / max(serial["launches"], 1)))
    l2_peak = L2_PEAK_GBS

    value = rate(("mixed", R))
    peak, peak_kind = measured_hbm_peak()
    achieved = serial["bytes"] / (serial["ms"] / 1e3) / 1e9
    # FP64 history vectors gathered from L2: 3 components x R cases per load;
    # 9 x 2 flops per block, time step and case
    l2_bytes = serial["vector_loads"] * 3 * R * 8
    l2_achieved = l2_bytes / (serial["ms"] / 1e3) / 1e9
    fp64_tflops = serial["block_steps"] * 18 * R / (serial["ms"] / 1e3) / 1e12
    fp1 = results[("fp64", 1)]
    mx1 = results[("mixed", 1)]
    launches_hist = serial["launches"]
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "timesteps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": hd["ms"] / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 history blocks + f64 refinement",
        "data": "synthetic",
        "config": {"workload": workload(args), "elements": single.n_elements, "domains": single.mesh.domains, "time_steps": N,
                   "load_cases": R, "precision": "mixed", "gmres_tol": args.tol,
                   "gmres_cluster": hd["rep"].gmres_cluster, "gmres_groups": hd["rep"].gmres_groups,
                   "history_steps": hd["rep"].history_steps,
                   "history_blocks": hd["rep"].history_blocks, "a_blocks": hd["rep"].a_blocks,
                   "l2": "inputs larger than L2 (history blocks %.2f GB FP32)" % (hd["rep"].history_blocks * 40 / 1e9),
                   "value_unit_meaning": "load-case time steps per second, whole job",
                   "parallelism": f"replicas x{world}"},
        "plain_fp64": {"value": rate(("fp64", 1)), "unit": "timesteps/s", "loads": 1,
                       "ms_per_step": fp1["ms"] / args.steps,
                       "rhs_achieved_gbs": fp1["rhs_bytes"] / (fp1["ms_rhs"] / 1e3) / 1e9,
                       "ms_rhs_per_march": fp1["ms_rhs"] / args.steps,
                       "ms_gmres_per_march": fp1["ms_gmres"] / args.steps, "assembly_s": fp1["asm"]},
        "mixed_single_load": {"value": rate(("mixed", 1)), "unit": "timesteps/s", "loads": 1,
                              "rhs_achieved_gbs": mx1["rhs_bytes"] / (mx1["ms_rhs"] / 1e3) / 1e9,
                              "ms_rhs_per_march": mx1["ms_rhs"] / args.steps,
                              "ms_gmres_per_march": mx1["ms_gmres"] / args.steps},
        "fp64_batched": {"value": rate(("fp64", R)), "unit": "timesteps/s", "loads": R},
        "speedup_per_load_vs_plain_fp64": value / rate(("fp64", 1)),
        "max_rel_err_vs_fp64": rel,
        "gmres_inner_per_step": hd["rep"].total_inner / (N * R),
        "gmres_cluster_ms_per_march": hd["ms_gmres"] / args.steps,
        "assembly_s": hd["asm"],
        "roofline": {"bound": "hbm",
                     "kernel": ("bulk_steps_kernel (history steps k >= %d of %d time steps, %d loads)"
                                % (2 * steps_per_pass + 1, steps_per_pass, R) if steps_per_pass > 1
                                else "rhs_kernel (history steps k >= 3 of one time step, %d loads)" % R),
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind,
                     "traffic": (None if profile_traffic_ratio() is None
                                 else profile_traffic_ratio() * serial["bytes"] / launches_hist),
                     "bytes_per_launch": serial["bytes"] / launches_hist,
                     "ms_per_launch": serial["ms"] / launches_hist,
                     "launches_per_march": launches_hist,
                     "timing": "one extra march with the history passes run after each step's GMRES instead of "
                               "beside it; CUDA events around those launches only",
                     "l2_state": {"achieved": l2_achieved, "peak": l2_peak, "unit": "GB/s",
                                  "frac": l2_achieved / l2_peak,
                                  "peak_kind": "ncu sustained peak of L2 tex-sector throughput (hardware counter "
                                               "peak, not a measured copy)",
                                  "bytes_per_launch": l2_bytes / launches_hist},
                     "fp64_tflops": fp64_tflops,
                     "limiter": "L2 gather of the FP64 history vectors (3 x R values per load) and FP64 issue; "
                                "the HBM fraction is low by construction at 32 load cases"},
        "e2e": {"value": world * args.steps * N * R / (ms_e2e / 1e3), "unit": "timesteps/s",
                "h2d_bytes_per_step": int(kh.numel() * 8), "d2h_bytes_per_step": int(2 * kh.numel() * 8)},
        "gpu_launches": args.steps * (2 * N + 1 + launches_hist),
        "clocks": hd["clocks"],
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            first, last = REF_STEADY + 1, REF_STEADY + 20
            rate_c, secs, setup = reference_rate(first, last, last, args.n, threads, args.tol)
            line["cpu_baseline"] = {"value": rate_c, "unit": "timesteps/s", "cores": threads, "kind": "reference",
                                    "assembly_s": setup,
                                    "sample": "reference solver (oracle/_ref) on the same bar, one load case, GMRES "
                                              "tolerance %g, time steps %d..%d of a %d-step run (every non-empty "
                                              "history step active), assembly excluded (%.2f s of march; its set-up, "
                                              "process start to step 1, %.1f s)" % (args.tol, first, last, last, secs,
                                                                                    setup)}
        except Exception as e:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    if rank == 0:
        print(json.dumps(line))
    hd["solver"].close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
