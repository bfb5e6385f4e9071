"""Benchmark: one-fill, one-factorisation port solve of the 16x16 dipole array.

Workload (one "step"): the 16 x 16 planar array of half-wave dipoles at
300 MHz (41 segments each, degree 2, 10,496 unknowns, 256 ports, seeded
+-1 % length jitter), solved for every port: Galerkin fill, LU, solve of all
256 port columns, Y = B^T X.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--precision mixed|fp64] [--workload array|yagi_sweep|somm]

Prints ONE JSON line on rank 0.  ``value`` is device-timed throughput with the
inputs resident in HBM (solves per second over all ranks) of the default
mixed-precision path (complex64 tensor-core LU + FP64 refinement against the
FP64 fill); ``fp64_ms_per_step`` times the plain complex128 path on the same
workload; ``e2e`` is the same metric through the public
``BSplineSolver(...).compute_port_solution()`` call, host tables in and
coefficients + Y out.  ``sweep`` adds the batched frequency sweep of seeded
Yagis (64 frequencies each), sharded over the ranks.  Under torchrun each
rank solves its own replica of the array ("replicas only": a single dense
solve does not shard) and its shard of the sweep.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "sweep pts/s & fill+LU time, mixed+batched vs FP64 GPU at |ΔZin|/|Zin|≤1e-6"
UNIT = "pts/s"
WORKLOAD = "dipole_array_16x16_300MHz_41seg_d2_256port"
# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) per
# algorithmic byte of the tensor-core update (C read and written plus the
# hi / lo operand planes), measured on three consecutive launches of the
# 12x12 array's factorisation (a next-block, a trailing and a right-hand-side
# update of one panel: 158.8 MB against 219.3 MB); the bench line scales it
# by the step's algorithmic bytes per launch
TC_TRAFFIC_PER_ALG_BYTE = 158.8 / 219.3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--pivoting", default="static", choices=["static", "partial"],
                    help="mixed path: pivots within each diagonal block (with fallback) or partial pivoting")
    ap.add_argument("--fp64-steps", type=int, default=2, help="steps of the FP64 path timed beside a mixed run")
    ap.add_argument("--sweep-structs", type=int, default=512,
                    help="Yagis per rank in the sweep part of the line (0: none)")
    ap.add_argument("--sweep-workers", type=int, default=8, help="host threads (one CUDA stream each) per rank")
    ap.add_argument("--sweep-mode", choices=("grouped", "workers"), default="grouped",
                    help="grouped: padded groups of structures share one batched solve; workers: one batched "
                         "solve per structure on --sweep-workers host threads")
    ap.add_argument("--e2e-steps", type=int, default=None,
                    help="public-API calls timed for e2e (default: --steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nx", type=int, default=16)
    ap.add_argument("--micro", default=None, choices=["cgemm_tc"], help="kernel microbenchmark instead")
    ap.add_argument("--m", type=int, default=8192)
    ap.add_argument("--k", type=int, default=64)
    ap.add_argument("--workload", default="array", choices=["array", "yagi_sweep", "somm", "plate"])
    ap.add_argument("--n-struct", type=int, default=512)
    ap.add_argument("--fp64-structs", type=int, default=4)
    ap.add_argument("--fp64-kstep", type=int, default=4)
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        import statistics

        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------ reference
def load_workloads():
    """The seeded workload generators, loaded from their file so that the
    package itself (and its native library) is not imported by the
    reference arm."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("_mw_workloads", ROOT / "momwire_b200" / "workloads.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def workload_config(n_unknowns, ports, nx=16):
    """The ``config`` object of both arms (identical keys and values)."""
    name = WORKLOAD if nx == 16 else WORKLOAD.replace("16x16", f"{nx}x{nx}").replace("256port", f"{ports}port")
    zb = n_unknowns ** 2 * 16
    l2 = (f"inputs larger than L2 (Z = {zb / 1e9:.2f} GB per step, no flush)" if zb > 126e6 else
          f"inputs smaller than L2 (Z = {zb / 1e6:.1f} MB; not a headline size)")
    return {"workload": name, "n_unknowns": int(n_unknowns), "ports": int(ports), "l2": l2}


def cpu_baseline_full(kw):
    """The reference's own ``compute_port_solution()`` (its C++ fill kernels
    with OpenMP and LAPACK zgesv) on the full workload, once, on every host
    core; with the reference's Y for the parity check of the GPU arm."""
    from oracle import ref_baseline

    cores = ref_baseline.pin_threads()
    mw = ref_baseline.import_reference()
    sol, ph = ref_baseline.time_solve(mw, kw)
    return {
        "value": 1.0 / ph["total_s"],
        "unit": UNIT,
        "cores": cores,
        "kind": "reference",
        "sample": (f"one full reference compute_port_solution() of the workload (no extrapolation): fill "
                   f"{ph['fill_s']:.2f} s + LU/solve {ph['solve_s']:.2f} s of {ph['total_s']:.2f} s, "
                   f"OMP_NUM_THREADS=OPENBLAS_NUM_THREADS={cores}"),
        "fill_s": ph["fill_s"],
        "solve_s": ph["solve_s"],
        "total_s": ph["total_s"],
    }, sol


def run_reference(args):
    """The reference arm: the reference's own public call on the same
    workload, one full solve per step, on rank 0 (other ranks exit)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import ref_baseline

    cores = ref_baseline.pin_threads()  # before numpy is imported
    kw = load_workloads().dipole_array(args.nx, args.nx)
    try:
        mw = ref_baseline.import_reference()
    except ImportError as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference package not staged: {e}"}), flush=True)
        return
    for _ in range(args.warmup):
        ref_baseline.time_solve(mw, kw)
    per = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sol, ph = ref_baseline.time_solve(mw, kw)
        per.append(ph)
    wall = time.perf_counter() - t0
    per_step = sum(p["total_s"] for p in per) / len(per)
    value = 1.0 / per_step
    n_b = int(sol.coeffs.shape[0])
    ports = int(sol.y.shape[0])
    mapped = [p for p in ref_baseline.loaded_native_objects() if str(ROOT) in p]
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": per_step * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "complex128",
        "data": "synthetic (seeded dipole array)",
        "config": workload_config(n_b, ports, args.nx),
        "parallelism": f"host threads x{cores}",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": (f"the full workload each step: reference BSplineSolver(...)."
                                    f"compute_port_solution() with its C++ kernels (OpenMP) and LAPACK zgesv, "
                                    f"OMP_NUM_THREADS=OPENBLAS_NUM_THREADS={cores}")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "phases_s": {"fill": sum(p["fill_s"] for p in per) / len(per),
                     "lu_solve": sum(p["solve_s"] for p in per) / len(per)},
        "timed_wall_s": wall,
        "native_objects_in_repo": mapped,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ b200
def run_b200(args, kw):
    import numpy as np
    import torch

    import momwire_b200
    from momwire_b200 import _lib

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    lib = _lib.load()
    lib.mw_set_mixed_pivoting(0 if args.pivoting == "static" else 1)

    solver = momwire_b200.BSplineSolver(**kw, precision=args.precision, device=local)
    buf = solver._alloc()
    stream = torch.cuda.current_stream(dev)
    st = stream.cuda_stream

    def step():
        solver._device_solve(buf, st)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    solver._check_info(buf)

    n0 = lib.mw_launch_count()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    if pg:
        pg.barrier()
    ms = e0.elapsed_time(e1)
    launches = (lib.mw_launch_count() - n0) // max(args.steps, 1)
    # per-kernel-class device times from a separate, untimed pass: the
    # library's profiler brackets every launch with CUDA events, which the
    # timed steps above must not carry
    prof_steps = max(1, min(args.steps, 3))
    _lib.profile_enable(True)
    for _ in range(prof_steps):
        step()
    torch.cuda.synchronize()
    prof = _lib.profile_read()
    _lib.profile_enable(False)
    if pg:
        t = torch.tensor([ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = world * args.steps / (ms / 1e3)

    # correctness of what was timed: the 16x16 golden Y when available
    y_dev = buf["Y"][: buf["n_p"], : buf["n_p"]].cpu().numpy().T
    golden = ROOT / "tests" / "golden" / "array16x16.npz"
    y_err = None
    if golden.exists() and args.nx == 16:
        g = np.load(golden)
        y_err = float(np.max(np.abs(y_dev - g["y"])) / np.max(np.abs(g["y"])))

    # e2e through the public API: host tables in, coefficients + Y out
    e2e_ms = []
    h2d = d2h = 0
    e2e_steps = args.steps if args.e2e_steps is None else args.e2e_steps
    for i in range(e2e_steps + 1 if e2e_steps > 0 else 0):
        s = momwire_b200.BSplineSolver(**kw, precision=args.precision, device=local)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sol = s.compute_port_solution()
        b.record(stream)
        torch.cuda.synchronize()
        if i:  # first call is warm-up
            e2e_ms.append(a.elapsed_time(b))
        h2d, d2h = s.last_stats["h2d_bytes"], s.last_stats["d2h_bytes"]
    e2e_step = sum(e2e_ms) / len(e2e_ms) if e2e_ms else float("nan")
    if pg:
        t = torch.tensor([e2e_step], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_step = float(t.item())

    # the plain FP64 path on the same workload, for the mixed-vs-FP64 ratio
    fp64_ms = None
    if args.precision == "mixed" and args.fp64_steps > 0:
        s64 = momwire_b200.BSplineSolver(**kw, precision="fp64", device=local)
        b64 = s64._alloc()
        s64._device_solve(b64, st)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        e0.record(stream)
        for _ in range(args.fp64_steps):
            s64._device_solve(b64, st)
        e1.record(stream)
        torch.cuda.synchronize()
        fp64_ms = e0.elapsed_time(e1) / args.fp64_steps
        if pg:
            t = torch.tensor([fp64_ms], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            fp64_ms = float(t.item())
        del s64, b64

    sweep_part = run_sweep_part(args, rank, world, local, pg) if args.sweep_structs > 0 else None

    # roofline of the dominant kernel class
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except OSError:
        pass
    # the roofline is stated for the dominant compute kernel: the tensor-core
    # update on the mixed path (the LU panel, often as long, is latency-
    # bound -- one cross-CTA pivot exchange per column -- and reported
    # beside it), the dominant kernel class otherwise
    walls = {k: prof.pop(k) for k in ("factor_wall", "solve_wall") if k in prof}
    by_time = max(prof.items(), key=lambda kv: kv[1][1]) if prof else None
    dom = ("cgemm_tc", prof["cgemm_tc"]) if "cgemm_tc" in prof else by_time
    roof = None
    if dom:
        name, (cnt, tms, fl, by) = dom
        achieved = fl / (tms / 1e3) / 1e12
        if name == "cgemm_tc":
            # tcgen05 kind::tf32: B200's TF32 tensor rate is half its BF16
            # rate; the 3xTF32 split issues three MMAs per algorithmic one
            measured = "bf16_tflops" in peaks
            bf16 = float(peaks.get("bf16_tflops", 1590.0))
            peak = bf16 / 2.0
            # DRAM bytes per launch: the measured DRAM-to-algorithmic ratio
            # (ncu cannot run inside the timed bench) times this step's
            # algorithmic bytes per launch
            traffic = TC_TRAFFIC_PER_ALG_BYTE * by / cnt if cnt else None
            roof = {"kernel": name, "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "tensor_pipe_frac": 3.0 * achieved / peak, "traffic": traffic,
                    "traffic_unit": "bytes per launch (dram read + write: ncu ratio to algorithmic bytes on "
                                    "three 12x12 launches, times this step's algorithmic bytes per launch)",
                    "algorithmic_bytes_per_launch": by / cnt if cnt else None,
                    "launches_per_step": cnt / prof_steps, "avg_launch_ms": tms / cnt,
                    "peak_source": ("of measured: MEASURED_PEAKS bf16_tflops / 2" if measured else
                                    "of fallback: 1590 TFLOP/s bf16 / 2 (MEASURED_PEAKS.json absent)")
                                   + " (TF32 rate); achieved counts 8mnk complex flops, the tensor pipe executes "
                                   "3x that (3xTF32)"}
        else:
            # FP64 work has no measured peak in MEASURED_PEAKS.json: the
            # nominal B200 FP64 rate is the denominator there.
            fp64_nominal = 37.0
            roof = {"kernel": name, "bound": "fp64", "achieved": achieved, "peak": fp64_nominal, "unit": "TFLOP/s",
                    "frac": achieved / fp64_nominal, "traffic": None, "launches_per_step": cnt / prof_steps,
                    "avg_launch_ms": tms / cnt,
                    "peak_source": "nominal B200 FP64 (no FP64 entry in MEASURED_PEAKS)"}
    breakdown = {k: {"launches": v[0] / prof_steps, "ms_per_step": v[1] / prof_steps,
                     "tflops": (v[2] / (v[1] / 1e3) / 1e12) if v[1] > 0 and v[2] > 0 else None}
                 for k, v in prof.items()}
    # the kernel class that takes the most device time, against its own
    # bound (latency-bound classes against the nominal FP32 rate, which
    # they are far from by design)
    roof_time = None
    if by_time and (dom is None or by_time[0] != dom[0]):
        name, (cnt, tms, fl, by) = by_time
        fp32_nominal = 75.0
        roof_time = {"kernel": name, "bound": "latency" if name in ("lu_panel", "trsm", "laswp") else "fp64",
                     "achieved": fl / (tms / 1e3) / 1e12 if fl > 0 else None, "unit": "TFLOP/s",
                     "peak": fp32_nominal if name in ("lu_panel", "trsm") else 37.0,
                     "ms_per_step": tms / prof_steps, "launches_per_step": cnt / prof_steps,
                     "peak_source": "nominal B200 FP32 (75) / FP64 (37) rates; no measured entry"}
        if roof_time["achieved"] is not None:
            roof_time["frac"] = roof_time["achieved"] / roof_time["peak"]
    # whole-phase rates: fill pairs/s (N_s^2 segment pairs per fill) and the
    # factorisation's (8/3) n^3 over its wall time
    n_seg = int(solver._geometry().n)
    phases = {}
    if "fill" in prof:
        f_ms = prof["fill"][1] / prof["fill"][0]
        phases["fill_ms"] = f_ms
        phases["fill_pairs_per_s"] = n_seg ** 2 / (f_ms / 1e3)
        phases["fill_segments"] = n_seg
    if "factor_wall" in walls:
        cnt, tms, fl, _by = walls["factor_wall"]
        phases["lu_ms"] = tms / cnt
        phases["lu_tflops"] = (8.0 / 3.0) * buf["n"] ** 3 / (tms / cnt / 1e3) / 1e12
        phases["lu_tflops_note"] = "(8/3) n^3 complex-LU flops over the factorisation's wall time"
    if "solve_wall" in walls:
        cnt, tms, _fl, _by = walls["solve_wall"]
        phases["triangular_solves_ms_per_step"] = tms / prof_steps

    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "complex128" if args.precision == "fp64" else "complex64+fp64-refine",
        "data": "synthetic (seeded dipole array)",
        "config": workload_config(buf["n"], buf["n_p"], args.nx),
        "precision": args.precision,
        "parallelism": f"replicas x{world}",
        "e2e": {"value": world * 1e3 / e2e_step, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_step},
        "gpu_launches": int(launches),
        "roofline": roof,
        "kernels": breakdown,
        "kernels_note": (f"per-class device times from {prof_steps} profiled steps after the timed ones "
                         "(the profiler brackets each launch with CUDA events; the timed steps run without it)"),
        "dominant_by_time": by_time[0] if by_time else None,
        "roofline_by_time": roof_time,
        "phases": phases,
        "pivoting": {0: "static (diagonal block)", 1: "partial", 2: "static rejected, then partial"}.get(
            int(lib.mw_last_mixed_pivoting()), None) if args.precision == "mixed" else "partial",
        "static_pivot_max_abs_l21": float(lib.mw_last_mixed_growth()) if args.precision == "mixed" else None,
        "refinement": dict(solver.last_refinement or {}, history=refine_history(lib)),
        "clocks": clocks.summary(),
        "y_rel_err_vs_reference": y_err,
        "fp64_ms_per_step": fp64_ms,
        "speedup_vs_fp64": (fp64_ms / ms_step) if fp64_ms else None,
        "sweep": sweep_part,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, ref_sol = cpu_baseline_full(kw)
        line["cpu_baseline"] = cpu
        # the timed GPU result against the reference's, run on this host
        line["y_rel_err_vs_reference_run"] = float(np.max(np.abs(y_dev - ref_sol.y)) / np.max(np.abs(ref_sol.y)))
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


def refine_history(lib):
    """The controlling relative correction of each refinement step of the
    last mixed solve on this thread."""
    import ctypes

    buf = (ctypes.c_double * 16)()
    n = lib.mw_last_mixed_history(buf, 16)
    return [float(buf[i]) for i in range(min(n, 16))]


def run_micro(args):
    """Kernel microbenchmark: C (m x m complex64) -= A (m x k) B (k x m)
    through mw_cgemm_tc_sub, timed with CUDA events."""
    import torch

    from momwire_b200 import _lib

    m, k = args.m, args.k
    dev = torch.device("cuda", 0)
    A = torch.randn(k, m, dtype=torch.complex64, device=dev)  # column-major (m x k)
    B = torch.randn(m, k, dtype=torch.complex64, device=dev)  # column-major (k x m)
    Cm = torch.randn(m, m, dtype=torch.complex64, device=dev)
    wsb = _lib.load().mw_cgemm_tc_workspace_size(m, m, k)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)

    def run():
        _lib.call("mw_cgemm_tc_sub", m, m, k, A.data_ptr(), m, B.data_ptr(), k, Cm.data_ptr(), m, ws.data_ptr(), wsb,
                  status.data_ptr(), None)

    run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    print(json.dumps({"micro": "cgemm_tc", "m": m, "n": m, "k": k, "ms": ms,
                      "tflops_algorithmic": 8.0 * m * m * k / (ms / 1e3) / 1e12, "status": int(status.item())}))


def run_sweep_part(args, rank, world, local, pg):
    """Sweep part of the headline line: world x --sweep-structs seeded Yagis
    at 64 frequencies, sharded over the ranks (LPT on n^3), each rank's
    shard device-timed; pts/s = all solves / the slowest rank.  Rank 0 also
    times the plain FP64 GPU path on a stratified sample (the median
    structure of each of 16 size strata, every 8th frequency), compares
    drive-point impedances, and at one GPU times the reference's CPU sweep
    on the same sample."""
    import numpy as np
    import torch

    import momwire_b200
    from momwire_b200 import sweep
    from momwire_b200.workloads import yagi_sweep

    structs, ks = yagi_sweep(n_structures=args.sweep_structs * world, n_freq=64, seed=0)
    parts = [sweep.shard_indices(structs, r, world) for r in range(world)]
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    fn = sweep.mixed_sweep_fn(local)
    # warm-up: one structure per autotuner bucket (tunes and caches its
    # panel width outside the timed region)
    from momwire_b200 import autotune

    if args.sweep_mode == "grouped":
        sweep.grouped_mixed_sweep(structs, ks[:8], device=local, indices=parts[rank])
    else:
        seen = set()
        for i in parts[rank]:
            s0 = momwire_b200.BSplineSolver(**structs[i], precision="mixed", device=local)
            key = autotune.key(s0._basis().n, s0.degree, "free")
            if key not in seen:
                seen.add(key)
                fn(structs[i], ks[:8])
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    if args.sweep_mode == "grouped":
        local_y = sweep.grouped_mixed_sweep(structs, ks, device=local, indices=parts[rank])
    else:
        local_y = sweep.solve_shard(structs, ks, parts[rank], fn, workers=args.sweep_workers, device=local)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    if pg:
        t = torch.tensor([ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    ys = sweep.gather(local_y)
    out = {"workload": f"yagi_sweep_{len(structs)}x64", "solves": len(structs) * len(ks),
           "pts_per_s": len(structs) * len(ks) / (ms / 1e3), "ms": ms, "sharding": f"LPT x{world}",
           "mode": args.sweep_mode}
    if args.sweep_mode == "workers":
        out["workers_per_rank"] = args.sweep_workers
    if rank == 0:
        out.update(fp64_sweep_sample(structs, ks, ys, local, stream))
        out["speedup_vs_fp64"] = out["pts_per_s"] / out["fp64_pts_per_s"]
        if world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_sweep_sample(structs, ks)
    return out


def sweep_strata(structs, n_strata=16):
    """Stratified sample of a structure population: sorted by unknown count
    and cut into n_strata equal strata; returns (the structure nearest each
    stratum's median, the stratum sizes)."""
    import numpy as np

    from momwire_b200 import sweep

    order = sorted(range(len(structs)), key=lambda i: (sweep.structure_cost(structs[i]), i))
    strata = [list(x) for x in np.array_split(order, min(n_strata, len(order))) if len(x)]
    return [st[len(st) // 2] for st in strata], [len(st) for st in strata]


def fp64_sweep_sample(structs, ks, ys, local, stream, kstep=8):
    """The plain FP64 GPU path (per-frequency complex128 solves) on a
    stratified sample -- the median structure of each of 16 size strata at
    every kstep-th frequency -- extrapolated to the whole sweep by stratum
    size; and the sample's drive-point impedances against the mixed sweep's."""
    import numpy as np
    import torch

    import momwire_b200

    picks, weights = sweep_strata(structs)
    sub = ks[::kstep]
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    momwire_b200.BSplineSolver(**structs[picks[0]], device=local).compute_y_matrix_swept(sub[:1])  # warm
    total_ms, err, sample_ms = 0.0, 0.0, 0.0
    for i, w in zip(picks, weights):
        s = momwire_b200.BSplineSolver(**structs[i], device=local)
        a.record(stream)
        y = s.compute_y_matrix_swept(sub)
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        sample_ms += ms
        total_ms += w * ms / len(sub) * len(ks)
        z64, zmx = 1.0 / y[:, 0, 0], 1.0 / ys[i][::kstep, 0, 0]
        err = max(err, float(np.max(np.abs(zmx - z64) / np.abs(z64))))
    return {"fp64_pts_per_s": len(structs) * len(ks) / (total_ms / 1e3), "max_rel_dZin_vs_fp64": err,
            "fp64_sample": (f"{len(picks)} structures (median of each of {len(picks)} size strata) x {len(sub)} "
                            f"frequencies (every {kstep}th), {sample_ms:.0f} ms device time, extrapolated by "
                            "stratum size to every structure and frequency")}


def cpu_sweep_sample(structs, ks, kstep=8):
    """The reference's own compute_y_matrix_swept (its C++ swept fill and
    LAPACK per frequency) on the same stratified sample, on every host
    core, extrapolated to the whole sweep by stratum size."""
    from oracle import ref_baseline

    cores = ref_baseline.pin_threads()
    mw = ref_baseline.import_reference()
    picks, weights = sweep_strata(structs)
    sub = ks[::kstep]
    total_s, sample_s = 0.0, 0.0
    for i, w in zip(picks, weights):
        t0 = time.perf_counter()
        mw.BSplineSolver(**structs[i]).compute_y_matrix_swept(sub)
        dt = time.perf_counter() - t0
        sample_s += dt
        total_s += w * dt / len(sub) * len(ks)
    return {"value": len(structs) * len(ks) / total_s, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": (f"reference compute_y_matrix_swept on {len(picks)} structures (median of each size "
                       f"stratum) x {len(sub)} frequencies: {sample_s:.1f} s, extrapolated by stratum size to "
                       f"{len(structs)} x {len(ks)} solves")}


def run_somm(args):
    """The Sommerfeld-ground workload: seeded structures (dipole, monopole +
    radials, inverted V) over random grounds and frequencies, each solved
    cold through the public API on the quadrature-grid path and on the
    surrogate path; solves per second and the impedance agreement."""
    import numpy as np
    import torch

    import momwire_b200
    from momwire_b200 import sommerfeld as P
    from momwire_b200.workloads import somm_structures

    structs = somm_structures(args.n_struct, seed=0)
    from momwire_b200 import surrogate

    arms = {"grid": dict(sommerfeld_method="grid"),
            "surrogate_at_1e-6": dict(sommerfeld_method="surrogate"),
            "surrogate_approx": dict(sommerfeld_method="surrogate", surrogate_tol=surrogate.APPROX_TOL)}
    for kw_arm in arms.values():
        momwire_b200.BSplineSolver(**structs[0], **kw_arm).compute_impedance()
    res, z = {}, {}
    for name, kw_arm in arms.items():
        P.clear_cache()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        zs, used = [], 0
        for kw in structs:
            s = momwire_b200.BSplineSolver(**kw, **kw_arm)
            zs.append(s.compute_impedance()[0])
            used += s.last_sommerfeld["method"] == "surrogate"
        torch.cuda.synchronize()
        res[name] = (time.perf_counter() - t0, used)
        z[name] = np.array(zs)
    line = {"workload": f"somm_structures_{len(structs)}", "grid_pts_per_s": len(structs) / res["grid"][0],
            "timing": "wall clock per cold structure, host + device"}
    for name in ("surrogate_at_1e-6", "surrogate_approx"):
        err = np.abs(z[name] - z["grid"]) / np.abs(z["grid"])
        line[name] = {"pts_per_s": len(structs) / res[name][0], "speedup_vs_grid": res["grid"][0] / res[name][0],
                      "served": res[name][1], "max_rel_dZin_vs_grid": float(err.max()),
                      "median_rel_dZin_vs_grid": float(np.median(err))}
    print(json.dumps(line), flush=True)


def run_plate(args):
    """The combined large case: 64x64-cell wire-grid plate (2 segments per
    wire) at 2 m over a Sommerfeld ground (13, 5e-3) with a 10 m monopole
    from its centre, 14.1 MHz, 8 ports (33,290 unknowns, 4,218 KCL rows).
    One warm-up and --steps timed solves per precision through the public
    API (device events around compute_port_solution), and the drive-point
    impedances of the mixed path against the FP64 path."""
    import numpy as np
    import torch

    import momwire_b200
    from momwire_b200 import _lib

    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from cases import wire_grid_plate

    kw = wire_grid_plate()
    stream = torch.cuda.current_stream()
    out, ys = {}, {}
    for prec in ("fp64", "mixed"):
        s = momwire_b200.BSplineSolver(**kw, precision=prec)
        s.compute_port_solution()
        torch.cuda.synchronize()
        _lib.profile_enable(True)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            sol = s.compute_port_solution()
        b.record(stream)
        torch.cuda.synchronize()
        prof = _lib.profile_read()
        _lib.profile_enable(False)
        out[prec] = {"ms_per_step": a.elapsed_time(b) / args.steps,
                     "kernels_ms": {k: round(v[1] / args.steps, 1) for k, v in prof.items()}}
        ys[prec] = sol.y
    z64, zmx = 1.0 / np.diag(ys["fp64"]), 1.0 / np.diag(ys["mixed"])
    print(json.dumps({"workload": "plate64_sommerfeld_33290_unknowns", "n_unknowns": int(s._basis().n), "ports": 8,
                      "fp64": out["fp64"], "mixed": out["mixed"],
                      "speedup_mixed_vs_fp64": out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"],
                      "max_rel_dZin_mixed_vs_fp64": float(np.max(np.abs(zmx - z64) / np.abs(z64))),
                      "timing": "device events around compute_port_solution (host tables, h2d, d2h included)"}),
          flush=True)


def run_sweep(args):
    """The batched-sweep workload: seeded Yagis, 64 frequencies each,
    25.2-30.8 MHz.  Mixed + batched over all structures (device-timed per
    structure with CUDA events, summed), against the plain FP64 GPU path
    (per-frequency complex128 solves) on the first --fp64-structs
    structures, extrapolated per solve."""
    import numpy as np
    import torch

    import momwire_b200
    from momwire_b200.workloads import yagi_sweep

    structs, ks = yagi_sweep(n_structures=args.n_struct, n_freq=64, seed=0)
    stream = torch.cuda.current_stream()

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        out = fn()
        b.record(stream)
        torch.cuda.synchronize()
        return out, a.elapsed_time(b)

    # warm-up (library init, kernels)
    momwire_b200.BSplineSolver(**structs[0], precision="mixed").compute_y_matrix_swept(ks[:4])
    total_ms, iters, max_err = 0.0, 0, 0.0
    ys = []
    for kw in structs:
        s = momwire_b200.BSplineSolver(**kw, precision="mixed")
        y, ms = timed(lambda: s.compute_y_matrix_swept(ks))
        total_ms += ms
        iters = max(iters, s.last_refinement["iterations"])
        ys.append(y)
    mixed_pts = len(structs) * len(ks) / (total_ms / 1e3)
    fp64_ms, n_fp64 = 0.0, 0
    for i, kw in enumerate(structs[: args.fp64_structs]):
        s = momwire_b200.BSplineSolver(**kw)
        sub = ks[:: args.fp64_kstep]
        y, ms = timed(lambda: s.compute_y_matrix_swept(sub))
        fp64_ms += ms
        n_fp64 += len(sub)
        z64 = 1.0 / y[:, 0, 0]
        zmx = 1.0 / ys[i][:: args.fp64_kstep, 0, 0]
        max_err = max(max_err, float(np.max(np.abs(zmx - z64) / np.abs(z64))))
    fp64_pts = n_fp64 / (fp64_ms / 1e3)
    print(json.dumps({"workload": f"yagi_sweep_{len(structs)}x64", "mixed_batched_pts_per_s": mixed_pts,
                      "mixed_total_s": total_ms / 1e3, "fp64_per_k_pts_per_s": fp64_pts,
                      "fp64_sample_solves": n_fp64, "speedup": mixed_pts / fp64_pts,
                      "max_rel_dZin_vs_fp64": max_err, "max_refinement_iterations": iters}), flush=True)


def main():
    args = parse()
    if args.micro:
        run_micro(args)
        return
    if args.workload == "yagi_sweep":
        run_sweep(args)
        return
    if args.workload == "somm":
        run_somm(args)
        return
    if args.workload == "plate":
        run_plate(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    from momwire_b200.workloads import dipole_array

    run_b200(args, dipole_array(args.nx, args.nx))


if __name__ == "__main__":
    main()
