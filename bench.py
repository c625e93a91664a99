"""Throughput of the polydisperse Mie solve on B200 (solves/s with Jacobian).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one step = one polydisperse solve with its Jacobian): the
forward-linearized FP64 cloud droplet -- gamma distribution r_eff = 10 um,
v_eff = 0.1, r in [0.01, 60] um, 4 intervals x 500 Gauss radii, lambda =
0.865 um, m = 1.335 + 1e-6 i, x_max ~ 436, 4 derivatives (mr, mi, r_eff,
v_eff), GSF expansion and 181-angle phase matrix.  Inputs are synthetic (the
reference's published case parameters), nothing is read from disk.

  value  device time of the solve on inputs resident in HBM (L2 flushed
         between steps), whole job over all ranks;
  e2e    the same solve through the public C call lmie_solution() with host
         buffers: host preparation, host->device and device->host copies inside
         the timed region.

With N > 1 (torchrun, one process per GPU) every rank solves its own case per
step (independent cases, no data-path collective): weak scaling.
`--impl reference` times the reference's own CPU lmie_solution (compiled from
its sources into oracle/_ref) on all host cores, on rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from lmie_b200 import abi  # noqa: E402

METRIC = "polydisperse solves/s (+Jacobian)"
UNIT = "solves/s"
WORKLOAD = ("cloud droplet, forward-linearized FP64: gamma r_eff=10um v_eff=0.1, "
            "r in [0.01,60]um, 4x500 Gauss radii, lambda=0.865um, m=1.335+1e-6i, x_max~436, "
            "4 derivatives (mr, mi, r_eff, v_eff), GSF + 181-angle phase matrix")


def workload_case() -> abi.Case:
    return abi.Case(dist="gamma", lam=0.865, mr=1.335, mi=1e-6, a1=10.0, a2=0.1, r1=0.01,
                    r2=60.0, n_int2=4, n_quad=500, n_angles=181, accuracy=1e-7,
                    derivs=abi.deriv_unit("mr", "mi", "a1", "a2"))


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference library (oracle/_ref) or the CPU oracle port
# ---------------------------------------------------------------------------
def _cpu_library():
    ref = ROOT / "oracle" / "_ref" / "liblmie_ref.so"
    if ref.exists():
        lib = C.CDLL(str(ref))
        abi.bind_product_like(lib)
        return lib, "reference"
    orc = ROOT / "oracle" / "liblmie_oracle.so"
    if not orc.exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    lib = C.CDLL(str(orc))
    abi.bind_oracle(lib)
    return lib, "port"


def cpu_solve_seconds(lib, kind: str, case: abi.Case, threads: int) -> float:
    t0 = time.perf_counter()
    if kind == "reference":
        r = abi.solve(lib, case, n_threads=threads)
    else:
        r = abi.solve(lib, case, kind="oracle")
    dt = time.perf_counter() - t0
    if r.rc != 0:
        raise RuntimeError("CPU baseline solve failed")
    return dt


def cpu_baseline(case: abi.Case, budget_s: float = 20.0) -> dict:
    lib, kind = _cpu_library()
    threads = os.cpu_count() if kind == "reference" else 1
    cpu_solve_seconds(lib, kind, case, threads)          # warm caches
    times = []
    t_start = time.perf_counter()
    while len(times) < 20 and (time.perf_counter() - t_start) < budget_s:
        times.append(cpu_solve_seconds(lib, kind, case, threads))
    per = statistics.median(times)
    return {"value": 1.0 / per, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{len(times)} full solves of the benchmark case "
                      f"(median {per * 1e3:.1f} ms each, lmie_solution with n_threads={threads})"}


def run_reference_arm(args) -> int:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    case = workload_case()
    lib, kind = _cpu_library()
    threads = os.cpu_count() if kind == "reference" else 1
    for _ in range(args.warmup):
        cpu_solve_seconds(lib, kind, case, threads)
    total = 0.0
    for _ in range(args.steps):
        total += cpu_solve_seconds(lib, kind, case, threads)
    value = args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (reference case parameters)",
        "config": {"workload": WORKLOAD, "n_radii": 2000, "n_derivs": 4},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{args.steps} full solves, lmie_solution(n_threads={threads})"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# the B200 arm
# ---------------------------------------------------------------------------
def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except ValueError:
            pass
    return {}


def run_b200(args) -> int:
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    import lmie_b200
    lib = lmie_b200.library()
    if lib.lmieb_set_device(local) != 0:
        raise RuntimeError("lmieb_set_device failed")
    case = workload_case()

    # warm-up through the public call (allocates and plans)
    for _ in range(max(args.warmup, 1)):
        r = abi.solve(lib, case)
        if r.rc != 0:
            raise RuntimeError("lmie_solution failed")
    flops = (C.c_double * 4)()
    launches = C.c_longlong()
    h2d, d2h = C.c_size_t(), C.c_size_t()
    lib.lmieb_last_work(flops, C.byref(launches), C.byref(h2d), C.byref(d2h))

    clocks = ClockSampler(local)
    clocks.start()

    # e2e: K public calls with host buffers
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = abi.solve(lib, case)
        if r.rc != 0:
            raise RuntimeError("lmie_solution failed")
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)

    # device: K re-runs on resident inputs, L2 flushed before each (untimed)
    ms_total = C.c_double()
    ms_stage = (C.c_double * lmie_b200.N_STAGES)()
    lib.lmieb_rerun_device(args.warmup, 1, C.byref(ms_total), ms_stage)   # warm
    barrier()
    if lib.lmieb_rerun_device(args.steps, 1, C.byref(ms_total), ms_stage) != 0:
        raise RuntimeError("device re-run failed")
    barrier()
    dev_ms = max_over_ranks(ms_total.value)
    clk = clocks.stop()

    value = world * args.steps / (dev_ms * 1e-3)
    e2e = world * args.steps / e2e_s
    ang_ms = ms_stage[3] / args.steps
    peak = C.c_double()
    lib.lmieb_fp64_peak(C.byref(peak))
    achieved = flops[0] / (ang_ms * 1e-3) / 1e12 if ang_ms > 0 else None

    if rank == 0:
        cpu = cpu_baseline(case) if world == 1 else None
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (reference case parameters, generated in-process)",
            "config": {"workload": WORKLOAD, "n_radii": 2000, "n_derivs": 4,
                       "n_gauss_angles": 948, "parallelism": f"independent cases x{world}",
                       "l2": "flushed (256 MiB write) before every timed step"},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d.value),
                    "d2h_bytes_per_step": int(d2h.value)},
            "gpu_launches": int(launches.value) * args.steps,
            "roofline": {
                "kernel": "k_angular (S1/S2 accumulation + phase-matrix forms, FP64)",
                "bound": "fp64", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                "frac": (achieved / peak.value) if achieved else None, "traffic": None,
                "peak_source": "live FP64 FMA microbenchmark (lmieb_fp64_peak); "
                               "MEASURED_PEAKS.json holds HBM and BF16 only",
                "flops_per_launch": flops[0], "ms_per_launch": ang_ms},
            "stage_ms": {n: ms_stage[i] / args.steps for i, n in enumerate(lmie_b200.STAGES)},
            "clocks": clk,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
