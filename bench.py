"""Throughput of the polydisperse Mie solve on B200 (solves/s with Jacobian).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one step = one batch): 4096 independent polydisperse cases of
uneven size, generated from a fixed seed (lmie_b200.workloads.batched_uneven:
r_eff log-uniform 0.05-20 um, v_eff 0.02-0.3, wavelength 0.34-2.1 um,
m = 1.33-1.60 + i 1e-8..0.1, gamma or log-normal distributions, 100-2000
radii scaled to the size parameter, size parameters 0.2-1063, n_max 9-1112),
each with its Jacobian w.r.t. mr, mi and the two distribution parameters, GSF
expansion and 181-angle phase matrix.  Inputs are synthetic; nothing is read
from disk.

  value  device time of the batch on inputs resident in HBM (the L2 is
         flushed before every step), solves/s over all ranks, with the
         angular S1/S2 contraction as an exact fixed-point sum on the int8
         tensor cores (lmie_solution_batch2(..., LMIEB_PRECISION_INT8): every
         output within 1e-9 of the FP64 form and the same truncation n_coef,
         cases near the truncation threshold solved again in FP64);
  e2e    the same batch through the public C call lmie_solution_batch2() on
         host buffers: host preparation, the host->device and device->host
         copies and the scatter into the caller's lmie_out_data are inside the
         timed region.

The same JSON line carries secondary measurements of the same run:
  int8_error_vs_fp64  the headline form's error against the FP64 form over
                the whole batch, per output array and per derivative slice;
  fp64          the same batch in FP64 throughout (lmie_solution_batch):
                device and e2e solves/s, stage times, roofline of its K3;
  split_tf32x3  the batch with the angular contraction in 3xTF32 on the
                tensor cores (LMIEB_PRECISION_TF32X3, FP32 accumulation):
                device and e2e solves/s, stage times, and its measured error
                against the FP64 form per output array over a sample;
  plain         the drop-in form: one lmie_solution() call per case (FP64),
                e2e solves/s over every case of the batch;
  single_case   the reference's cloud-droplet case (2000 radii, x_max ~436,
                4 derivatives) through lmie_solution();
  adjoint       the retrieval workload (256 wavelengths sharing 64 bins x 32
                Gauss radii, 181 angles) through lmie_solution_adjoint():
                loss and gradient w.r.t. 512 refractive-index parameters and
                64 bin weights per call, wavelength-solves/s, next to the
                reference's forward mode on a sample of its per-radius
                SIZE_DIST_MONO solves on the host cores.

With N > 1 (torchrun, one process per GPU) every rank solves its own batch
(independent cases, no data-path collective): weak scaling.
`--impl reference` times the reference's own CPU lmie_solution (compiled from
its sources into oracle/_ref) on all host cores, one case per host thread,
in steps of 256 of the same cases, on rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from lmie_b200 import abi, shard, workloads  # noqa: E402

METRIC = "polydisperse solves/s (+Jacobian)"
UNIT = "solves/s"
N_CASES = 4096
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one k_angular /
# k_angular_tc / k_angular_oz launch on this workload: measured with ncu on a
# 256-case batch of the same generator and scaled by the ratio of angular work
# (13.33; 13.0 in chunks of the int8 product: 317.6 MB -> 4.13 GB, about the
# B operand digits read once).
ANGULAR_TRAFFIC = {"fp64": 12.21e9, "tf32x3": 5.15e9, "int8": 4.13e9}
WORKLOAD = ("batched uneven: 4096 seeded cases (r_eff 0.05-20 um, v_eff 0.02-0.3, lambda 0.34-2.1 um, "
            "mr 1.33-1.60, mi 1e-8-0.1, gamma/log-normal, 100-2000 radii, x_max 0.2-1063), "
            "4 derivatives each (mr, mi, a1, a2), GSF + 181-angle phase matrix")


def single_case() -> abi.Case:
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
# C-level batch: in/out structs built once, outputs preallocated
# ---------------------------------------------------------------------------
class CBatch:
    """lmie_in_data / lmie_out_data arrays for a list of cases, with outputs
    allocated once by the library (the caller-owned arrays of alloc_out = 0)."""

    def __init__(self, lib, cases):
        self.lib = lib
        self.cases = cases
        self.blocks = [abi.InputBlock(c) for c in cases]
        n = len(cases)
        self.ins = (abi.lmie_in_data * n)(*[b.s for b in self.blocks])
        self.outs = (abi.lmie_out_data * n)()
        lib.lmie_out_alloc.argtypes = [C.POINTER(abi.lmie_in_data), C.POINTER(abi.lmie_out_data), C.c_int]
        for i, c in enumerate(cases):
            mc = lib.lmie_calc_max_coef(c.lam, self.ins[i].dist_type, c.a1, c.a2, c.a3, c.r1, c.r2)
            lib.lmie_out_alloc(C.byref(self.ins[i]), C.byref(self.outs[i]), mc)

    def solve_batch(self, n_threads: int, precision: int = abi.PRECISION_FP64) -> int:
        f = self.lib.lmie_solution_batch2
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.POINTER(abi.lmie_in_data), C.POINTER(abi.lmie_out_data), C.c_int,
                      C.c_int, C.c_int, C.c_int]
        return f(len(self.cases), self.ins, self.outs, 0, 0, n_threads, precision)

    def autotune(self, n_threads: int, precision: int) -> dict:
        f = self.lib.lmie_solution_autotune
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.POINTER(abi.lmie_in_data), C.POINTER(abi.lmie_out_data), C.c_int, C.c_int,
                      C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        ch, it, ms = C.c_int(), C.c_double(), C.c_double()
        if f(len(self.cases), self.ins, self.outs, n_threads, precision, C.byref(ch), C.byref(it), C.byref(ms)):
            raise RuntimeError("lmie_solution_autotune failed")
        return {"pipeline_parts": ch.value, "angular_items_per_sm": it.value, "ms_per_call": ms.value}

    def solve_each(self, n_threads: int, count: int = -1) -> int:
        for i in range(len(self.cases) if count < 0 else count):
            rc = self.lib.lmie_solution(C.byref(self.ins[i]), C.byref(self.outs[i]), 0, 0, n_threads, 0)
            if rc != 0:
                return rc
        return 0


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


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def _seeded_order(n: int):
    import random
    order = list(range(n))
    random.Random(workloads.SEED).shuffle(order)
    return order


def _cpu_solve(lib, kind, case, n_threads):
    r = abi.solve(lib, case, n_threads=n_threads) if kind == "reference" else abi.solve(lib, case, kind="oracle")
    if r.rc != 0:
        raise RuntimeError("CPU solve failed")


def cpu_radius_parallel(cases, order, budget_s: float) -> dict:
    """The reference's own threading: one case after another, each
    lmie_solution() spreading its radii over all host threads."""
    lib, kind = _cpu_library()
    threads = os.cpu_count() if kind == "reference" else 1
    t0 = time.perf_counter()
    done = 0
    for i in order:
        _cpu_solve(lib, kind, cases[i], threads)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    wall = time.perf_counter() - t0
    return {"value": done / wall, "unit": UNIT, "cores": threads, "kind": kind, "cases": done, "seconds": wall,
            "mode": f"radius-parallel: one case after another, lmie_solution(n_threads={threads})"}


def cpu_case_parallel(cases, order) -> dict:
    """One case per host thread: every host thread takes the next case of
    `order` and solves it with lmie_solution(n_threads=1) (ctypes releases the
    interpreter lock during the call); wall time until all are done."""
    import concurrent.futures as cf
    lib, kind = _cpu_library()
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(lambda i: _cpu_solve(lib, kind, cases[i], 1), order))
    wall = time.perf_counter() - t0
    return {"value": len(order) / wall, "unit": UNIT, "cores": threads, "kind": kind, "cases": len(order),
            "seconds": wall, "mode": "case-parallel: one case per host thread, lmie_solution(n_threads=1)"}


def cpu_baseline(cases, budget_s: float = 20.0) -> dict:
    """The CPU implementation on the host cores in both of its parallel forms
    over bounded samples of the batch (seeded order, so sizes are
    represented); the faster one is the baseline value."""
    order = _seeded_order(len(cases))
    radius = cpu_radius_parallel(cases, order, budget_s / 2)
    n_case = max(len(order) // 16, min(len(order), int(radius["value"] * budget_s / 2)))
    case = cpu_case_parallel(cases, order[:n_case])
    best = max((radius, case), key=lambda v: v["value"])
    return {"value": best["value"], "unit": UNIT, "cores": best["cores"], "kind": best["kind"],
            "cpu_model": cpu_model(),
            "sample": f"{best['cases']} of the {len(cases)} batch cases in seeded random order "
                      f"({best['seconds']:.1f} s), {best['mode']}",
            "variants": {"radius_parallel": radius, "case_parallel": case}}


def _relmax(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = float(np.max(np.abs(b))) if b.size else 0.0
    num = float(np.max(np.abs(a - b))) if b.size else 0.0
    return num / den if den > 0 else num


def split_errors(lib, cases, n_threads: int) -> dict:
    """Largest error of the split-precision form against the FP64 form over
    `cases`, per output: max|split - fp64| / max|fp64| per case and array
    (GSF/Legendre arrays over the shorter n_coef), then the worst case."""
    ref = abi.solve_batch(lib, cases, n_threads=n_threads, precision=abi.PRECISION_FP64)
    got = abi.solve_batch(lib, cases, n_threads=n_threads, precision=abi.PRECISION_TF32X3)
    worst, n_same = {}, 0
    for g, r in zip(got, ref):
        if g.rc != 0 or r.rc != 0:
            raise RuntimeError("solve failed while measuring the split-precision error")
        err = {"cext": _relmax(g.scalars["cext"], r.scalars["cext"]), "g": _relmax(g.scalars["g"], r.scalars["g"])}
        nc = min(g.n_coef, r.n_coef)
        for name in ("gc", "pf", "gc_l", "pf_l"):
            a, b = getattr(g, name), getattr(r, name)
            if b is None:
                continue
            if name == "gc":
                a, b = a[:, :nc], b[:, :nc]
            elif name == "gc_l":
                a, b = a[:, :, :nc], b[:, :, :nc]
            err[name] = _relmax(a, b)
        same_n = g.n_coef == r.n_coef
        n_same += same_n
        for k, v in err.items():
            if k in ("pf", "pf_l") and not same_n:
                k = k + "_truncated_differently"
            worst[k] = max(worst.get(k, 0.0), float(v))
    return {"cases": len(cases), "max_rel_err": worst, "cases_with_same_n_coef": n_same,
            "metric": "max over cases of max|split - fp64| / max|fp64| per output array (gc over the "
                      "shorter n_coef; pf where both forms kept the same number of coefficients, and "
                      "separately where the truncation at `accuracy` differed)"}


def precision_stress_measurement(lib, n_threads: int, n_cases: int = 8) -> dict:
    """The large-particle configuration (size parameter up to 5000, 8000 radii,
    10154 Gauss angles, four derivatives) on a sample of its cases: each
    tensor-core form's error per output array against the FP64 form, and the
    forms' throughput through the public batch call (wall clock, host
    buffers)."""
    cases = workloads.precision_stress(n_cases)
    lib.lmieb_set_pipeline(0)
    out = {"workload": f"workloads.precision_stress: first {n_cases} of 256 seeded cases "
                       "(gamma, r_eff 150-400 um, x_max 5000, 16x500 radii, 4 derivatives)"}
    res = {}
    forms = (("fp64", abi.PRECISION_FP64), ("tf32x3", abi.PRECISION_TF32X3), ("int8", abi.PRECISION_INT8))
    for name, prec in forms:
        abi.solve_batch(lib, cases[:1], n_threads=n_threads, precision=prec)   # settle buffers
        t0 = time.perf_counter()
        res[name] = abi.solve_batch(lib, cases, n_threads=n_threads, precision=prec)
        out[name] = {"e2e": n_cases / (time.perf_counter() - t0), "unit": UNIT}
    for name in ("tf32x3", "int8"):
        worst, same = {}, 0
        for g, r in zip(res[name], res["fp64"]):
            if g.rc != 0 or r.rc != 0:
                raise RuntimeError("precision-stress solve failed")
            nc = min(g.n_coef, r.n_coef)
            err = {"gc": _relmax(g.gc[:, :nc], r.gc[:, :nc]), "gc_l": _relmax(g.gc_l[:, :, :nc], r.gc_l[:, :, :nc])}
            if g.n_coef == r.n_coef:
                same += 1
                err.update(pf=_relmax(g.pf, r.pf), pf_l=_relmax(g.pf_l, r.pf_l))
            for k in ("cext", "csca", "cbak", "g"):
                err[k] = _relmax(g.scalars[k], r.scalars[k])
            for k, v in err.items():
                worst[k] = max(worst.get(k, 0.0), float(v))
        out[name]["error_vs_fp64"] = {"max_rel_err": worst, "cases_with_same_n_coef": same,
                                      "metric": "max over cases of max|form - fp64| / max|fp64| per output array"}
    return out


def save_reweight_measurement(lib, reps: int = 10) -> dict:
    """A retrieval loop on the cloud-droplet case without index1 derivatives:
    one save_control 1 solve, then save_control 2 calls that re-weight its
    per-radius kernels for new effective variances, the kernels staying on
    the device between calls; also one call whose kernels changed (uploaded)."""
    import dataclasses
    case = dataclasses.replace(single_case(), derivs=abi.deriv_unit("a1", "a2"), save_control=1)
    blk = abi.InputBlock(case)
    out = abi.lmie_out_data()
    t0 = time.perf_counter()
    if lib.lmie_solution(C.byref(blk.s), C.byref(out), 1, 0, 16, 0) != 0:
        raise RuntimeError("save_control 1 solve failed")
    t_full = time.perf_counter() - t0
    h0, m0 = C.c_longlong(), C.c_longlong()
    lib.lmieb_save_cache_stats(C.byref(h0), C.byref(m0))
    times = []
    for i in range(reps):
        blk2 = abi.InputBlock(dataclasses.replace(case, a2=0.1 + 0.002 * (i + 1), save_control=2))
        t0 = time.perf_counter()
        if lib.lmie_solution(C.byref(blk2.s), C.byref(out), 0, 0, 16, 0) != 0:
            raise RuntimeError("save_control 2 solve failed")
        times.append(time.perf_counter() - t0)
    h1, m1 = C.c_longlong(), C.c_longlong()
    lib.lmieb_save_cache_stats(C.byref(h1), C.byref(m1))
    # one call whose kernels differ from the kept set (one value changed, then restored)
    keep = out.save2[0][0][0]
    out.save2[0][0][0] = keep * (1.0 + 2.0 ** -40)
    t0 = time.perf_counter()
    lib.lmie_solution(C.byref(blk2.s), C.byref(out), 0, 0, 16, 0)
    t_miss = time.perf_counter() - t0
    out.save2[0][0][0] = keep
    return {"workload": "cloud droplet (gamma r_eff 10 um, 4x500 radii, 948 Gauss angles), derivatives a1, a2",
            "save_control1_ms": t_full * 1e3, "save_control2_kept_ms": statistics.median(times) * 1e3,
            "save_control2_uploaded_ms": t_miss * 1e3,
            "kept_calls": h1.value - h0.value, "uploaded_calls": m1.value - m0.value}


def adjoint_measurement(lib, steps: int) -> dict:
    import lmie_b200
    p = workloads.adjoint_retrieval()
    for _ in range(2):
        lmie_b200.adjoint(p)
    t0 = time.perf_counter()
    for _ in range(steps):
        r = lmie_b200.adjoint(p)
    dt = (time.perf_counter() - t0) / steps
    # the reference's forward mode on a sample of the per-radius MONO solves
    cpu_lib, kind = _cpu_library()
    rng = np.random.Generator(np.random.PCG64(workloads.SEED))
    n_sample, t_cpu = 0, 0.0
    radii = np.exp(rng.uniform(math.log(p.edges[0]), math.log(p.edges[-1]), 64))
    ks = rng.integers(0, p.n_lambda, 64)
    for r_, k in zip(radii, ks):
        case = abi.Case(dist="mono", lam=float(p.lam[k]), mr=float(p.mr[k]), mi=float(p.mi[k]), a1=float(r_),
                        r1=float(r_), r2=float(r_), n_angles=p.n_angles, accuracy=0.0,
                        derivs=abi.deriv_unit("mr", "mi"))
        t1 = time.perf_counter()
        res = abi.solve(cpu_lib, case, n_threads=1) if kind == "reference" else abi.solve(cpu_lib, case, kind="oracle")
        t_cpu += time.perf_counter() - t1
        if res.rc != 0:
            raise RuntimeError("CPU MONO solve failed")
        n_sample += 1
    per_mono = t_cpu / n_sample
    n_radii = p.n_bins * p.n_quad
    return {
        "workload": f"{p.n_lambda} wavelengths log-spaced 0.34-2.25 um, {p.n_bins} log-spaced bins over "
                    f"0.02-20 um x {p.n_quad} Gauss radii, {p.n_angles} angles, seeded bin weights, mr, mi "
                    "and loss weights; gradient w.r.t. 512 refractive-index parameters + 64 bin weights",
        "ms_per_call": dt * 1e3, "value": p.n_lambda / dt, "unit": "wavelength-solves/s (loss + full gradient)",
        "dtype": "f64", "loss": r["loss"],
        "cpu_forward_mode": {
            "value": 1.0 / (per_mono * n_radii), "unit": "wavelength-solves/s (loss + gradient, 1 core)",
            "kind": kind, "cores": 1,
            "sample": f"{n_sample} seeded per-radius SIZE_DIST_MONO solves (accuracy 0, mr/mi derivatives, "
                      f"{p.n_angles} angles) at {per_mono * 1e3:.2f} ms each, times {n_radii} radii per wavelength"},
    }


def bench_config(world: int, scaling: str) -> dict:
    return {"workload": WORKLOAD, "n_cases": N_CASES, "n_derivs": 4,
            "parallelism": (f"independent batches x{world}" if scaling == "weak" else
                            f"one batch in {world} cost-balanced case ranges"),
            "l2": "flushed (256 MiB write) before every timed device step; "
                  "the batch's working set (~8 GB) exceeds L2 in any case"}


REF_STEP_CASES = 256


def run_reference_arm(args) -> int:
    """The reference's CPU lmie_solution on the host cores.  Step i solves the
    REF_STEP_CASES cases at positions [i m, (i + 1) m) of the batch's seeded
    order (wrapping around), one case per host thread (the faster of the
    reference's two parallel forms on this workload, both measured in the
    warm-up); steps and ms_per_step are the ones that ran."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cases = workloads.batched_uneven(N_CASES)
    order = _seeded_order(N_CASES)
    m = REF_STEP_CASES

    def step_cases(i):
        return [order[(i * m + j) % N_CASES] for j in range(m)]

    radius = None
    for w in range(args.warmup):
        if w == 0:
            radius = cpu_radius_parallel(cases, step_cases(w), 10.0)
        else:
            cpu_case_parallel(cases, step_cases(w))
    times = []
    for i in range(args.steps):
        times.append(cpu_case_parallel(cases, step_cases(args.warmup + i))["seconds"])
    total = sum(times)
    value = m * args.steps / total
    lib, kind = _cpu_library()
    threads = os.cpu_count() or 1
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator)",
        "config": bench_config(args.gpus, "weak"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "cpu_model": cpu_model(),
                         "sample": f"{args.steps} steps of {m} cases each ({m * args.steps} solves, "
                                   f"{total:.1f} s) taken in the batch's seeded order, one case per host "
                                   "thread, lmie_solution(n_threads=1)",
                         "variants": {"radius_parallel": radius}},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def int8_errors(lib, cases, n_threads: int) -> dict:
    """The int8 fixed-point form against the FP64 form over `cases`: per
    output array max|int8 - fp64| / max|fp64|, per derivative slice the same
    over the slice's own maximum, the truncations that agree, the cases
    solved again in FP64."""
    ref = abi.solve_batch(lib, cases, n_threads=n_threads, precision=abi.PRECISION_FP64)
    got = abi.solve_batch(lib, cases, n_threads=n_threads, precision=abi.PRECISION_INT8)
    redo = C.c_longlong()
    lib.lmieb_last_redo(C.byref(redo))
    worst, n_same = {}, 0
    for g, r in zip(got, ref):
        if g.rc != 0 or r.rc != 0:
            raise RuntimeError("solve failed while measuring the int8 error")
        n_same += g.n_coef == r.n_coef
        err = {k: _relmax(g.scalars[k], r.scalars[k]) for k in ("cext", "csca", "cbak", "g")}
        for name in ("gc", "pf", "gc_l", "pf_l"):
            a, b = getattr(g, name), getattr(r, name)
            if b is None:
                continue
            if a.shape != b.shape:
                raise RuntimeError("int8 and fp64 outputs differ in shape")
            err[name] = _relmax(a, b)
            if name.endswith("_l"):
                sl = 0.0
                for i in range(b.shape[0]):
                    for e in range(b.shape[1]):
                        m = float(np.max(np.abs(b[i, e])))
                        if m > 0:
                            sl = max(sl, float(np.max(np.abs(a[i, e] - b[i, e]))) / m)
                err[name + "_per_slice"] = sl
        for k, v in err.items():
            worst[k] = max(worst.get(k, 0.0), float(v))
    return {"cases": len(cases), "max_rel_err": worst, "cases_with_same_n_coef": n_same,
            "solved_again_in_fp64": int(redo.value),
            "metric": "max over cases of max|int8 - fp64| / max|fp64| per output array (*_per_slice: per "
                      "derivative and element over that slice's own maximum)"}


def _peaks() -> dict:
    peaks = ROOT / "MEASURED_PEAKS.json"
    try:
        return json.loads(peaks.read_text()) if peaks.exists() else {}
    except ValueError:
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
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
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
    lib.lmieb_last_redo.argtypes = [C.POINTER(C.c_longlong)]
    lib.lmieb_last_int8_kernel.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
    if lib.lmieb_set_device(local) != 0:
        raise RuntimeError("lmieb_set_device failed")
    threads = max(1, (os.cpu_count() or 1) // max(1, world))
    if args.scaling == "weak":
        # every rank solves its own seeded batch (independent cases)
        cases = workloads.batched_uneven(N_CASES, seed=shard.weak_seed(workloads.SEED, rank))
        n_job = world * N_CASES
    else:
        # the ranks split one batch into cost-balanced contiguous ranges
        allc = workloads.batched_uneven(N_CASES)
        a, b = shard.strong_slice(allc, rank, world)
        cases = allc[a:b]
        n_job = N_CASES
    batch = CBatch(lib, cases)

    def measure(precision: int, steps: int, warmup: int) -> dict:
        """One arithmetic form: autotuned public batch calls on host buffers
        (e2e), then the resident batch re-run on the device with the L2
        flushed before every step (value), with stage times and work."""
        tuned = batch.autotune(threads, precision)
        for _ in range(warmup):
            if batch.solve_batch(threads, precision) != 0:
                raise RuntimeError("lmie_solution_batch2 failed")
        barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            if batch.solve_batch(threads, precision) != 0:
                raise RuntimeError("lmie_solution_batch2 failed")
        barrier()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        hm = (C.c_double * 7)()
        lib.lmieb_last_host_timing(hm, 7)
        lib.lmieb_set_pipeline(1)
        if batch.solve_batch(threads, precision) != 0:
            raise RuntimeError("lmie_solution_batch2 failed")
        flops = (C.c_double * 4)()
        launches = C.c_longlong()
        h2d, d2h = C.c_size_t(), C.c_size_t()
        lib.lmieb_last_work(flops, C.byref(launches), C.byref(h2d), C.byref(d2h))
        redo = C.c_longlong()
        lib.lmieb_last_redo(C.byref(redo))
        ms_total = C.c_double()
        ms_stage = (C.c_double * lmie_b200.N_STAGES)()
        if lib.lmieb_rerun_device(1, 1, C.byref(ms_total), ms_stage) != 0:
            raise RuntimeError("device re-run failed (batch did not fit one sub-batch)")
        barrier()
        if lib.lmieb_rerun_device(steps, 1, C.byref(ms_total), ms_stage) != 0:
            raise RuntimeError("device re-run failed")
        barrier()
        dev_ms = max_over_ranks(ms_total.value)
        ops, k3 = C.c_double(), C.c_double()
        lib.lmieb_last_int8_kernel(C.byref(ops), C.byref(k3))
        lib.lmieb_set_pipeline(tuned["pipeline_parts"])
        return {"value": n_job * steps / (dev_ms * 1e-3), "e2e": n_job * steps / e2e_s, "unit": UNIT,
                "ms_per_step": dev_ms / steps,
                "stage_ms": {n: ms_stage[i] / steps for i, n in enumerate(lmie_b200.STAGES)},
                "host_ms": dict(zip(("prepare", "pack", "device_and_copies", "unpack", "scatter", "device_span",
                                     "device_sum_of_parts"), list(hm))),
                "autotuned": tuned, "flops": list(flops), "launches": int(launches.value),
                "h2d": int(h2d.value), "d2h": int(d2h.value), "solved_again_in_fp64": int(redo.value),
                "int8_ops": ops.value, "int8_kernel_ms": k3.value / steps}

    clocks = ClockSampler(local)
    clocks.start()
    m8 = measure(abi.PRECISION_INT8, args.steps, args.warmup)
    m64 = measure(abi.PRECISION_FP64, args.steps, 2)
    mtf = measure(abi.PRECISION_TF32X3, max(3, args.steps // 2), 2)
    clk = clocks.stop()

    peaks = _peaks()
    bf16 = peaks.get("bf16_tflops")
    fp64_peak = C.c_double()
    lib.lmieb_fp64_peak(C.byref(fp64_peak))
    f_ang = m8["flops"][0]
    k3_ms = m8["int8_kernel_ms"]
    tops = m8["int8_ops"] / (k3_ms * 1e-3) / 1e12 if k3_ms > 0 else None
    int8_peak = 2.0 * float(bf16) if bf16 else None
    roofline = {
        "kernel": "k_angular_oz (S1/S2 contraction as exact int8 fixed point: tcgen05.mma kind::i8, A digits in "
                  "tensor memory, 21 digit products per chunk of 32 orders, int32 accumulation)",
        "bound": "tensor", "achieved": tops, "peak": int8_peak, "unit": "TOPS",
        "frac": (tops / int8_peak) if (tops and int8_peak) else None,
        "traffic": ANGULAR_TRAFFIC.get("int8"),
        "peak_source": "dense int8 = 2x the measured bf16 burst in MEASURED_PEAKS.json (of measured)",
        "ops_per_launch": m8["int8_ops"], "ms_per_launch": k3_ms,
        "fp64_equivalent_tflops": f_ang / (k3_ms * 1e-3) / 1e12 if k3_ms > 0 else None,
        "fp64_equivalent_note": "algorithmic S1/S2 flops (8 per angle, order, radius, Mie column) per second "
                                "of this kernel, against the FP64 FMA peak below",
        "fp64_fma_peak_tflops": fp64_peak.value}
    ang64 = m64["stage_ms"]["angular"]
    fp64 = {k: m64[k] for k in ("value", "e2e", "unit", "ms_per_step", "stage_ms", "host_ms", "autotuned")}
    fp64["roofline"] = {
        "kernel": "k_angular (S1/S2 accumulation + phase-matrix forms, FP64)", "bound": "fp64",
        "achieved": m64["flops"][0] / (ang64 * 1e-3) / 1e12 if ang64 > 0 else None, "peak": fp64_peak.value,
        "unit": "TFLOP/s", "traffic": ANGULAR_TRAFFIC["fp64"],
        "frac": (m64["flops"][0] / (ang64 * 1e-3) / 1e12 / fp64_peak.value) if ang64 > 0 else None,
        "peak_source": "live FP64 FMA microbenchmark (lmieb_fp64_peak)"}

    single = split = plain = adj = stress = reweight = errs8 = None
    if rank == 0:
        errs8 = int8_errors(lib, cases, threads)
        split = {k: mtf[k] for k in ("value", "e2e", "unit", "ms_per_step", "stage_ms", "autotuned")}
        split["dtype"] = "f64 with tf32x3 angular contraction (fp32 accumulation in segments of 32 orders)"
        split["error_vs_fp64"] = split_errors(lib, cases[:256], threads)
        tang = mtf["stage_ms"]["angular"]
        tc_tflops = 3 * m64["flops"][0] / (tang * 1e-3) / 1e12 if tang > 0 else None
        split["roofline"] = {
            "kernel": "k_angular_tc (tcgen05.mma kind::tf32, 3 products per operand pair)", "bound": "tensor",
            "achieved": tc_tflops, "peak": float(bf16) / 2 if bf16 else None, "unit": "TFLOP/s",
            "frac": (tc_tflops / (float(bf16) / 2)) if (tc_tflops and bf16) else None,
            "traffic": ANGULAR_TRAFFIC["tf32x3"],
            "peak_source": "dense tf32 = half of the measured bf16 burst in MEASURED_PEAKS.json"}
        # the plain form on the same cases as the batched numbers
        batch.solve_each(threads, 16)
        t1 = time.perf_counter()
        if batch.solve_each(threads) != 0:
            raise RuntimeError("lmie_solution failed")
        plain_s = time.perf_counter() - t1
        plain = {"value": len(cases) / plain_s, "unit": UNIT, "dtype": "f64",
                 "sample": f"all {len(cases)} cases of the batch, one lmie_solution() call each"}
        adj = adjoint_measurement(lib, 5)
        stress = precision_stress_measurement(lib, threads)
        reweight = save_reweight_measurement(lib)

        one = CBatch(lib, [single_case()])
        for _ in range(3):
            one.solve_each(1)
        t1 = time.perf_counter()
        for _ in range(10):
            one.solve_each(1)
        single_e2e = 10 / (time.perf_counter() - t1)
        ms_total = C.c_double()
        ms_stage = (C.c_double * lmie_b200.N_STAGES)()
        lib.lmieb_rerun_device(2, 1, C.byref(ms_total), ms_stage)
        lib.lmieb_rerun_device(10, 1, C.byref(ms_total), ms_stage)
        single = {"workload": "cloud droplet: gamma r_eff=10um v_eff=0.1, 4x500 radii, x_max~436, 4 derivatives",
                  "value": 10 / (ms_total.value * 1e-3), "e2e": single_e2e, "unit": UNIT,
                  "stage_ms": {n: ms_stage[i] / 10 for i, n in enumerate(lmie_b200.STAGES)}}

    if rank == 0:
        cpu = cpu_baseline(cases, 20.0) if world == 1 else None
        line = {
            "metric": METRIC, "value": m8["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": m8["ms_per_step"], "higher_is_better": True,
            "scaling": args.scaling, "vs_baseline": None,
            "dtype": "f64 (angular contraction as exact int8 fixed point, within 1e-9 of f64)",
            "data": ("synthetic (seeded generator, rank r uses seed + r)" if args.scaling == "weak" else
                     "synthetic (seeded generator, one batch split by estimated cost over the ranks)"),
            "config": bench_config(world, args.scaling),
            "path": "lmie_solution_batch2(..., LMIEB_PRECISION_INT8)",
            "autotuned": m8["autotuned"],
            "e2e": {"value": m8["e2e"], "unit": UNIT, "h2d_bytes_per_step": m8["h2d"],
                    "d2h_bytes_per_step": m8["d2h"], "host_threads": threads},
            "gpu_launches": m8["launches"] * args.steps,
            "roofline": roofline,
            "stage_ms": m8["stage_ms"],
            "host_ms": m8["host_ms"],
            "solved_again_in_fp64_per_step": m8["solved_again_in_fp64"],
            "int8_error_vs_fp64": errs8,
            "fp64": fp64,
            "split_tf32x3": split,
            "plain": plain,
            "adjoint": adj,
            "precision_stress": stress,
            "save_reweight": reweight,
            "single_case": single,
            "clocks": clk,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_profile(args) -> int:
    """Only the device work of one path, `warmup` + `steps` times, for launch
    lists and kernel captures under a profiler (prints no bench line)."""
    import lmie_b200
    lib = lmie_b200.library()
    if args.profile == "adjoint":
        p = workloads.adjoint_retrieval()
        if args.cases < N_CASES:
            p = workloads.adjoint_retrieval(n_lambda=max(1, 256 * args.cases // N_CASES))
        for _ in range(args.warmup + args.steps):
            lmie_b200.adjoint(p)
        print(f"profiled adjoint: {p.n_lambda} wavelengths, {args.warmup} + {args.steps} calls")
        return 0
    precision = {"tf32x3": abi.PRECISION_TF32X3, "int8": abi.PRECISION_INT8}.get(args.profile, abi.PRECISION_FP64)
    lib.lmieb_set_pipeline(1)            # one sub-batch: the launches the device-time `value` measures
    batch = CBatch(lib, workloads.batched_uneven(args.cases))
    threads = os.cpu_count() or 1
    for _ in range(args.warmup + args.steps):
        if batch.solve_batch(threads, precision) != 0:
            raise RuntimeError("lmie_solution_batch2 failed")
    print(f"profiled {args.profile}: {args.cases} cases, {args.warmup} + {args.steps} batch calls")
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--profile", choices=("fp64", "tf32x3", "int8", "adjoint"), default=None,
                    help="run only this path's batch calls (for profilers); no bench line")
    ap.add_argument("--cases", type=int, default=N_CASES, help="cases of the profiled batch")
    ap.add_argument("--scaling", choices=("weak", "strong"), default="weak",
                    help="weak: each rank its own 4096-case batch; strong: the ranks split one batch")
    args = ap.parse_args(argv)
    if args.profile:
        return run_profile(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
