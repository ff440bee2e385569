#!/usr/bin/env python
"""Benchmark: dipole-solves/s of the coupled-dipole solve at N = 30,000.

Workload (one "step" = one converged solve from x0 = 0 at one wavelength):
Au cuboid 60 x 50 x 10 nm on a cell-centred 1 nm lattice (N = 30,000),
vacuum, RRCM polarisabilities from the Johnson & Christy table, FCD with
cell = 1 nm, +z x-polarised plane wave, restarted GMRES(30) to 1e-8 on the
FP64 residual, on-the-fly operator.  The product mode is FP32+refine (FP32
operator inside FP64 Arnoldi/Givens, FP64 restart residuals); one plain FP64
solve at the first wavelength is timed beside it for the speed-up and for
the C_ext error gate (<= 1e-6).

value  = N * solves (all ranks) / max-over-ranks device time, inputs
         resident in HBM.
e2e    = the same metric through the public CdaSolver API with host arrays
         (positions, polarisabilities in; moments out) every step.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Multi-GPU runs are independent replicas (weak scaling): each rank solves its
own wavelengths, no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "dipole-solves/s at N=30k: FP32+refine vs FP64 plain, C_ext rel err <=1e-6"
UNIT = "dipole-solves/s"
FLOPS_PER_PAIR = 86.0  # canonical point-dipole pair cost (FMA = 2), + 1 rsqrt + 1 sincos


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--tol", type=float, default=1e-8)
    p.add_argument("--max-iter", type=int, default=3000)
    p.add_argument("--wavelengths", default="520,650,800")
    p.add_argument("--size", default="60,50,10", help="cuboid size in nm (1 nm lattice)")
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    return p.parse_args()


def workload_config(args, n):
    size = [float(v) for v in args.size.split(",")]
    return {"workload": f"Au cuboid {size[0]:g}x{size[1]:g}x{size[2]:g} nm, 1 nm cell-centred "
                        f"lattice, N={n}, FCD cell 1 nm, RRCM, vacuum, x-pol +z",
            "n_dipoles": n, "solver": "GMRES(30)", "tol": args.tol,
            "wavelengths_nm": [float(v) for v in args.wavelengths.split(",")],
            "operator": "on-the-fly", "l2": "inputs+operator traffic > L2 not applicable: "
            "compute-bound pair kernel; x (0.7 MB) is L2-resident by design",
            "data": "synthetic"}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, FileNotFoundError):
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if s[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


# ---------------------------------------------------------------- inputs
def build_inputs(args, lams):
    from lumina_b200 import configs
    size = tuple(float(v) for v in args.size.split(","))
    base = configs.cuboid_au(size, 1.0, lams[0])
    per = []
    for lam in lams:
        w = configs.au_workload(base.name, base.positions, 1.0, lam)
        per.append(w)
    return base, per


def cpu_baseline(w, matvecs_per_solve, seconds, threads=0):
    """Oracle (FP64 on-the-fly matvec + GMRES restatement) on the host cores:
    a bounded sample of rows of one matvec, scaled to one solve with the
    reference-equivalent matvec count of the GPU solve."""
    from oracle import oracle as orc
    n = w.n
    x = np.random.default_rng(7).standard_normal(3 * n) * (1 + 1j)
    nt = threads or orc.max_threads()
    rows = max(1, min(n, 64))
    t0 = time.perf_counter()
    orc.matvec_onthefly_rows(w.positions, w.alpha, x, w.k, True, w.cell_size, 0, rows, nt)
    dt = time.perf_counter() - t0
    # grow the sample to ~`seconds` of work
    rows = int(min(n, max(rows, rows * seconds / max(dt, 1e-3))))
    t0 = time.perf_counter()
    orc.matvec_onthefly_rows(w.positions, w.alpha, x, w.k, True, w.cell_size, 0, rows, nt)
    dt = time.perf_counter() - t0
    t_matvec = dt * n / rows
    t_solve = t_matvec * matvecs_per_solve
    return {"value": n / t_solve, "unit": UNIT, "cores": nt, "kind": "port",
            "sample": f"{rows} of {n} rows of one FP64 on-the-fly matvec ({dt:.1f} s), scaled "
                      f"to {matvecs_per_solve} matvecs per solve",
            "matvec_seconds": t_matvec, "cpu": _cpu_model()}


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    lams = [float(v) for v in args.wavelengths.split(",")]
    base, per = build_inputs(args, lams)
    # matvecs per solve: the reference's GMRES at this configuration needs the
    # same Krylov iterations as the FP64 device solve (same algorithm); the
    # sample below is scaled by a fixed, stated count.
    mv = int(os.environ.get("LUMINA_REF_MATVECS", "0")) or _ref_matvec_count(base.n)
    times = []
    for s in range(args.warmup + args.steps):
        r = cpu_baseline(per[s % len(per)], mv, min(args.cpu_seconds, 20.0))
        if s >= args.warmup:
            times.append(base.n / r["value"])
    t = sum(times)
    val = base.n * args.steps / t
    line = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": workload_config(args, base.n),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": r["cores"], "kind": "port",
                             "sample": r["sample"]},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _ref_matvec_count(n):
    # GMRES(30) iterations measured for this workload on the device (FP64,
    # 520/650/800 nm) are recorded in profiles/; without them use 1000
    path = os.path.join(ROOT, "profiles", "solve_counts_cuboid30k.json")
    try:
        with open(path) as f:
            return int(json.load(f)["matvecs_reference_fp64"])
    except (OSError, KeyError, ValueError):
        return 1000


# ---------------------------------------------------------------- our arm
def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import lumina_b200 as lb
    from lumina_b200 import _ffi

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from lumina_b200 import replicas
    lams_all = [float(v) for v in args.wavelengths.split(",")]
    # replicas (weak scaling): every rank solves K steps over the wavelength
    # list, starting at its own offset; no collective on the data path
    lams = replicas.rotated(lams_all, rank, world)
    base, per = build_inputs(args, lams)
    n = base.n
    bk = lb.CudaBackend(local)
    fp32_peak, fp64_peak = bk.measure_fma_peak()
    # one dedicated stream for torch's events/copies and the library's kernels
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    inv = [lb.invert_polarisability(w.alpha) for w in per]
    rhs = [lb.incident_field(w.positions, w.k, lb.IncidentField()) for w in per]
    sess = bk.create_onthefly_session(base.positions, inv[0], per[0].k, True, 1.0)
    sess.set_stream(stream.cuda_stream)
    b_dev = [torch.from_numpy(r).to("cuda") for r in rhs]
    x_dev = [torch.zeros(3 * n, dtype=torch.complex128, device="cuda") for _ in per]
    torch.cuda.synchronize()

    def step(s, mode="fp32_refine", out=None):
        i = s % len(per)
        sess.set_wavelength(per[i].k, inv[i])
        x = out if out is not None else x_dev[i]
        return sess.solve_device(b_dev[i].data_ptr(), x.data_ptr(), args.tol, args.max_iter,
                                 30, mode, stream.cuda_stream)

    for s in range(args.warmup):
        step(s)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sess.profile(True)
    infos = []
    launches0 = _ffi.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for s in range(args.steps):
            infos.append(step(s))
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = _ffi.launch_count() - launches0
    dt_ms = ev0.elapsed_time(ev1)
    k32, ms32 = sess.kernel_time("fp32")
    k64, ms64 = sess.kernel_time("fp64")
    sess.profile(False)
    units, t_max_s = replicas.reduce_job(n * args.steps, dt_ms * 1e-3, dist, "cuda")
    t_max = t_max_s * 1e3
    value = units / t_max_s

    # Plain FP64 GMRES(30) at every timed wavelength (same solves, same
    # tolerance) for the speed-up and the C_ext gate against the timed
    # FP32+refine solutions.
    fp64 = None
    if not args.no_fp64:
        inc = lb.IncidentField()
        x64 = torch.zeros(3 * n, dtype=torch.complex128, device="cuda")
        per_lam = []
        ms64_tot = 0.0
        for i in range(min(len(per), args.steps)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            info64 = step(i, "fp64", out=x64)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            ms64_tot += ms
            cs32 = lb.cross_sections(base.positions, inv[i], x_dev[i].cpu().numpy(), per[i].k, inc)
            cs64 = lb.cross_sections(base.positions, inv[i], x64.cpu().numpy(), per[i].k, inc)
            per_lam.append({"wavelength_nm": lams[i], "ms_fp64": ms,
                            "ms_fp32_refine": infos[i]["seconds"] * 1e3,
                            "iterations_fp64": info64["iterations"],
                            "iterations_fp32_refine": infos[i]["iterations"],
                            "matvecs_reference": info64["matvecs_reference"],
                            "cext_fp64": cs64[0], "cext_fp32_refine": cs32[0],
                            "cext_rel_err": abs(cs32[0] - cs64[0]) / abs(cs64[0]),
                            "cabs_rel_err": abs(cs32[1] - cs64[1]) / abs(cs64[1])})
        nl = len(per_lam)
        fp32_ms = sum(p["ms_fp32_refine"] for p in per_lam)
        fp64 = {"value": n * nl / (ms64_tot * 1e-3), "unit": UNIT,
                "ms_per_solve": ms64_tot / nl, "fp32_refine_ms_per_solve": fp32_ms / nl,
                "speedup_same_solves": ms64_tot / fp32_ms,
                "max_cext_rel_err": max(p["cext_rel_err"] for p in per_lam),
                "max_cabs_rel_err": max(p["cabs_rel_err"] for p in per_lam),
                "per_wavelength": per_lam}

    # e2e through the public API with host arrays
    e2e = None
    if not args.no_e2e:
        solver = lb.CdaSolver(backend=bk, iterative_threshold=0, use_fcd=True, cell_size=1.0,
                              matrix_memory_budget=0, precision="fp32_refine")
        params = lb.SimulationParams(solver_tolerance=args.tol, max_iterations=args.max_iter)
        ds = [lb.DipoleSet(w.positions, w.alpha) for w in per]
        solver.compute_cross_sections(ds[0], lams[0], params)  # warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in range(args.steps):
            solver.compute_cross_sections(ds[s % len(ds)], lams[s % len(lams)], params)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        e2e_units, dt = replicas.reduce_job(n * args.steps, dt, dist, "cuda")
        e2e = {"value": e2e_units / dt, "unit": UNIT,
               "h2d_bytes_per_step": n * 3 * 8 + n * 9 * 16 + 3 * n * 16,
               "d2h_bytes_per_step": 3 * n * 16}

    # roofline of the dominant kernel (the FP32 dense pair kernel)
    # Launches enqueued after a cycle converged exit at once (a few us each);
    # the average is taken over the operator applications actually performed.
    pairs = float(n) * (n - 1)
    real32 = sum(i["matvecs_fp32"] for i in infos) or 1
    real64 = sum(i["matvecs_fp64"] for i in infos) or 1
    avg32 = ms32 / real32
    avg64 = ms64 / real64
    achieved = pairs * FLOPS_PER_PAIR / (avg32 * 1e-3) / 1e12
    peak = fp32_peak / 1e3
    roof = {"bound": "fp32", "kernel": "otf_pairs_f32", "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
            "peak_source": "FP32 FMA-chain microbenchmark in this run (MEASURED_PEAKS.json has "
                           "HBM and bf16 only); of measured",
            "traffic": _traffic_from_profiles(), "launches": k32, "applications": real32,
            "avg_launch_ms": avg32, "flops_per_launch": pairs * FLOPS_PER_PAIR,
            "kernel_config": sess.kernel_config(),
            "fp64_kernel": {"launches": k64, "applications": real64, "avg_launch_ms": avg64,
                            "achieved_tflops": pairs * FLOPS_PER_PAIR / (avg64 * 1e-3) / 1e12,
                            "peak_tflops": fp64_peak / 1e3}}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # the reference's FP64 GMRES(30) needs the same Arnoldi steps as the
        # device FP64 solve; scale by the mean reference-equivalent count
        if fp64:
            mv_ref = int(round(statistics.mean(p["matvecs_reference"] for p in fp64["per_wavelength"])))
        else:
            mv_ref = int(round(statistics.mean(i["matvecs_reference"] for i in infos)))
        cpu = cpu_baseline(per[0], mv_ref, args.cpu_seconds)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic", "config": workload_config(args, n), "mode": "fp32_refine",
            "clocks": clk.summary(), "e2e": e2e, "gpu_launches": launches, "roofline": roof,
            "cpu_baseline": cpu, "fp64_plain": fp64,
            "speedup_vs_fp64_plain": fp64["speedup_same_solves"] if fp64 else None,
            "solves": [{k: v for k, v in i.items()} for i in infos]}
    print(json.dumps(line), flush=True)
    return 0


def _traffic_from_profiles():
    path = os.path.join(ROOT, "profiles", "otf_pairs_f32_cuboid30k.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1])
    except (OSError, ValueError):
        pass
    return None


if __name__ == "__main__":
    sys.exit(main())
