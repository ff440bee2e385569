#!/usr/bin/env python
"""Benchmark: dipole-solves/s of the coupled-dipole solve at N = 30,000.

Workload: Au cuboid 60 x 50 x 10 nm on a cell-centred 1 nm lattice
(N = 30,000), vacuum, RRCM polarisabilities from the Johnson & Christy table,
FCD with cell = 1 nm, +z x-polarised plane wave, restarted GMRES(30) from
x0 = 0 to 1e-8 on the FP64 residual, on-the-fly operator, over the 51-point
400-900 nm sweep (every 10 nm).  The product mode is FP32+refine (FP32
operator inside FP64 Arnoldi/Givens, FP64 restart residuals).

Steps: the K timed steps partition the sweep (repeated ceil(K/51) times):
step s solves sweep entries s, s+K, s+2K, ..., so every wavelength is solved
equally often and the value does not depend on K.  Plain FP64 solves of the
same wavelengths give the speed-up and the per-wavelength C_ext / C_abs
error (gate <= 1e-6); the solutions are also compared with the full FP64
oracle solves stored in tests/golden/cuboid30k_oracle.json.

value  = N * solves (all ranks) / max-over-ranks device time, inputs
         resident in HBM.
e2e    = the same metric through the public CdaSolver API with host arrays
         (positions, polarisabilities in; moments out) for the same solves.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Multi-GPU runs are independent replicas (weak scaling): each rank solves the
whole sweep from its own offset, no collective on the data path.
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
    p.add_argument("--max-iter", type=int, default=5000)
    p.add_argument("--wavelengths", default="sweep",
                   help="'sweep' (51 points, 400-900 nm every 10 nm) or a comma list in nm")
    p.add_argument("--size", default="60,50,10", help="cuboid size in nm (1 nm lattice)")
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--fp64-stride", type=int, default=1,
                   help="plain-FP64 comparison solves at every S-th wavelength")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-oracle-solve", action="store_true",
                   help="reference arm: skip the full oracle solve at 520 nm")
    p.add_argument("--workload", default="cuboid",
                   choices=["cuboid", "clusters", "dimer", "metasurface", "cached", "fields",
                            "fft", "directions", "sommerfeld", "harmonic"],
                   help="cuboid: the headline N=30k sweep; clusters: 256 Drude ellipsoids x 2 "
                        "polarisations in one batch; dimer: helix-dimer adjoint gradients; "
                        "metasurface: periodic Ewald + substrate sweep; cached: the assembled "
                        "3N x 3N matrix, single-vector GEMV and multi-RHS tensor-core product; "
                        "fields: near-field map and far field from solved moments; fft: the "
                        "headline cuboid through the block-Toeplitz FFT operator; directions: "
                        "many incidence directions of one cached matrix on the tensor cores; "
                        "sommerfeld: an Au sphere above glass with the Sommerfeld substrate; "
                        "harmonic: second-harmonic response of the headline cuboid")
    p.add_argument("--nrhs", type=int, default=128, help="right-hand sides (cached workload)")
    p.add_argument("--clusters", type=int, default=256)
    p.add_argument("--spacing", type=float, default=None)
    return p.parse_args()


# The wavelength sweep of the headline configuration: 51 points, 400-900 nm.
SWEEP_NM = [400.0 + 10.0 * i for i in range(51)]
GOLD_TABLE_END_NM = 892.0


def wavelength_list(args, default="sweep"):
    spec = args.wavelengths if args.wavelengths != "sweep" else default
    if spec == "sweep":
        return list(SWEEP_NM)
    return [float(v) for v in spec.split(",")]


def sweep_plan(n_lams, steps):
    """Partition of the timed solves over the K steps: the wavelength list is
    repeated reps = ceil(K / L) times and step s solves its entries s, s + K,
    s + 2K, ...  Every wavelength is solved exactly reps times whatever K is,
    so each is weighted equally and --steps does not change the value."""
    reps = max(1, -(-steps // n_lams))
    total = n_lams * reps
    return [[j % n_lams for j in range(s, total, steps)] for s in range(steps)], reps


def warmup_plan(n_lams, warmup):
    """Warm-up step w solves one wavelength, spread over the list."""
    return [[(w * max(1, n_lams // 5)) % n_lams] for w in range(warmup)]


def workload_config(args, n, lams=None):
    size = [float(v) for v in args.size.split(",")]
    lams = lams if lams is not None else wavelength_list(args)
    cfg = {"workload": f"Au cuboid {size[0]:g}x{size[1]:g}x{size[2]:g} nm, 1 nm cell-centred "
                       f"lattice, N={n}, FCD cell 1 nm, RRCM (J&C gold), vacuum, x-pol +z",
           "n_dipoles": n, "solver": "GMRES(30)", "tol": args.tol,
           "wavelengths_nm": lams if len(lams) <= 8 else
           {"first": lams[0], "last": lams[-1], "count": len(lams),
            "step": lams[1] - lams[0]},
           "operator": "on-the-fly", "l2": "flushed: 256 MB written before each timed solve "
           "(outside its events); within a solve x (0.7 MB) stays L2-resident by design",
           "data": "synthetic"}
    if any(l > GOLD_TABLE_END_NM for l in lams):
        cfg["gold_beyond_table"] = (f"J&C gold ends at {GOLD_TABLE_END_NM:g} nm; wavelengths "
                                    "past it use the natural spline's last interval extended "
                                    "(its boundary cubic)")
    return cfg


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


def cpu_matvec_sample(w, seconds, threads=0, periodic=None):
    """Seconds of one FP64 on-the-fly oracle matvec (assembly.rs:209-318 with
    FCD; with ``periodic`` its Ewald lattice, Bloch vector and substrate
    image) on the host cores, from a bounded sample of rows grown to about
    ``seconds`` of work.  The cost does not depend on the wavelength."""
    from oracle import oracle as orc
    n = w.n
    x = np.random.default_rng(7).standard_normal(3 * n) * (1 + 1j)
    nt = threads or orc.max_threads()

    def run(rows):
        if periodic is None:
            orc.matvec_onthefly_rows(w.positions, w.alpha, x, w.k, True, w.cell_size, 0, rows,
                                     nt)
        else:
            orc.matvec_onthefly_rows_ex(w.positions, w.alpha, x, w.k, True, w.cell_size, 0, rows,
                                        lattice=periodic.lattice, k_bloch=periodic.k_bloch,
                                        substrate=periodic.substrate, nthreads=nt)

    rows = max(1, min(n, 64 if periodic is None else nt))
    t0 = time.perf_counter()
    run(rows)
    dt = time.perf_counter() - t0
    rows = int(min(n, max(rows, rows * seconds / max(dt, 1e-3))))
    t0 = time.perf_counter()
    run(rows)
    dt = time.perf_counter() - t0
    return dt * n / rows, rows, dt, nt


def cpu_baseline(w, counts, seconds, threads=0):
    """The oracle (FP64 on-the-fly matvec + GMRES restatement) on the host
    cores: a bounded sample of rows of one matvec, scaled by the operator
    applications the reference's GMRES(30) issues at each wavelength
    (``counts``, one per solve).  An extrapolation, stated as such."""
    t_mv, rows, dt, nt = cpu_matvec_sample(w, seconds, threads)
    n = w.n
    t_total = t_mv * float(sum(counts))
    return {"value": n * len(counts) / t_total, "unit": UNIT, "cores": nt, "kind": "port",
            "sample": f"{rows} of {n} rows of one FP64 on-the-fly oracle matvec ({dt:.1f} s), "
                      f"scaled by the reference GMRES(30)'s operator applications: "
                      f"{int(sum(counts))} over {len(counts)} solves",
            "extrapolated": True, "matvec_seconds": t_mv, "cpu": _cpu_model()}


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


ORACLE_FIXTURE = os.path.join(ROOT, "tests", "golden", "cuboid30k_oracle.json")
COUNTS_FIXTURE = os.path.join(ROOT, "tests", "golden", "cuboid30k_sweep_counts.json")


def _load_json(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def reference_counts(n, tol):
    """Operator applications of the reference's GMRES(30) per wavelength for
    the N = 30,000 cuboid at tol 1e-8 (iterative.rs:53-159: the Arnoldi
    products plus each cycle's start and end residuals), as counted by the
    plain-FP64 device solve, which runs the same algorithm
    (tests/golden/cuboid30k_sweep_counts.json); None for any other case."""
    data = _load_json(COUNTS_FIXTURE)
    if not data or n != data.get("n_dipoles") or tol != data.get("tol"):
        return None
    return {float(k): int(v) for k, v in data["matvecs_reference"].items()}


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    lams = wavelength_list(args)
    base, per = build_inputs(args, lams)
    n = base.n
    counts = reference_counts(n, args.tol)
    missing = [l for l in lams if counts is None or l not in counts]
    if missing:
        print(json.dumps({"impl": "reference", "metric": METRIC, "unavailable":
                          f"no reference operator-application count for N={n}, tol "
                          f"{args.tol:g} at {len(missing)} wavelengths (e.g. {missing[0]:g} nm); "
                          "the reference arm covers the N=30000 cuboid sweep at tol 1e-8"}),
              flush=True)
        return 0
    # One full oracle FP64 GMRES(30) solve at 520 nm: the measured anchor of
    # the per-wavelength extrapolation below (its operator applications
    # against the count table, its time against the sampled matvec time).
    anchor = None
    if not args.no_oracle_solve and 520.0 in lams and n == 30000:
        from oracle import oracle as orc
        w = per[lams.index(520.0)]
        b = orc.incident_field(w.positions, w.k)
        nt = orc.max_threads()
        t0 = time.perf_counter()
        r = orc.gmres_onthefly(w.positions, w.alpha, b, w.k, True, w.cell_size, tol=args.tol,
                               max_iter=args.max_iter, nthreads=nt)
        secs = time.perf_counter() - t0
        cs = orc.cross_sections(w.positions, w.alpha, r.x, w.k)
        anchor = {"wavelength_nm": 520.0, "measured_s": secs, "threads": nt,
                  "status": r.status, "iterations": r.iterations, "matvecs": r.matvecs,
                  "count_table_matvecs": counts[520.0], "rel_residual": r.rel_residual,
                  "c_ext": cs[0], "c_abs": cs[1]}
    plan, reps = sweep_plan(len(lams), args.steps)
    warm = warmup_plan(len(lams), args.warmup)
    budget = max(2.0, min(args.cpu_seconds, 90.0 / max(1, args.warmup + args.steps)))
    step_s, t_mv_all, nt = [], [], 1
    for s, step in enumerate(warm + plan):
        t_mv, rows, dt, nt = cpu_matvec_sample(per[step[0]], budget)
        if s >= len(warm):
            t_mv_all.append(t_mv)
            step_s.append(sum(t_mv * counts[lams[i]] for i in step))
    t = sum(step_s)
    solves = sum(len(st) for st in plan)
    val = n * solves / t
    t_mv_mean = statistics.mean(t_mv_all)
    if anchor:
        anchor["extrapolated_s"] = t_mv_mean * anchor["matvecs"]
        anchor["measured_over_extrapolated"] = anchor["measured_s"] / anchor["extrapolated_s"]
    sample = (f"each step: a {budget:.0f} s row sample of one FP64 on-the-fly oracle matvec on "
              f"{nt} threads, scaled by the reference GMRES(30)'s operator applications at the "
              f"step's wavelengths ({sum(counts[l] for l in lams) * reps} over the {len(lams)}-point "
              f"sweep x {reps}); extrapolated" +
              ("; anchored by one full oracle solve at 520 nm (oracle_solve)" if anchor else ""))
    line = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": workload_config(args, n, lams),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": nt, "kind": "port",
                             "sample": sample, "extrapolated": True, "cpu": _cpu_model()},
            "matvec_seconds": t_mv_mean, "oracle_solve": anchor,
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- our arm
def main():
    args = parse()
    if args.workload != "cuboid":
        return run_secondary(args)
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
    # replicas (weak scaling): every rank solves the whole sweep, starting at
    # its own offset; no collective on the data path
    lams = replicas.rotated(wavelength_list(args), rank, world)
    nl = len(lams)
    base, per = build_inputs(args, lams)
    n = base.n
    bk = lb.CudaBackend(local)
    fp32_peak, fp64_peak = bk.measure_fma_peak()
    fma2_peak = bk.measure_fma2_peak()
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

    def solve(i, mode="fp32_refine", out=None):
        sess.set_wavelength(per[i].k, inv[i])
        x = out if out is not None else x_dev[i]
        return sess.solve_device(b_dev[i].data_ptr(), x.data_ptr(), args.tol, args.max_iter,
                                 30, mode, stream.cuda_stream)

    plan, reps = sweep_plan(nl, args.steps)
    for step in warmup_plan(nl, args.warmup):
        for i in step:
            solve(i)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sess.profile(True)
    # 256 MB written before every timed solve evicts the 126 MB L2, so no solve
    # starts from operands the previous one left cached; the write sits
    # outside the events that time the solve.
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    launches0 = _ffi.launch_count()
    solves = []  # (wavelength index, info, ms)
    step_ms = []
    with ClockSampler(torch.cuda.current_device()) as clk:
        torch.cuda.synchronize()
        for step in plan:
            t = 0.0
            for i in step:
                flush.zero_()
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ev0.record(stream)
                info = solve(i)
                ev1.record(stream)
                torch.cuda.synchronize()
                ms = ev0.elapsed_time(ev1)
                t += ms
                solves.append((i, info, ms))
            step_ms.append(t)
    launches = _ffi.launch_count() - launches0
    k32, ms32 = sess.kernel_time("fp32")
    k64, ms64 = sess.kernel_time("fp64")
    sess.profile(False)
    dt_ms = sum(step_ms)
    units, t_max_s = replicas.reduce_job(n * len(solves), dt_ms * 1e-3, dist, "cuda")
    value = units / t_max_s
    infos = [s[1] for s in solves]
    ms_lam = {}
    info_lam = {}
    for i, info, ms in solves:
        ms_lam.setdefault(i, []).append(ms)
        info_lam[i] = info

    inc = lb.IncidentField()
    cs32 = {i: lb.cross_sections(base.positions, inv[i], x_dev[i].cpu().numpy(), per[i].k, inc)
            for i in range(nl)}

    # Plain FP64 GMRES(30) at every (or every S-th) wavelength, same tolerance:
    # the speed-up on the same solves and the per-wavelength C_ext / C_abs
    # error of the timed FP32+refine solutions.
    fp64 = None
    x64_keep = {}
    fixture = _load_json(ORACLE_FIXTURE)
    fix_lams = {float(r["wavelength_nm"]) for r in fixture["solves"]} if fixture else set()
    if not args.no_fp64:
        x64 = torch.zeros(3 * n, dtype=torch.complex128, device="cuda")
        rows = []
        t64 = t32 = 0.0
        for i in range(0, nl, max(1, args.fp64_stride)):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            info64 = solve(i, "fp64", out=x64)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            xh = x64.cpu().numpy()
            if lams[i] in fix_lams:
                x64_keep[i] = xh
            c64 = lb.cross_sections(base.positions, inv[i], xh, per[i].k, inc)
            m32 = statistics.mean(ms_lam[i])
            t64 += ms
            t32 += m32
            rows.append({"wavelength_nm": lams[i], "ms_fp64": ms, "ms_fp32_refine": m32,
                         "iterations_fp64": info64["iterations"],
                         "iterations_fp32_refine": info_lam[i]["iterations"],
                         "restarts_fp32_refine": info_lam[i]["restarts"],
                         "matvecs_reference": info64["matvecs_reference"],
                         "cext_fp64": c64[0], "cext_fp32_refine": cs32[i][0],
                         "cext_rel_err": abs(cs32[i][0] - c64[0]) / abs(c64[0]),
                         "cabs_rel_err": abs(cs32[i][1] - c64[1]) / abs(c64[1])})
        fp64 = {"value": n * len(rows) / (t64 * 1e-3), "unit": UNIT,
                "ms_per_solve": t64 / len(rows), "fp32_refine_ms_per_solve": t32 / len(rows),
                "solves": len(rows), "speedup_same_solves": t64 / t32,
                "max_cext_rel_err": max(p["cext_rel_err"] for p in rows),
                "max_cabs_rel_err": max(p["cabs_rel_err"] for p in rows),
                "gate_cext_rel_err_le_1e-6": all(p["cext_rel_err"] <= 1e-6 for p in rows),
                "per_wavelength": rows}

    # C_ext / C_abs / moments against the full FP64 oracle solves stored in
    # tests/golden/cuboid30k_oracle.json (the precision gate, literally).
    oracle_pin = None
    if fixture and n == fixture["solves"][0]["n_dipoles"]:
        oracle_pin = []
        for rec in fixture["solves"]:
            lam = float(rec["wavelength_nm"])
            if lam not in lams or abs(rec["tol"] - args.tol) > 0:
                continue
            i = lams.index(lam)
            idx = np.asarray(rec["sample_dipoles"])
            pref = (np.asarray(rec["sample_moments_re"]) +
                    1j * np.asarray(rec["sample_moments_im"])).reshape(-1, 3)
            ent = {"wavelength_nm": lam, "oracle_c_ext": rec["c_ext"],
                   "oracle_iterations": rec["iterations"], "oracle_matvecs": rec["matvecs"],
                   "oracle_solve_measured_s": rec["seconds"], "oracle_threads": rec["threads"],
                   "oracle_cpu": rec["cpu"]}
            for tag, x in (("fp32_refine", x_dev[i].cpu().numpy()), ("fp64", x64_keep.get(i))):
                if x is None:
                    continue
                cs = lb.cross_sections(base.positions, inv[i], x, per[i].k, inc)
                p = x.reshape(-1, 3)[idx]
                ent[f"cext_rel_err_{tag}"] = abs(cs[0] - rec["c_ext"]) / abs(rec["c_ext"])
                ent[f"cabs_rel_err_{tag}"] = abs(cs[1] - rec["c_abs"]) / abs(rec["c_abs"])
                ent[f"moments_rel_err_{tag}"] = float(np.max(np.abs(p - pref)) /
                                                      np.max(np.abs(pref)))
            oracle_pin.append(ent)

    # e2e through the public API with host arrays, over the same solves
    e2e = None
    if not args.no_e2e:
        # the on-the-fly operator, as the device-timed value (the solver's FFT
        # branch has its own line: --workload fft)
        solver = lb.CdaSolver(backend=bk, iterative_threshold=0, use_fcd=True, cell_size=1.0,
                              matrix_memory_budget=0, precision="fp32_refine", use_fft=False)
        params = lb.SimulationParams(solver_tolerance=args.tol, max_iterations=args.max_iter)
        ds = [lb.DipoleSet(w.positions, w.alpha) for w in per]
        solver.compute_cross_sections(ds[plan[0][0]], lams[plan[0][0]], params)  # warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for step in plan:
            for i in step:
                solver.compute_cross_sections(ds[i], lams[i], params)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        solver.close()
        e2e_units, dt = replicas.reduce_job(n * len(solves), dt, dist, "cuda")
        per_solve_h2d = n * 3 * 8 + n * 9 * 16 + 3 * n * 16
        per_solve_d2h = 3 * n * 16
        spp = len(solves) / args.steps
        e2e = {"value": e2e_units / dt, "unit": UNIT,
               "h2d_bytes_per_step": int(round(per_solve_h2d * spp)),
               "d2h_bytes_per_step": int(round(per_solve_d2h * spp))}

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
    kcfg = sess.kernel_config()
    kname = "otf_pairs_f32_sym" if kcfg.get("f32_sym") else "otf_pairs_f32"
    k64name = "otf_pairs_f64_sym" if kcfg.get("f64_sym") else "otf_pairs_f64"
    a64 = pairs * FLOPS_PER_PAIR / (avg64 * 1e-3) / 1e12
    roof = {"bound": "fp32", "kernel": kname, "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
            "peak_source": "FP32 FMA-chain microbenchmark in this run (MEASURED_PEAKS.json has "
                           "HBM and bf16 only); of measured",
            "traffic": _traffic_from_profiles(kname), "launches": k32, "applications": real32,
            "avg_launch_ms": avg32, "flops_per_launch": pairs * FLOPS_PER_PAIR,
            "kernel_config": kcfg,
            "packed_fma2_peak_tflops": fma2_peak / 1e3,
            "frac_of_packed_fma2_peak": achieved / (fma2_peak / 1e3) if fma2_peak else None,
            "fp64_kernel": {"kernel": k64name, "launches": k64, "applications": real64,
                            "avg_launch_ms": avg64, "achieved_tflops": a64,
                            "peak_tflops": fp64_peak / 1e3,
                            "frac": a64 / (fp64_peak / 1e3) if fp64_peak else None}}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # the reference's FP64 GMRES(30) issues the operator applications the
        # device FP64 solve counts (same algorithm); the FP32+refine solves'
        # reference-equivalent counts stand in where no FP64 solve ran
        cnt = {r["wavelength_nm"]: r["matvecs_reference"] for r in (fp64 or {}).get(
            "per_wavelength", [])}
        counts = [cnt.get(lams[i], info["matvecs_reference"]) for i, info, _ in solves]
        cpu = cpu_baseline(per[0], counts, args.cpu_seconds)
        if oracle_pin:
            for ent in oracle_pin:
                ent["oracle_solve_extrapolated_s"] = cpu["matvec_seconds"] * ent["oracle_matvecs"]
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    per_lam = [{"wavelength_nm": lams[i], "ms_fp32_refine": statistics.mean(ms_lam[i]),
                "iterations": info_lam[i]["iterations"], "restarts": info_lam[i]["restarts"],
                "matvecs_fp32": info_lam[i]["matvecs_fp32"],
                "matvecs_fp64": info_lam[i]["matvecs_fp64"],
                "rel_residual": info_lam[i]["rel_residual"],
                "converged": info_lam[i]["converged"], "c_ext": cs32[i][0], "c_abs": cs32[i][1]}
               for i in sorted(ms_lam)]
    # the headline figures quote the 520 nm solve, the one the reference arm
    # repeats live; the other fixture wavelengths are in oracle_pin
    pin0 = next((p for p in (oracle_pin or []) if p["wavelength_nm"] == 520.0),
                (oracle_pin or [{}])[0])
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max_s * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic",
            "config": dict(workload_config(args, n, lams), sweep_repetitions=reps,
                           solves=len(solves),
                           step_rule="step s solves sweep entries s, s+K, s+2K, ... (each "
                                     "wavelength equally often)"),
            "mode": "fp32_refine", "clocks": clk.summary(), "e2e": e2e, "gpu_launches": launches,
            "roofline": roof, "cpu_baseline": cpu, "fp64_plain": fp64,
            "speedup_vs_fp64_plain": fp64["speedup_same_solves"] if fp64 else None,
            "cext_rel_err_vs_oracle": pin0.get("cext_rel_err_fp32_refine"),
            "reference_solve_measured_s": pin0.get("oracle_solve_measured_s"),
            "oracle_pin": oracle_pin, "per_wavelength": per_lam}
    print(json.dumps(line), flush=True)
    return 0


def _traffic_from_profiles(kernel="otf_pairs_f32", workload="cuboid30k"):
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1])
    except (OSError, ValueError):
        pass
    return None


# ---------------------------------------------------------------- secondary workloads
# Not the headline line: the batched-cluster, adjoint-gradient and periodic
# workloads, each printed as one JSON line of the same shape, for the record.
def _timed(stream, fn):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1)


def _plane_wave(pos, k, direction, pol, amplitude=1.0):
    ph = np.exp(1j * k * (pos @ np.asarray(direction, np.float64)))
    return (amplitude * ph[:, None] * np.asarray(pol, np.complex128)[None, :]).ravel()


def run_secondary(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0  # single-GPU records; other ranks have nothing to do
    if args.impl == "reference":
        print(json.dumps({"impl": "reference", "workload": args.workload,
                          "unavailable": "secondary workloads have no CPU reference arm; the "
                                         "headline workload carries it"}), flush=True)
        return 0
    import torch
    import lumina_b200 as lb
    from lumina_b200 import _ffi, configs
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    bk = lb.CudaBackend(0)
    fp32_peak, fp64_peak = bk.measure_fma_peak()
    launches0 = _ffi.launch_count()
    with ClockSampler(0) as clk:
        if args.workload == "clusters":
            line = _bench_clusters(args, bk, stream, torch, lb, configs, fp32_peak)
        elif args.workload == "dimer":
            line = _bench_dimer(args, bk, stream, torch, lb, configs)
        elif args.workload == "cached":
            line = _bench_cached(args, bk, stream, torch, lb, configs)
        elif args.workload == "directions":
            line = _bench_directions(args, bk, stream, torch, lb, configs)
        elif args.workload == "fft":
            line = _bench_fft(args, bk, stream, torch, lb, configs)
        elif args.workload == "fields":
            line = _bench_fields(args, bk, stream, torch, lb, configs, fp64_peak)
        elif args.workload == "sommerfeld":
            line = _bench_sommerfeld(args, bk, stream, torch, lb, configs, fp32_peak)
        elif args.workload == "harmonic":
            line = _bench_harmonic(args, bk, stream, torch, lb, configs)
        else:
            line = _bench_metasurface(args, bk, stream, torch, lb, configs)
    line["gpu_launches"] = _ffi.launch_count() - launches0
    line["clocks"] = clk.summary()
    line.update({"n_gpus": 1, "warmup": args.warmup, "data": "synthetic", "vs_baseline": None})
    print(json.dumps(line), flush=True)
    return 0


def _bench_clusters(args, bk, stream, torch, lb, configs, fp32_peak):
    w = configs.batch_clusters(args.clusters, 0, spacing=args.spacing or 1.5)
    systems = w.systems()
    specs = [(p, lb.invert_polarisability(a), k, cell) for p, a, k, cell, _ in systems]
    rhs = np.concatenate([lb.incident_field(p, k, inc) for p, _, k, _, inc in systems])
    B = bk.create_batch(specs)
    B.set_stream(stream.cuda_stream)
    b_dev = torch.from_numpy(rhs).to("cuda")
    x_dev = torch.zeros_like(b_dev)
    tol, max_iter = args.tol, max(args.max_iter, 20000)
    for _ in range(args.warmup):  # short solves: capture both cycle graphs
        for mode in ("fp32_refine", "fp64"):
            try:
                B.solve_device(b_dev.data_ptr(), x_dev.data_ptr(), tol, 31, 30, mode)
            except lb.ConvergenceFailure:
                pass
    ns = np.array(B.sizes, np.float64)
    pairs = float(np.sum(ns * (ns - 1)))
    mv = {}
    xr = torch.randn(B.dim * 2, dtype=torch.float64, device="cuda")
    yr = torch.empty_like(xr)
    for prec in ("fp32", "fp64"):
        B.matvec_device(xr.data_ptr(), yr.data_ptr(), prec)
        _, ms = _timed(stream, lambda: [B.matvec_device(xr.data_ptr(), yr.data_ptr(), prec)
                                        for _ in range(5)])
        mv[prec] = ms / 5
    info32, ms32 = _timed(stream, lambda: [B.solve_device(b_dev.data_ptr(), x_dev.data_ptr(), tol,
                                                          max_iter, 30, "fp32_refine")
                                           for _ in range(args.steps)][-1])
    x32 = x_dev.cpu().numpy()
    x64_dev = torch.zeros_like(b_dev)
    info64, ms64 = _timed(stream, lambda: B.solve_device(b_dev.data_ptr(), x64_dev.data_ptr(), tol,
                                                         max_iter, 30, "fp64"))
    x64 = x64_dev.cpu().numpy()
    err = 0.0
    for s, (p, inv, k, cell) in enumerate(specs):
        inc = systems[s][4]
        sl = slice(3 * int(B.offsets[s]), 3 * int(B.offsets[s + 1]))
        c32 = lb.cross_sections(p, inv, x32[sl], k, inc)[0]
        c64 = lb.cross_sections(p, inv, x64[sl], k, inc)[0]
        err = max(err, abs(c32 - c64) / abs(c64))
    t0 = time.perf_counter()
    B.solve(rhs, tol, max_iter, 30, "fp32_refine")  # e2e: host arrays in and out
    e2e_s = time.perf_counter() - t0
    its = [i["iterations"] for i in info32]
    nd = w.n_dipoles
    value = nd * args.steps / (ms32 * 1e-3)
    info = B.info()
    kcfg = B.kernel_config()
    achieved = pairs * FLOPS_PER_PAIR / (mv["fp32"] * 1e-3) / 1e12
    return {"metric": "dipole-solves/s, batched clusters (FP32+refine, C_ext rel err <=1e-6 vs "
                      "FP64)", "value": value, "unit": UNIT, "steps": args.steps,
            "ms_per_step": ms32 / args.steps, "higher_is_better": True, "scaling": "weak",
            "dtype": "f32+f64", "mode": "fp32_refine",
            "config": {"workload": f"{args.clusters} Drude ellipsoid clusters (1.5 nm lattice, "
                                   f"anisotropic ellipsoid alpha, 600 nm) x 2 polarisations, "
                                   f"splitmix64 seed 0", "systems": len(specs),
                       "dipoles_total": nd, "n_min": int(ns.min()), "n_max": int(ns.max()),
                       "tol": tol, "max_iter": max_iter, "batch": info,
                       "kernels": kcfg},
            "fp64_plain": {"value": nd / (ms64 * 1e-3), "ms_per_solve": ms64,
                           "speedup_same_solves": ms64 / (ms32 / args.steps),
                           "max_cext_rel_err": err},
            "iterations": {"min": min(its), "mean": float(np.mean(its)), "max": max(its),
                           "converged": sum(i["converged"] for i in info32)},
            "e2e": {"value": nd / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(rhs.nbytes),
                    "d2h_bytes_per_step": int(rhs.nbytes)},
            # a full-batch FP32 application (pair kernel + epilogue) of the scheme chosen at
            # creation; in a solve, cycles with few active systems take the split list
            "roofline": {"bound": "fp32",
                         "kernel": ("batch_pairs_f32_sym" if kcfg.get("sym32") else
                                    "batch_pairs_f32"), "achieved": achieved,
                         "peak": fp32_peak / 1e3, "unit": "TFLOP/s",
                         "frac": achieved / (fp32_peak / 1e3), "avg_launch_ms": mv["fp32"],
                         "pairs_per_launch": pairs, "fp64_matvec_ms": mv["fp64"],
                         "peak_source": "FP32 FMA-chain microbenchmark in this run; of measured"}}


def _bench_dimer(args, bk, stream, torch, lb, configs):
    d = configs.helix_dimer(args.spacing or 1.0)
    w = d.workload
    n = w.n
    inv = lb.invert_polarisability(w.alpha)
    dinv = d.dinv_alpha_deps()
    tol, max_iter = args.tol, args.max_iter
    S = bk.create_onthefly_session(w.positions, inv, w.k, True, w.cell_size)
    S.set_stream(stream.cuda_stream)
    bL = torch.from_numpy(_plane_wave(w.positions, w.k, d.direction, d.lcp)).to("cuda")
    x = torch.zeros_like(bL)
    def grad(pol):
        return S.grad_cext(d.direction, pol, 1.0, dinv, tol=tol, max_iter=max_iter,
                           mode="fp32_refine")

    for _ in range(args.warmup):  # both paths warm (tuning, workspaces, module loads)
        S.solve_device(bL.data_ptr(), x.data_ptr(), tol, max_iter, 30, "fp32_refine",
                       stream.cuda_stream)
        grad(d.lcp)
    # Timed passes (CUDA events on the session stream, no per-kernel profiling):
    # the LCP forward solve, and the LCP / RCP gradients (forward + adjoint
    # solves in lockstep, gradient kernels, results copied to the host).
    fwd, ms_fwd = _timed(stream, lambda: S.solve_device(bL.data_ptr(), x.data_ptr(), tol, max_iter,
                                                        30, "fp32_refine", stream.cuda_stream))
    res = {}
    for name, pol in (("lcp", d.lcp), ("rcp", d.rcp)):
        res[name], ms = _timed(stream, lambda: grad(pol))
        res[name]["ms"] = ms
    # Per-kernel breakdown from separate, profiled passes (not timed)
    kern = {}
    S.profile(True)
    S.solve_device(bL.data_ptr(), x.data_ptr(), tol, max_iter, 30, "fp32_refine",
                   stream.cuda_stream)
    for p in ("fp32", "fp64"):
        c, ms = S.kernel_time(p)
        kern[f"forward_{p}"] = {"launches": c, "ms": ms, "avg_ms": ms / c if c else None}
    S.profile(True)
    grad(d.lcp)
    for p in ("fp32x2", "fp64x2"):
        c, ms = S.kernel_time(p)
        kern[f"gradient_{p}"] = {"launches": c, "ms": ms, "avg_ms": ms / c if c else None}
    S.profile(False)
    # the reference's CD (fields.rs:236-253) from x and y linear solves
    from lumina_b200.solver import circular_dichroism
    from lumina_b200.types import DipoleResponse
    mom = {}
    for name, pol in (("x", (1.0, 0.0, 0.0)), ("y", (0.0, 1.0, 0.0))):
        b = _plane_wave(w.positions, w.k, d.direction, pol)
        xx, _ = S.solve(b, tol, max_iter, 30, "fp32_refine")
        mom[name] = DipoleResponse(650.0, 1.0, xx.reshape(-1, 3), xx.reshape(-1, 3))
    cd_ref = circular_dichroism(mom["x"], mom["y"], w.k)
    ms_grad = res["lcp"]["ms"]
    gL, gR = res["lcp"], res["rcp"]
    return {"metric": "adjoint gradient cost / forward solve (dC_ext/dr, dC_ext/deps), helix "
                      "dimer", "value": ms_grad / ms_fwd, "unit": "x forward solve",
            "higher_is_better": False, "steps": 1, "ms_per_step": ms_grad, "scaling": "weak",
            "dtype": "f32+f64", "mode": "fp32_refine",
            "config": {"workload": f"two left-handed Au helices (pitch 40, R 15, wire 5 nm, 2 "
                                   f"turns, {w.cell_size:g} nm lattice, 20 nm gap), 650 nm, "
                                   f"LCP/RCP along +z", "n_dipoles": n, "tol": tol},
            "forward_ms": ms_fwd, "gradient_ms_lcp": gL["ms"], "gradient_ms_rcp": gR["ms"],
            "pair_kernels": kern, "kernel_config": S.kernel_config(),
            "adjoint_overhead": (ms_grad - ms_fwd) / ms_fwd,
            "forward_solve_s": fwd["seconds"],
            "gradient_lockstep_solve_s": gL["info_forward"]["seconds"],
            "iterations_forward": gL["info_forward"]["iterations"],
            "iterations_adjoint": gL["info_adjoint"]["iterations"],
            "c_ext_lcp": gL["c_ext"], "c_ext_rcp": gR["c_ext"],
            "cd_true": gL["c_ext"] - gR["c_ext"], "cd_reference_formula": cd_ref,
            "grad_cd_r_norm": float(np.linalg.norm(gL["grad_r"] - gR["grad_r"])),
            "e2e": {"value": n / (ms_grad * 1e-3), "unit": "dipole-gradients/s",
                    "h2d_bytes_per_step": n * 9 * 16, "d2h_bytes_per_step": n * (3 * 16 + 5 * 8)}}


def _bench_cached(args, bk, stream, torch, lb, configs):
    """The cached-matrix path: device assembly of the FP32 3N x 3N matrix of
    an Au cuboid (FCD), then (a) the single-vector GEMV, HBM-bound, and (b)
    Y = A X for --nrhs vectors on the tensor cores (3xTF32) beside the
    CUDA-core product.  The matrix (>= 1 GB) is far larger than L2."""
    import json as _json
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = _json.load(f)
    except (OSError, ValueError):
        pass
    # MEASURED_PEAKS.json (written per pool) when present, else the pool's
    # earlier measurement (6.65 TB/s, 1.59 PFLOP/s bf16); the line says which
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    tf32_peak = float(peaks.get("bf16_tflops", 1590.0)) / 2.0  # dense TF32 = half of BF16
    hbm_src = "MEASURED_PEAKS.json hbm_gbs; of measured" if "hbm_gbs" in peaks else \
        "no MEASURED_PEAKS.json: the pool's earlier copy measurement, 6650 GB/s; of fallback"
    tf32_src = ("TF32 dense = MEASURED_PEAKS.json bf16_tflops / 2; of measured"
                if "bf16_tflops" in peaks else
                "no MEASURED_PEAKS.json: TF32 dense = 1590 / 2 TFLOP/s (earlier bf16 "
                "measurement on this pool); of fallback")
    size = tuple(float(v) for v in (args.size if args.size != "60,50,10" else "30,20,10").split(","))
    w = configs.cuboid_au(size, 1.0, 520.0)
    n, dim = w.n, 3 * w.n
    inv = lb.invert_polarisability(w.alpha)
    t0 = time.perf_counter()
    S = bk.assemble_and_create_session(w.positions, w.k, inv, True, 1.0, precision="fp32")
    S.set_stream(stream.cuda_stream)
    torch.cuda.synchronize()
    assemble_s = time.perf_counter() - t0
    R = args.nrhs
    gen = torch.Generator(device="cuda").manual_seed(0)
    X = torch.randn(R * dim, dtype=torch.complex128, device="cuda", generator=gen)
    Y = torch.empty_like(X)
    Yc = torch.empty_like(X)
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    reps = max(args.steps, 3)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        ms = []
        for _ in range(reps):
            flush.zero_()
            _, t = _timed(stream, fn)
            ms.append(t)
        return statistics.median(ms)

    x1 = X[:dim]
    ms_gemv = timed(lambda: S.matvec_device(x1.data_ptr(), Y.data_ptr(), "fp32", stream.cuda_stream))
    ms_tc = timed(lambda: S.matmul_vectors_device(X.data_ptr(), Y.data_ptr(), R, "tensor",
                                                  stream.cuda_stream))
    ms_cc = timed(lambda: S.matmul_vectors_device(X.data_ptr(), Yc.data_ptr(), R, "cuda_cores",
                                                  stream.cuda_stream))
    torch.cuda.synchronize()
    err = float(torch.max(torch.abs(Y - Yc)) / torch.max(torch.abs(Yc)))
    # the same matrix in symmetric tile storage (free space: A = A^T): the
    # upper-triangle tiles only, each read once and applied twice
    y_dense = torch.empty(dim, dtype=torch.complex128, device="cuda")
    S.matvec_device(x1.data_ptr(), y_dense.data_ptr(), "fp32", stream.cuda_stream)
    Ssym = bk.assemble_and_create_session(w.positions, w.k, inv, True, 1.0, precision="fp32",
                                          symmetric=True)
    Ssym.set_stream(stream.cuda_stream)
    y_sym = torch.empty_like(y_dense)
    ms_sym = timed(lambda: Ssym.matvec_device(x1.data_ptr(), y_sym.data_ptr(), "fp32",
                                              stream.cuda_stream))
    torch.cuda.synchronize()
    sym_diff = float(torch.max(torch.abs(y_sym - y_dense)) / torch.max(torch.abs(y_dense)))
    Ssym.close()
    tile = 192  # the library's tile side (kSymTile, 64 dipoles)
    nt = -(-dim // tile)
    sym_bytes = 8.0 * tile * tile * nt * (nt + 1) / 2   # stored tiles, zero padding included
    slot_bytes = 2.0 * 16.0 * nt * dim                  # per-tile partials written and summed
    # FP64 storage (the reference's cached matrix is complex FP64): the same
    # GEMV over dense rows and over symmetric tiles, FP64 arithmetic
    fp64 = {}
    for name, sym in (("dense_rows", False), ("symmetric_tiles", True)):
        S64 = bk.assemble_and_create_session(w.positions, w.k, inv, True, 1.0, precision="fp64",
                                             symmetric=sym)
        S64.set_stream(stream.cuda_stream)
        y64 = torch.empty(dim, dtype=torch.complex128, device="cuda")
        ms64 = timed(lambda: S64.matvec_device(x1.data_ptr(), y64.data_ptr(), "fp64",
                                               stream.cuda_stream))
        S64.close()
        b64 = 2.0 * (sym_bytes if sym else 8.0 * dim * dim)   # 16 bytes per stored entry
        fp64[name] = {"ms": ms64, "bytes_gb": b64 / 1e9,
                      "achieved_gbs": b64 / (ms64 * 1e-3) / 1e9,
                      "frac": b64 / (ms64 * 1e-3) / 1e9 / hbm_peak}
        del y64
    fp64["kernel"] = "gemv_sym_tiles<double2, dense rows | symmetric tiles> + gemv_reduce"
    fp64["peak_source"] = hbm_src
    # e2e: the same GEMV through the host-array call (vector in, product out)
    x1h = x1.cpu().numpy()
    S.matvec(x1h, "fp32")
    e2e_ms = []
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        S.matvec(x1h, "fp32")
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_gemv = statistics.median(e2e_ms)
    a_bytes = 8.0 * dim * dim
    cflops = 8.0 * dim * dim * R            # complex multiply-adds x 8 real flops
    tc_flops = 3.0 * cflops                 # three TF32 products per operand pair
    S.close()
    return {"metric": "cached 3N x 3N matrix: GEMV HBM GB/s and multi-RHS tensor-core product",
            "value": a_bytes / (ms_gemv * 1e-3) / 1e9, "unit": "GB/s (GEMV)",
            "higher_is_better": True, "steps": reps, "ms_per_step": ms_gemv, "scaling": "weak",
            "dtype": "f32 (complex)", "mode": "cached",
            "config": {"workload": f"Au cuboid {size[0]:g}x{size[1]:g}x{size[2]:g} nm, 1 nm "
                                   f"lattice, N={n}, FCD, 520 nm, FP32 device-assembled matrix",
                       "n_dipoles": n, "dim": dim, "matrix_gb": a_bytes / 1e9, "nrhs": R,
                       "l2": "256 MB flush before each timed product; matrix >> L2"},
            "assemble_s": assemble_s,
            "roofline": {"bound": "hbm",
                         "kernel": ("gemv_part<float2> + gemv_reduce"
                                    if os.environ.get("LUMINA_DENSE_GEMV") == "rows" else
                                    "gemv_sym_tiles<float2, dense rows> + gemv_reduce"),
                         # DRAM bytes of one launch from the ncu capture of this workload
                         "traffic_source": "profiles/gemv_dense_blocks_cuboid6k.md",
                         "achieved": a_bytes / (ms_gemv * 1e-3) / 1e9, "peak": hbm_peak,
                         "unit": "GB/s", "frac": a_bytes / (ms_gemv * 1e-3) / 1e9 / hbm_peak,
                         "traffic": (_traffic_from_profiles("gemv_dense_blocks", "cuboid6k")
                                     if os.environ.get("LUMINA_DENSE_GEMV") != "rows" else None),
                         "peak_source": hbm_src},
            "tensor_product": {
                "kernel": "cgemm_tf32x3_kernel", "nrhs": R, "ms": ms_tc,
                "complex_tflops": cflops / (ms_tc * 1e-3) / 1e12,
                "tf32_tflops": tc_flops / (ms_tc * 1e-3) / 1e12,
                "tf32_peak_tflops": tf32_peak,
                "tf32_frac": tc_flops / (ms_tc * 1e-3) / 1e12 / tf32_peak,
                "hbm_gbs": a_bytes / (ms_tc * 1e-3) / 1e9,
                "hbm_frac": a_bytes / (ms_tc * 1e-3) / 1e9 / hbm_peak,
                "bound_ms": max(a_bytes / (hbm_peak * 1e9), tc_flops / (tf32_peak * 1e12)) * 1e3,
                "peak_source": tf32_src,
                "speedup_vs_cuda_cores": ms_cc / ms_tc, "cuda_cores_ms": ms_cc,
                "rel_diff_vs_cuda_cores": err,
                "gemv_equivalent_ms": ms_gemv * R},
            "symmetric_tiles": {
                "kernel": "gemv_sym_tiles<float2> + gemv_reduce", "ms": ms_sym,
                "speedup_vs_dense_rows": ms_gemv / ms_sym,
                "stored_gb": sym_bytes / 1e9, "dense_gb": a_bytes / 1e9,
                "achieved_gbs": sym_bytes / (ms_sym * 1e-3) / 1e9,
                "frac": sym_bytes / (ms_sym * 1e-3) / 1e9 / hbm_peak,
                "slot_traffic_gb": slot_bytes / 1e9,
                "dense_equivalent_gbs": a_bytes / (ms_sym * 1e-3) / 1e9,
                "rel_diff_vs_dense_rows": sym_diff, "peak_source": hbm_src},
            "fp64_storage": fp64,
            "e2e": {"value": a_bytes / (e2e_gemv * 1e-3) / 1e9, "unit": "GB/s (GEMV)",
                    "h2d_bytes_per_step": dim * 16, "d2h_bytes_per_step": dim * 16}}


def _incidence_set(m):
    """m directions on a cone (polar 0.3-0.8 rad) with real transverse
    polarisations: an orientation sweep of one target."""
    out = []
    for q in range(m):
        th = 0.3 + 0.5 * q / max(m - 1, 1)
        ph = 2 * math.pi * q / m
        d = np.array([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)])
        e = np.cross(d, [0.0, 0.0, 1.0])
        out.append((d, e / np.linalg.norm(e)))
    return out


def _bench_directions(args, bk, stream, torch, lb, configs):
    """Many right-hand sides of one operator: --nrhs incidence directions of
    the Au cuboid (default 30x20x10 nm, N = 6,000, FCD, 520 nm), FP32+refine
    to --tol.  (a) the device-assembled FP32 matrix, every FP32 step one
    tensor-core product over all directions (lum_batch_create_rhs);
    (b) the on-the-fly operator, two directions per pair-kernel launch
    (lum_solve_gmres_multi)."""
    size = tuple(float(v) for v in (args.size if args.size != "60,50,10" else "30,20,10").split(","))
    w = configs.cuboid_au(size, 1.0, 520.0)
    n, R = w.n, args.nrhs
    inv = lb.invert_polarisability(w.alpha)
    dirs = _incidence_set(R)
    rhs = np.concatenate([lb.incident_field(w.positions, w.k, lb.IncidentField(tuple(d), tuple(e)))
                          for d, e in dirs])
    b_dev = torch.from_numpy(rhs).to("cuda")
    x_dev = torch.zeros_like(b_dev)
    tol, max_iter = args.tol, max(args.max_iter, 5000)
    t0 = time.perf_counter()
    C = bk.assemble_and_create_session(w.positions, w.k, inv, True, 1.0, precision="fp32")
    torch.cuda.synchronize()
    assemble_s = time.perf_counter() - t0
    B = C.rhs_batch(R)
    for _ in range(args.warmup):
        B.solve_device(b_dev.data_ptr(), x_dev.data_ptr(), tol, max_iter, 30, "fp32_refine")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    info_tc = B.solve_device(b_dev.data_ptr(), x_dev.data_ptr(), tol, max_iter, 30, "fp32_refine")
    torch.cuda.synchronize()
    t_tc = time.perf_counter() - t0
    x_tc = x_dev.cpu().numpy()
    t0 = time.perf_counter()
    B.solve(rhs, tol, max_iter, 30, "fp32_refine")  # e2e: host arrays in and out
    t_e2e = time.perf_counter() - t0
    B.close()
    C.close()
    O = bk.create_onthefly_session(w.positions, inv, w.k, True, 1.0)
    O.set_stream(stream.cuda_stream)
    for _ in range(args.warmup):
        O.solve_multi_device(R, b_dev.data_ptr(), x_dev.data_ptr(), tol, max_iter, 30,
                             "fp32_refine", stream.cuda_stream)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    O.solve_multi_device(R, b_dev.data_ptr(), x_dev.data_ptr(), tol, max_iter, 30, "fp32_refine",
                         stream.cuda_stream)
    torch.cuda.synchronize()
    t_otf = time.perf_counter() - t0
    x_otf = x_dev.cpu().numpy()
    O.close()
    err = 0.0
    for q, (d, e) in enumerate(dirs):
        sl = slice(3 * n * q, 3 * n * (q + 1))
        inc = lb.IncidentField(tuple(d), tuple(e))
        a = lb.cross_sections(w.positions, inv, x_tc[sl], w.k, inc)[0]
        b = lb.cross_sections(w.positions, inv, x_otf[sl], w.k, inc)[0]
        err = max(err, abs(a - b) / abs(b))
    its = [i["iterations"] for i in info_tc]
    return {"metric": "dipole-solves/s, many incidence directions of one cached matrix "
                      "(tensor-core products, FP32+refine)", "value": n * R / t_tc, "unit": UNIT,
            "higher_is_better": True, "steps": 1, "ms_per_step": t_tc * 1e3, "scaling": "weak",
            "dtype": "tf32x3+f64", "mode": "fp32_refine",
            "config": {"workload": f"Au cuboid {size[0]:g}x{size[1]:g}x{size[2]:g} nm, 1 nm "
                                   f"lattice, N={n}, FCD, 520 nm, {R} incidence directions",
                       "n_dipoles": n, "nrhs": R, "tol": tol,
                       "matrix_gb": 8.0 * (3 * n) ** 2 / 1e9},
            "assemble_s": assemble_s,
            "iterations": {"min": min(its), "max": max(its)},
            "onthefly_two_at_a_time": {"value": n * R / t_otf, "seconds": t_otf,
                                       "speedup_of_tensor_path": t_otf / t_tc},
            "max_cext_rel_diff_vs_onthefly": err,
            "e2e": {"value": n * R / t_e2e, "unit": UNIT, "h2d_bytes_per_step": int(rhs.nbytes),
                    "d2h_bytes_per_step": int(rhs.nbytes)}}


def _bench_fft(args, bk, stream, torch, lb, configs):
    """The headline cuboid (60x50x10 nm, N = 30,000, FCD cell 1 nm, tol 1e-8,
    520/650/800 nm) solved through the block-Toeplitz FFT operator
    (fft_matvec.rs, widened to FCD): FP32+refine and plain FP64 solves, C_ext
    against the on-the-fly FP64 solve, and the time of one operator
    application in each precision."""
    lams = wavelength_list(args, "520,650,800")
    base, per = build_inputs(args, lams)
    n = base.n
    inv = [lb.invert_polarisability(w.alpha) for w in per]
    rhs = [lb.incident_field(w.positions, w.k, lb.IncidentField()) for w in per]
    F = bk.create_fft_session(base.positions, inv[0], per[0].k, True, 1.0)
    F.set_stream(stream.cuda_stream)
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    b_dev = [torch.from_numpy(r).to("cuda") for r in rhs]
    x_dev = torch.zeros(3 * n, dtype=torch.complex128, device="cuda")
    rows, t32, t64 = [], 0.0, 0.0
    for i, lam in enumerate(lams):
        F.set_wavelength(per[i].k, inv[i])
        for _ in range(args.warmup):
            F.solve_device(b_dev[i].data_ptr(), x_dev.data_ptr(), args.tol, args.max_iter, 30,
                           "fp32_refine", stream.cuda_stream)
        flush.zero_()
        info32, ms32 = _timed(stream, lambda: F.solve_device(
            b_dev[i].data_ptr(), x_dev.data_ptr(), args.tol, args.max_iter, 30, "fp32_refine",
            stream.cuda_stream))
        x32 = x_dev.cpu().numpy()
        flush.zero_()
        info64, ms64 = _timed(stream, lambda: F.solve_device(
            b_dev[i].data_ptr(), x_dev.data_ptr(), args.tol, args.max_iter, 30, "fp64",
            stream.cuda_stream))
        x64 = x_dev.cpu().numpy()
        c32 = lb.cross_sections(base.positions, inv[i], x32, per[i].k, lb.IncidentField())
        c64 = lb.cross_sections(base.positions, inv[i], x64, per[i].k, lb.IncidentField())
        # the on-the-fly FP64 operator's C_ext at this wavelength (reference semantics)
        with bk.create_onthefly_session(base.positions, inv[i], per[i].k, True, 1.0) as O:
            xo, _ = O.solve(rhs[i], args.tol, args.max_iter, 30, "fp64")
        co = lb.cross_sections(base.positions, inv[i], xo, per[i].k, lb.IncidentField())
        t32 += ms32
        t64 += ms64
        rows.append({"wavelength_nm": lam, "ms_fp32_refine": ms32, "ms_fp64": ms64,
                     "iterations": info32["iterations"], "iterations_fp64": info64["iterations"],
                     "cext_fft_fp32_refine": c32[0], "cext_onthefly_fp64": co[0],
                     "cext_rel_err_vs_onthefly": abs(c32[0] - co[0]) / abs(co[0]),
                     "cext_rel_err_fp64": abs(c64[0] - co[0]) / abs(co[0])})
    xr = torch.randn(3 * n, dtype=torch.complex128, device="cuda")
    yr = torch.empty_like(xr)
    apply_ms = {}
    for prec in ("fp32", "fp64"):
        for _ in range(3):
            F.matvec_device(xr.data_ptr(), yr.data_ptr(), prec, stream.cuda_stream)
        _, ms = _timed(stream, lambda: [F.matvec_device(xr.data_ptr(), yr.data_ptr(), prec,
                                                        stream.cuda_stream) for _ in range(20)])
        apply_ms[prec] = ms / 20
    cfg = F.kernel_config()
    F.close()
    # e2e: the solver's FFT branch with host arrays over the same wavelengths
    solver = lb.CdaSolver(backend=bk, iterative_threshold=0, use_fcd=True, cell_size=1.0,
                          matrix_memory_budget=0, precision="fp32_refine", use_fft=True)
    params = lb.SimulationParams(solver_tolerance=args.tol, max_iterations=args.max_iter)
    ds = [lb.DipoleSet(w.positions, w.alpha) for w in per]
    solver.compute_cross_sections(ds[0], lams[0], params)  # warm
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i, lam in enumerate(lams):
        solver.compute_cross_sections(ds[i], lam, params)
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    solver.close()
    # roofline of one FP32 application: the pass structure's L2 traffic -- six
    # axis passes (three forward, three inverse) and the spectral product each
    # read and write the three-component grid (M complex FP32 per component),
    # and the product reads the six kernel spectra; no credit is taken for the
    # lines the passes skip, so this over-counts and the fraction is an upper
    # bound
    size = [float(v) for v in args.size.split(",")]
    m = 1
    for L in size:
        c = 1
        while c < 2 * int(round(L)) - 1:
            c *= 2
        m *= c
    fft_bytes = 6.0 * m * 8.0 + 7.0 * 2.0 * 3.0 * m * 8.0
    l2_peak = bk.measure_l2_peak()
    nl = len(rows)
    return {"metric": "dipole-solves/s at N=30k through the FFT (block-Toeplitz) operator, "
                      "FP32+refine", "value": n * nl / (t32 * 1e-3), "unit": UNIT,
            "higher_is_better": True, "steps": nl, "ms_per_step": t32 / nl, "scaling": "weak",
            "dtype": "f32+f64", "mode": "fp32_refine",
            "config": dict(workload_config(args, n, lams), operator="fft (circulant 128x128x32)"),
            "fp64_plain": {"value": n * nl / (t64 * 1e-3), "speedup_same_solves": t64 / t32},
            "apply_ms": apply_ms,
            "max_cext_rel_err_vs_onthefly_fp64": max(r["cext_rel_err_vs_onthefly"] for r in rows),
            "per_wavelength": rows, "kernel_config": cfg,
            "roofline": {"bound": "l2", "kernel": "fft_lines + fft_spectral_product",
                         "achieved": fft_bytes / (apply_ms["fp32"] * 1e-3) / 1e9,
                         "peak": l2_peak, "unit": "GB/s",
                         "frac": fft_bytes / (apply_ms["fp32"] * 1e-3) / 1e9 / l2_peak,
                         "bytes_model": f"{fft_bytes / 1e6:.0f} MB per FP32 application: 7 "
                                        f"passes x read+write of 3 x {m} complex FP32 + 6 "
                                        f"spectra (skipped lines not credited: upper bound)",
                         "peak_source": "L2 read microbenchmark in this run "
                                        "(lum_measure_l2_peak); of measured", "traffic": None},
            "e2e": {"value": n * nl / t_e2e, "unit": UNIT,
                    "h2d_bytes_per_step": n * 3 * 8 + n * 9 * 16,
                    "d2h_bytes_per_step": 3 * n * 16}}


def _bench_fields(args, bk, stream, torch, lb, configs, fp64_peak):
    """fields.rs on the device: a 256 x 256 near-field map 5 nm above the
    N = 30,000 cuboid and a 181 x 360 far-field pattern, from the moments of
    an FP32+refine solve at 520 nm (the solve is not timed).  Host arrays in
    and out (the reference's call shape); FP64 throughout."""
    from lumina_b200 import fields
    w = configs.cuboid_au_30k(520.0)
    inv = lb.invert_polarisability(w.alpha)
    with bk.create_onthefly_session(w.positions, inv, w.k, True, 1.0) as S:
        b = lb.incident_field(w.positions, w.k, lb.IncidentField())
        x, _ = S.solve(b, args.tol, args.max_iter, 30, "fp32_refine")
    mom = x.reshape(-1, 3)
    n = w.n
    top = float(np.max(w.positions[:, 2]))
    plane = fields.NearFieldPlane((0.0, 0.0, top + 5.0), (0.0, 0.0, 1.0), 40.0, 35.0, 256, 256)
    resp = lb.DipoleResponse(520.0, 1.0, mom, mom)

    def near():
        return fields.compute_near_field_map(bk, w.positions, mom, plane, w.k)

    def far():
        return fields.compute_far_field(bk, w.positions, resp, w.k, 181, 360)

    for _ in range(args.warmup):
        near()
        far()
    reps = max(args.steps, 3)
    t_near, t_far = [], []
    for _ in range(reps):
        t0 = time.perf_counter()
        near()
        t_near.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        far()
        t_far.append(time.perf_counter() - t0)
    tn, tf = statistics.median(t_near), statistics.median(t_far)
    pn, pf = float(n) * 256 * 256, float(n) * 181 * 360
    return {"metric": "observation-dipole pairs/s, near-field map (fields.rs, FP64)",
            "value": pn / tn, "unit": "pairs/s", "higher_is_better": True, "steps": reps,
            "ms_per_step": tn * 1e3, "scaling": "weak", "dtype": "f64", "mode": "fields",
            "config": {"workload": "Au cuboid 60x50x10 nm (N=30,000) moments at 520 nm; "
                                   "near-field map 256x256 on z = top + 5 nm (80 x 70 nm); far "
                                   "field 181 x 360 directions", "n_dipoles": n},
            "near_field_ms": tn * 1e3, "far_field_ms": tf * 1e3,
            "far_field_pairs_per_s": pf / tf,
            "roofline": {"bound": "fp64", "kernel": "near_field_part",
                         "achieved": pn * FLOPS_PER_PAIR / tn / 1e12, "peak": fp64_peak / 1e3,
                         "unit": "TFLOP/s", "frac": pn * FLOPS_PER_PAIR / tn / 1e12 / (fp64_peak / 1e3),
                         "note": "86 flops per pair (the operator's canonical pair count; the "
                                 "field kernel contracts the same tensor); host-timed including "
                                 "the host<->device copies; FP64 FMA-chain peak; of measured"},
            "e2e": {"value": pn / tn, "unit": "pairs/s", "h2d_bytes_per_step": n * (24 + 48),
                    "d2h_bytes_per_step": 256 * 256 * 8}}


SOMM_FLOPS_PER_PAIR = 100.0  # block from a record (24) + 3x3 complex product (72) + rho, cos/sin


def _bench_sommerfeld(args, bk, stream, torch, lb, configs, fp32_peak):
    """An Au sphere (R = 30 nm, 2 nm lattice, N = 14,147) 5 nm above glass
    (eps 2.25) in air at 520 nm with the Sommerfeld substrate (sommerfeld.rs,
    SubstrateRuntime::Sommerfeld): session set-up including the reflected-
    integral table, FP32+refine and FP64 GMRES(30) solves at tol 1e-8 with C_ext
    compared, one operator application per precision, and the host oracle's
    reflected-tensor cost per pair scaled to the reference's on-the-fly solve,
    which re-evaluates G_refl for every ordered pair of every matvec."""
    from lumina_b200.geometry import Sphere, discretise_primitive
    from lumina_b200.lattice import SommerfeldRuntime
    radius, gap, lam = 30.0, 5.0, 520.0
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), radius), 2.0).copy()
    pos[:, 2] += radius + gap
    w = configs.au_workload("sphere_on_glass", pos, 2.0, lam)
    n = w.n
    inv = lb.invert_polarisability(w.alpha)
    somm = SommerfeldRuntime(0.0, lam, 2.25 + 0.0j, 1.0)
    rhs = lb.incident_field(w.positions, w.k, lb.IncidentField())
    tol, max_iter = 1e-8, max(args.max_iter, 20000)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    S = bk.create_onthefly_session(w.positions, inv, w.k, True, 2.0, substrate=somm)
    setup_ms = (time.perf_counter() - t0) * 1e3
    S.set_stream(stream.cuda_stream)
    b_dev = torch.from_numpy(rhs).to("cuda")
    x_dev = torch.zeros_like(b_dev)
    for _ in range(args.warmup):
        for mode in ("fp32_refine", "fp64"):
            try:
                S.solve_device(b_dev.data_ptr(), x_dev.data_ptr(), tol, 31, 30, mode,
                               stream.cuda_stream)
            except lb.ConvergenceFailure:
                pass
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    t32 = []
    for _ in range(max(args.steps, 1)):
        flush.zero_()
        info32, ms = _timed(stream, lambda: S.solve_device(b_dev.data_ptr(), x_dev.data_ptr(), tol,
                                                           max_iter, 30, "fp32_refine",
                                                           stream.cuda_stream))
        t32.append(ms)
    x32 = x_dev.cpu().numpy()
    c32 = lb.cross_sections(w.positions, inv, x32, w.k, lb.IncidentField())[0]
    info64, ms64, c64 = info32, float("nan"), c32
    if not args.no_fp64:
        flush.zero_()
        info64, ms64 = _timed(stream, lambda: S.solve_device(b_dev.data_ptr(), x_dev.data_ptr(),
                                                             tol, max_iter, 30, "fp64",
                                                             stream.cuda_stream))
        x64 = x_dev.cpu().numpy()
        c64 = lb.cross_sections(w.positions, inv, x64, w.k, lb.IncidentField())[0]
    xr = torch.randn(3 * n, dtype=torch.complex128, device="cuda")
    yr = torch.empty_like(xr)
    apply_ms = {}
    for prec in ("fp32", "fp64"):
        for _ in range(3):
            S.matvec_device(xr.data_ptr(), yr.data_ptr(), prec, stream.cuda_stream)
        _, ms = _timed(stream, lambda: [S.matvec_device(xr.data_ptr(), yr.data_ptr(), prec,
                                                        stream.cuda_stream) for _ in range(20)])
        apply_ms[prec] = ms / 20
    # end to end through the public host-array call (copies included)
    e2e_s = float("nan")
    if not args.no_e2e:
        t0 = time.perf_counter()
        S.solve(rhs, tol, max_iter, 30, "fp32_refine")
        e2e_s = time.perf_counter() - t0
    cfg = S.kernel_config()
    S.close()
    # the same system through the FFT operator: the reflected term as a second
    # convolution in the z-mirrored coordinate
    F = bk.create_fft_session(w.positions, inv, w.k, True, 2.0, substrate=somm)
    F.set_stream(stream.cuda_stream)
    for _ in range(args.warmup):
        try:
            F.solve_device(b_dev.data_ptr(), x_dev.data_ptr(), tol, 31, 30, "fp32_refine",
                           stream.cuda_stream)
        except lb.ConvergenceFailure:
            pass
    flush.zero_()
    infof, msf = _timed(stream, lambda: F.solve_device(b_dev.data_ptr(), x_dev.data_ptr(), tol,
                                                       max_iter, 30, "fp32_refine",
                                                       stream.cuda_stream))
    cf = lb.cross_sections(w.positions, inv, x_dev.cpu().numpy(), w.k, lb.IncidentField())[0]
    fft_apply = {}
    for prec in ("fp32", "fp64"):
        for _ in range(3):
            F.matvec_device(xr.data_ptr(), yr.data_ptr(), prec, stream.cuda_stream)
        _, ms = _timed(stream, lambda: [F.matvec_device(xr.data_ptr(), yr.data_ptr(), prec,
                                                        stream.cuda_stream) for _ in range(20)])
        fft_apply[prec] = ms / 20
    F.close()
    ms32 = statistics.median(t32)
    line = {"metric": "dipole-solves/s, Au sphere above glass with the Sommerfeld substrate, "
                      "FP32+refine", "value": n / (ms32 * 1e-3), "unit": UNIT,
            "higher_is_better": True, "steps": len(t32), "ms_per_step": ms32, "scaling": "weak",
            "dtype": "f32+f64", "mode": "fp32_refine",
            "config": {"workload": "Au sphere R = 30 nm, 2 nm lattice, 5 nm above glass "
                                   "(eps 2.25) in air, 520 nm, FCD, Sommerfeld substrate, "
                                   "GMRES(30) tol 1e-8", "n_dipoles": n,
                       "l2": "64 MB flush before each timed solve"},
            "setup_ms": setup_ms, "iterations": info32["iterations"],
            "iterations_fp64": info64["iterations"], "converged": bool(info32["converged"]),
            "fp64_plain": None if args.no_fp64 else {"value": n / (ms64 * 1e-3), "ms": ms64,
                                                     "speedup_same_solves": ms64 / ms32},
            "cext_rel_err_fp32_refine_vs_fp64": None if args.no_fp64 else abs(c32 - c64) / abs(c64),
            "apply_ms": apply_ms, "kernel_config": cfg,
            "fft_operator": {"value": n / (msf * 1e-3), "ms": msf,
                             "iterations": infof["iterations"], "apply_ms": fft_apply,
                             "cext_rel_err_vs_onthefly": abs(cf - c32) / abs(c32)},
            "e2e": None if args.no_e2e else {"value": n / e2e_s, "unit": UNIT,
                                             "h2d_bytes_per_step": rhs.nbytes,
                                             "d2h_bytes_per_step": rhs.nbytes}}
    pairs = float(n) * n
    achieved = pairs * SOMM_FLOPS_PER_PAIR / (apply_ms["fp32"] * 1e-3) / 1e12
    line["roofline"] = {"bound": "fp32", "kernel": "somm_apply_keyed<float> + free-space pairs",
                        "achieved": achieved, "peak": fp32_peak / 1e3, "unit": "TFLOP/s",
                        "frac": achieved / (fp32_peak / 1e3),
                        "note": "lower bound: the whole FP32 application timed, only the "
                                "reflected term's ~100 flops per ordered pair counted; FP32 "
                                "FMA-chain peak; of measured"}
    if not args.no_cpu:
        from oracle import oracle as orc
        nt = orc.max_threads()
        rng = np.random.default_rng(5)
        m = 512
        dt = 0.0
        while True:
            ii, jj = rng.integers(0, n, m), rng.integers(0, n, m)
            t0 = time.perf_counter()
            orc.sommerfeld_tensor(somm, w.positions[ii], w.positions[jj], nt)
            dt = time.perf_counter() - t0
            if dt > min(args.cpu_seconds, 10.0) / 4 or m >= (1 << 22):
                break
            m *= 4
        t_pair = dt / m
        mv_ref = int(info64.get("matvecs_reference", info64["iterations"]))
        t_solve = t_pair * pairs * mv_ref
        line["cpu_baseline"] = {"value": n / t_solve, "unit": UNIT, "cores": nt, "kind": "port",
                                "sample": f"{m} random pairs of the reflected tensor "
                                          f"({dt:.1f} s), scaled to N^2 pairs per matvec x "
                                          f"{mv_ref} matvecs of the FP64 solve (free-space "
                                          f"term not counted: a lower bound on the "
                                          f"reference's time)", "cpu": _cpu_model()}
    return line


def _bench_harmonic(args, bk, stream, torch, lb, configs):
    """Second-harmonic response (nonlinear.rs:108-240) of the headline cuboid
    (60x50x10 nm Au, N = 30,000, FCD cell 1 nm): the linear FP32+refine solve
    at 800 nm (untimed), then compute_shg_response at 400 nm -- chi(2)
    sources from the local fields on the device and the harmonic GMRES(30)
    solve at tol 1e-8 through the solver's session dispatch (matrix-free at
    this size) -- timed end to end through the public call with host arrays."""
    from lumina_b200 import nonlinear
    w1 = configs.cuboid_au_30k(800.0)
    w2 = configs.cuboid_au_30k(400.0)
    n = w1.n
    solver = lb.CdaSolver(iterative_threshold=1000, use_fcd=True, cell_size=1.0, backend=bk,
                          precision="fp32_refine")
    params = lb.SimulationParams(solver_tolerance=1e-8, max_iterations=max(args.max_iter, 20000))
    resp = solver.solve_dipoles(lb.DipoleSet(w1.positions, w1.alpha), 800.0, params)
    d2 = lb.DipoleSet(w2.positions, w2.alpha)
    chi2 = [nonlinear.Chi2Tensor.isotropic_surface(1.0 + 0.2j, 0.4)]
    for _ in range(max(args.warmup, 1)):
        nonlinear.compute_shg_response(solver, resp, d2, chi2, params)
    times, r = [], None
    for _ in range(max(args.steps, 1)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = nonlinear.compute_shg_response(solver, resp, d2, chi2, params)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    info = r.solve_info
    line = {"metric": "dipole-solves/s, second-harmonic response of the N=30k cuboid "
                      "(sources + harmonic solve, FP32+refine)", "value": n / t, "unit": UNIT,
            "higher_is_better": True, "steps": len(times), "ms_per_step": t * 1e3,
            "scaling": "weak", "dtype": "f32+f64", "mode": "fp32_refine",
            "config": {"workload": "Au cuboid 60x50x10 nm (N=30,000), FCD 1 nm, fundamental "
                                   "800 nm, SHG at 400 nm, isotropic-surface chi(2), "
                                   "GMRES(30) tol 1e-8", "n_dipoles": n,
                       "operator": "the solver's dispatch: the block-Toeplitz FFT session "
                                   "for this lattice"},
            "iterations": info.get("iterations"), "converged": bool(info.get("converged")),
            "shg_intensity": r.intensity,
            "e2e": {"value": n / t, "unit": UNIT, "h2d_bytes_per_step": n * (24 + 144 + 48),
                    "d2h_bytes_per_step": n * 48}}
    if not args.no_cpu:
        mv = int(info.get("matvecs_reference") or info.get("iterations") or 1)
        line["cpu_baseline"] = cpu_baseline(w2, [mv], args.cpu_seconds)
    return line


# The periodic configuration's sweep: 101 points, 500-1000 nm; the bench
# samples every tenth (11 wavelengths) unless --wavelengths names others.
MSURF_SAMPLE_NM = ",".join(f"{500.0 + 50.0 * i:g}" for i in range(11))


def _bench_metasurface(args, bk, stream, torch, lb, configs):
    from oracle import oracle as orc
    lams = wavelength_list(args, MSURF_SAMPLE_NM)
    # 4 nm lattice: 5,379 dipoles per cell, the size the configuration quotes
    # (~4,900); its stated 2 nm lattice gives 41,181 (--spacing 2: ~3,100
    # Arnoldi steps per solve over the sample, minutes per wavelength)
    spacing = args.spacing or 4.0
    tol, max_iter = args.tol, max(args.max_iter, 20000)
    l2_peak = bk.measure_l2_peak()
    rows, parity, counts = [], None, []
    apply_ms, applies = 0.0, 0
    w0 = pw0 = None
    for lam in lams:
        pw = configs.metasurface(spacing=spacing, wavelength_nm=lam)
        w = pw.workload
        inv = lb.invert_polarisability(w.alpha)
        t0 = time.perf_counter()
        S = bk.create_onthefly_session(w.positions, inv, w.k, True, w.cell_size,
                                       lattice=pw.lattice, k_bloch=pw.k_bloch,
                                       substrate=pw.substrate)
        S.set_stream(stream.cuda_stream)
        setup_ms = (time.perf_counter() - t0) * 1e3
        b = torch.from_numpy(lb.incident_field(w.positions, w.k, pw.incident)).to("cuda")
        x32, x64 = torch.zeros_like(b), torch.zeros_like(b)
        for _ in range(args.warmup):
            try:
                S.solve_device(b.data_ptr(), x32.data_ptr(), tol, 31, 30, "fp32_refine",
                               stream.cuda_stream)
            except lb.ConvergenceFailure:
                pass
        S.profile(True)
        i32, ms32 = _timed(stream, lambda: S.solve_device(b.data_ptr(), x32.data_ptr(), tol,
                                                          max_iter, 30, "fp32_refine",
                                                          stream.cuda_stream))
        k32, kms32 = S.kernel_time("fp32")
        S.profile(False)
        apply_ms += kms32
        applies += i32["matvecs_fp32"]
        i64, ms64 = _timed(stream, lambda: S.solve_device(b.data_ptr(), x64.data_ptr(), tol,
                                                          max_iter, 30, "fp64",
                                                          stream.cuda_stream))
        counts.append(i64["matvecs_reference"])
        c32 = lb.cross_sections(w.positions, inv, x32.cpu().numpy(), w.k, pw.incident)
        c64 = lb.cross_sections(w.positions, inv, x64.cpu().numpy(), w.k, pw.incident)
        if parity is None:
            # both operators against the oracle's periodic rows (Ewald 5/5, Bloch
            # phase, Fresnel image) on 16 rows spread over the cell
            xr = np.random.default_rng(11).standard_normal(3 * w.n) * (1 + 0.5j)
            y64, y32 = S.matvec(xr, "fp64"), S.matvec(xr, "fp32")
            idx = np.linspace(0, w.n - 1, 16).astype(int)
            yref = np.concatenate([orc.matvec_onthefly_rows_ex(
                w.positions, w.alpha, xr, w.k, True, w.cell_size, i, i + 1, lattice=pw.lattice,
                k_bloch=pw.k_bloch, substrate=pw.substrate) for i in idx])
            sel = np.concatenate([np.arange(3 * i, 3 * i + 3) for i in idx])
            scale = np.max(np.abs(yref))
            parity = {"rows": len(idx), "wavelength_nm": lam,
                      "fp64_rel_err": float(np.max(np.abs(y64[sel] - yref)) / scale),
                      "fp32_rel_err": float(np.max(np.abs(y32[sel] - yref)) / scale)}
            w0, pw0 = w, pw
        rows.append({"wavelength_nm": lam, "n": w.n, "setup_ms": setup_ms, "ms_fp32_refine": ms32,
                     "ms_fp64": ms64, "iterations": i32["iterations"],
                     "iterations_fp64": i64["iterations"],
                     "converged": bool(i32["converged"] and i64["converged"]),
                     "cext_fp32_refine": c32[0], "cext_fp64": c64[0],
                     "cext_rel_err": abs(c32[0] - c64[0]) / abs(c64[0]),
                     "kernel_config": S.kernel_config()})
        S.close()
    n = rows[0]["n"]
    t32 = sum(r["ms_fp32_refine"] for r in rows)
    t64 = sum(r["ms_fp64"] for r in rows)
    # roofline of the FP32 table gather (tab_pairs): one 48-byte table entry
    # per ordered pair (self included) for the direct term and one for the
    # image term, gathered from L2
    avg_apply = apply_ms / max(applies, 1)
    bytes_apply = 2.0 * 48.0 * float(n) * float(n)
    achieved = bytes_apply / (avg_apply * 1e-3) / 1e9
    line = {"metric": "dipole-solves/s, periodic metasurface on a substrate (FP32+refine)",
            "value": n * len(rows) / (t32 * 1e-3), "unit": UNIT, "higher_is_better": True,
            "steps": len(rows), "ms_per_step": t32 / len(rows), "scaling": "weak",
            "dtype": "f32+f64", "mode": "fp32_refine",
            "config": {"workload": f"Au cylinder d100 h40 on a {spacing:g} nm lattice, square "
                                   f"period 400 nm, Ewald 5/5, 10 deg incidence, n=1.45 "
                                   f"substrate (Fresnel image)", "n_dipoles": n,
                       "wavelengths_nm": lams, "tol": tol,
                       "sweep": "every tenth point of the 101-point 500-1000 nm sweep"
                                if args.wavelengths == "sweep" else "as given",
                       "gold_beyond_table": f"J&C gold ends at {GOLD_TABLE_END_NM:g} nm; "
                                            "wavelengths past it use the natural spline's "
                                            "last interval extended"},
            "fp64_plain": {"value": n * len(rows) / (t64 * 1e-3), "speedup_same_solves": t64 / t32,
                           "max_cext_rel_err": max(r["cext_rel_err"] for r in rows)},
            "parity_vs_oracle_rows": parity,
            "roofline": {"bound": "l2", "kernel": "tab_pairs", "achieved": achieved,
                         "peak": l2_peak, "unit": "GB/s", "frac": achieved / l2_peak,
                         "peak_source": "L2 read microbenchmark in this run "
                                        "(lum_measure_l2_peak); of measured",
                         "avg_launch_ms": avg_apply, "bytes_per_launch": bytes_apply,
                         "applications": applies, "traffic": None},
            "per_wavelength": rows,
            "e2e": None}
    if not args.no_e2e:
        # e2e: the same wavelengths through CdaSolver with host arrays (its
        # on-the-fly branch with the lattice sum and the Fresnel image; a new
        # session per wavelength, as k_bloch changes with it), setup included
        t_e2e = 0.0
        for lam in lams:
            pw = configs.metasurface(spacing=spacing, wavelength_nm=lam)
            w = pw.workload
            solver = lb.CdaSolver(backend=bk, iterative_threshold=0, use_fcd=True,
                                  cell_size=w.cell_size, lattice=pw.lattice,
                                  incident_field=pw.incident, matrix_memory_budget=0,
                                  precision="fp32_refine", use_fft=False)
            params = lb.SimulationParams(solver_tolerance=tol, max_iterations=max_iter,
                                         k_bloch=pw.k_bloch, substrate_runtime=pw.substrate)
            ds = lb.DipoleSet(w.positions, w.alpha)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            solver.compute_cross_sections(ds, lam, params)
            t_e2e += time.perf_counter() - t0
            solver.close()
        line["e2e"] = {"value": n * len(lams) / t_e2e, "unit": UNIT,
                       "h2d_bytes_per_step": n * (24 + 144),
                       "d2h_bytes_per_step": n * 48,
                       "includes": "session setup (lattice tables) per wavelength"}
    if not args.no_cpu:
        t_mv, nrows, dt, nt = cpu_matvec_sample(w0, args.cpu_seconds, periodic=pw0)
        line["cpu_baseline"] = {
            "value": n * len(counts) / (t_mv * sum(counts)), "unit": UNIT, "cores": nt,
            "kind": "port",
            "sample": f"{nrows} of {n} rows of one FP64 periodic oracle matvec (Ewald 5/5 + "
                      f"Fresnel image, {dt:.1f} s), scaled by the reference GMRES(30)'s "
                      f"operator applications ({sum(counts)} over {len(counts)} wavelengths, "
                      f"counted by the device FP64 solves)",
            "extrapolated": True, "matvec_seconds": t_mv}
    return line


if __name__ == "__main__":
    sys.exit(main())
