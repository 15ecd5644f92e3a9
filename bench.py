"""Benchmark: grid-pt*state*steps/s of the split-operator propagator on B200.

Workload (the reference configuration the headline metric is quoted on): the
1-D two-state avoided crossing, V11 = 0.01 tanh(1.6x) = -V22,
V12 = 0.005 exp(-x^2), mass 2000, 8192 points on [-24, 24], Gaussians at
x0 = -10 with sigma = 20/p0 for p0 in {10, 15, 20, 25, 30} (5 jobs), dt = 1,
4000 steps, adiabatic populations recorded every step.  One bench step is one
full propagation of the 5-job batch (5 x 8192 x 2 x 4000 grid-pt*state*steps).
Inputs are synthetic (generated here), no dataset is involved.

Legs printed in one JSON line:
  value      FP32 batched form, tables resident on the device, device time
             (CUDA events on the library's stream), L2 flushed between steps;
  fp64       the plain FP64 form on the same batch;
  e2e        zqd_run_batch through the public API from host options to host
             results (table setup, H2D, D2H inside the timed region);
  roofline   the resident line kernel against the measured HBM copy bandwidth;
  cpu_baseline  the oracle port, single thread, on a bounded sample;
  nd         2-D 512^2 x 3 states, 3-D 128^3 (ITP and real time), 2-D 2048^2 x 2
             states (larger than L2): FP32 and FP64 device time, HBM roofline;
  serving    a seeded stream of 600 jobs (Poisson arrivals, 200 jobs/s) through
             the job server: p50/p99 latency, throughput, burst throughput, FP32 vs
             FP64 error, and the plain FP64 form on the same stream (each job alone
             through zqd_run, one after another);
  fp32_errors  per configuration, FP32 against FP64: wavefunction rel. L2,
             largest population error, energy difference and drift;
  fft_brackets cuFFT against the library's FFT seam on the device, pocketfft
             (scipy.fft, every host thread) against the oracle's FFT on the host.
`--impl reference` times the CPU restatement of the reference path (the
oracle) with all host threads on the same workload.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grid-pt*state*steps/s (FP32-batched vs FP64, 1 B200)"
UNIT = "grid-pt*state*steps/s"
MOMENTA = (10.0, 15.0, 20.0, 25.0, 30.0)
NPOINT, NSTATE, ITERS = 8192, 2, 4000
# algorithmic bytes per grid-pt*state*step of a 1-D two-state step:
# psi read+write once (2*S*c per point) plus two reads of the complex R table (2*S^2*c), over S
BYTES_PER_UNIT = {"fp64": (2 * 1 * NSTATE * 16 + 2 * NSTATE**2 * 16) / NSTATE,
                  "fp32": (2 * 1 * NSTATE * 8 + 2 * NSTATE**2 * 8) / NSTATE}


def workload(iters=ITERS):
    opts = []
    for p0 in MOMENTA:
        opts.append({
            "grid": {"bounds": [[-24, 24]], "npoint": NPOINT},
            "initial_conditions": {"position": [-10.0], "momentum": [p0], "gamma": [p0 * p0 / 400.0], "state": 0,
                                   "adiabatic": True},
            "potential": {"custom": {"ndim": 1, "matrix": [["0.01*tanh(1.6*r1)", "0.005*exp(-r1^2)"],
                                                           ["0.005*exp(-r1^2)", "-0.01*tanh(1.6*r1)"]]}},
            "mass": [2000.0], "iterations": iters, "time_step": 1.0, "adiabatic": True,
            "write": {"population": "POP.mat"},
        })
    return opts


def units(opts):
    return sum(o["grid"]["npoint"] ** len(o["grid"]["bounds"]) * NSTATE * o["iterations"] for o in opts)


# ---------------------------------------------------------------- N-D workloads (reported beside the headline)
def coupled_harmonic_2d(npoint=512, iters=2000):
    """2-D three-state coupled harmonic surfaces, 512^2 on [-12, 12]^2, dt 0.05; constants from a fixed seed."""
    import numpy as np

    rng = np.random.default_rng(20261203)
    a, b, c = rng.uniform(-1, 1, 3), rng.uniform(-1, 1, 3), rng.uniform(0, 0.2, 3)
    coup = "0.05*exp(-(r1^2+r2^2)/2)"
    mat = [[(f"0.5*(r1^2+r2^2)+{a[i]:.17g}*r1+{b[i]:.17g}*r2+{c[i]:.17g}" if i == j else coup) for j in range(3)]
           for i in range(3)]
    return {"grid": {"bounds": [[-12, 12], [-12, 12]], "npoint": npoint},
            "initial_conditions": {"position": [-2, 0], "momentum": [1, 0], "gamma": [1, 1], "state": 0,
                                   "adiabatic": False},
            "potential": {"custom": {"ndim": 2, "matrix": mat}}, "mass": [1, 1], "iterations": iters,
            "time_step": 0.05, "adiabatic": False, "write": {"population": "P", "total_energy": "E", "norm": "N"}}


def anharmonic_3d(iters, imaginary):
    """3-D anharmonic well, 128^3 on [-8, 8]^3, dt 0.02: imaginary-time relaxation or real time with the ACF."""
    opt = {"grid": {"bounds": [[-8, 8]] * 3, "npoint": 128},
           "initial_conditions": {"position": [1, 1, 1], "momentum": [0, 0, 0], "gamma": [1, 1, 1], "state": 0,
                                  "adiabatic": False},
           "potential": {"custom": {"ndim": 3, "matrix": [["0.5*(r1^2+r2^2+r3^2)+0.1*(r1^2*r2-r2^3/3)+0.05*r3^4"]]}},
           "mass": [1, 1, 1], "iterations": iters, "time_step": 0.02, "adiabatic": False,
           "write": {} if imaginary else {"acf": "A"}}
    if imaginary:
        opt["imaginary"] = {"nstate": 1}
    return opt


def wide_grid_2d(iters=100):
    """2-D two-state grid of 2048^2 (134 MB of FP64 wavefunction, larger than L2): the HBM-bound case."""
    mat = [["0.5*(r1^2+r2^2)", "0.01*exp(-r1^2)"], ["0.01*exp(-r1^2)", "0.5*(r1^2+r2^2)+0.1"]]
    return {"grid": {"bounds": [[-20, 20], [-20, 20]], "npoint": 2048},
            "initial_conditions": {"position": [-2, 0], "momentum": [1, 0], "gamma": [1, 1], "state": 0,
                                   "adiabatic": False},
            "potential": {"custom": {"ndim": 2, "matrix": mat}}, "mass": [1, 1], "iterations": iters,
            "time_step": 0.05, "adiabatic": False, "write": {"population": "P"}}


def nd_bytes_per_step(opt, c):
    """Algorithmic bytes of one step: N [2 (2d-1) S c + 2 S^2 c + a S c] (+ (2d-1) S N c with ekin/mom)."""
    d = len(opt["grid"]["bounds"])
    N = opt["grid"]["npoint"] ** d
    S = len(opt["potential"]["custom"]["matrix"])
    w = opt.get("write") or {}
    a = 1 if "acf" in w else 0
    b = N * (2 * (2 * d - 1) * S * c + 2 * S * S * c + a * S * c)
    if any(k in w for k in ("kinetic_energy", "momentum", "total_energy")):
        b += (2 * d - 1) * S * N * c
    return b


def nd_bytes_moved(opt, c):
    """Bytes the N-D kernels themselves read and write in one step (each array once per pass):
    the row pass reads and writes psi and reads the upper triangle of R (16-byte entries in both
    forms: FP32 keeps an FP64-accurate hi + lo pair), the autocorrelation reference, the CAP weight
    and the eigenvectors where they are used (stop_norm, a time-dependent potential and imaginary
    time with earlier states split it into three launches, and imaginary time renormalises; one
    relaxed state defers its renormalisation into the next step's passes and moves what real time
    moves); every tile pass (one in 2-D, three in 3-D) reads
    and writes psi; a step that records momentum observables also writes phi and runs the momentum
    tile passes over it."""
    d = len(opt["grid"]["bounds"])
    N = opt["grid"]["npoint"] ** d
    S = len(opt["potential"]["custom"]["matrix"])
    w = opt.get("write") or {}
    nsym = S * (S + 1) // 2
    b = N * (2 * S * c + nsym * 16)
    if "acf" in w:
        b += N * S * c
    if opt.get("absorbing_potential", {}).get("track_population"):
        b += N * 8
    if opt.get("adiabatic") and S > 1 and "population" in w:
        b += N * S * S * 8
    if any(k in w for k in ("potential_energy", "total_energy")):
        b += N * S * (S + 1) // 2 * 8
    cap = bool(opt.get("absorbing_potential"))
    if opt.get("imaginary") and (opt["imaginary"].get("nstate", 1) == 1) and not cap:
        pass  # the renormalisation rides on the step's own passes
    elif opt.get("imaginary") or opt.get("absorbing_potential", {}).get("stop_norm"):
        # the row pass runs in three launches (end of step, observables, start of the next step)
        b += 3 * N * S * c + nsym * 16 * N
        if opt.get("imaginary"):
            b += 3 * N * S * c  # renormalisation: the norm's sums, then psi rescaled
    tile_passes = 1 if d == 2 else 3
    b += tile_passes * 2 * S * N * c
    if any(k in w for k in ("kinetic_energy", "momentum", "total_energy")):
        b += N * S * c + (2 * (d - 2) + 1) * S * N * c  # phi written; momentum tile passes
    return b


def nd_units(opt):
    d = len(opt["grid"]["bounds"])
    return opt["grid"]["npoint"] ** d * len(opt["potential"]["custom"]["matrix"]) * opt["iterations"]


def config(extra=None):
    c = {"workload": "1-D two-state tanh crossing, 8192 pts x 2 states, 5 momenta, 4000 steps, dt 1",
         "jobs": len(MOMENTA), "npoint": NPOINT, "nstate": NSTATE, "iterations": ITERS,
         "l2": "flushed between timed steps (512 MiB write)"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------- CPU legs
def oracle_sample(opts, threads, per_job=1):
    """The oracle on opts: `threads` jobs at a time, each with `per_job` threads of its own."""
    from oracle import qd_ref

    t0 = time.perf_counter()
    if threads == 1:
        res = [qd_ref.run(o, nthreads=per_job, want_wavefunction=False) for o in opts]
    else:
        with cf.ThreadPoolExecutor(max_workers=threads) as ex:
            res = list(ex.map(lambda o: qd_ref.run(o, nthreads=per_job, want_wavefunction=False), opts))
    return time.perf_counter() - t0, res


def reference_arm(args, rank):
    if rank != 0:
        return
    sample_iters = ITERS  # the whole workload per step: 5 jobs x 4000 steps, all jobs in parallel threads
    opts = workload(sample_iters)
    nproc = os.cpu_count() or 1
    threads = min(len(opts), nproc)
    per_job = max(1, nproc // threads)  # every host thread: the jobs side by side, each on its share of the cores
    for _ in range(args.warmup):
        oracle_sample(opts, threads, per_job)
    tot = 0.0
    for _ in range(args.steps):
        dt, _ = oracle_sample(opts, threads, per_job)
        tot += dt
    value = units(opts) * args.steps / tot
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": config({"sample": f"{len(opts)} jobs x {sample_iters} steps per bench step (the whole workload)"}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads * per_job, "kind": "port",
                             "sample": f"{len(opts)} jobs x {sample_iters} steps, the jobs in parallel, "
                                       f"{per_job} threads each"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU legs
class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, gpu_index, path):
        self.path = path
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.proc = None
        try:
            self.f = open(path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(gpu_index), "-lms", "50"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.1)
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


TRAFFIC_FILE = os.path.join(ROOT, "profiles", "traffic.txt")


def read_traffic(kernel, precision):
    """DRAM bytes per launch from profiles/traffic.txt: an ncu capture of the same kernel on the same
    workload, tabulated by `python bench.py --traffic-table <ncu csv> <label>` (the capture's
    command heads that file; this run does not measure it)."""
    if not os.path.exists(TRAFFIC_FILE):
        return None
    for line in open(TRAFFIC_FILE):
        p = line.split()
        if len(p) >= 3 and p[0] == kernel and p[1] == precision:
            return float(p[2])
    return None


def traffic_table(csv_path, label):
    """Rows "kernel precision[_label] dram_bytes_per_launch" from an ncu --csv capture with
    gpu__time_duration.sum, dram__bytes_read.sum and dram__bytes_write.sum: per kernel and
    precision, the mean read + write bytes of the launches of its dominant grid (the grid with the
    most device time, e.g. the bench's batched launch rather than the autotuner's candidates)."""
    import csv

    per = {}
    with open(csv_path) as f:
        lines = [ln for ln in f if ln.startswith('"')]
    for row in csv.DictReader(lines):
        metric = row.get("Metric Name", "")
        full = row["Kernel Name"]
        name = full.split("<")[0].split("(")[0].replace("void ", "").replace("zqd::", "").strip()
        prec = "fp32" if "<float" in full else "fp64" if "<double" in full else "-"
        rec = per.setdefault(row["ID"], {"key": (name, prec, row.get("Grid Size", "")), "bytes": 0.0, "ns": 0.0})
        unit = row.get("Metric Unit", "").lower()
        v = float(row["Metric Value"].replace(",", ""))
        if metric in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
            rec["bytes"] += v * {"byte": 1, "kbyte": 1e3, "mbyte": 1e6, "gbyte": 1e9}.get(unit, 1)
        elif metric == "gpu__time_duration.sum":
            rec["ns"] += v * {"ns": 1, "nsecond": 1, "us": 1e3, "usecond": 1e3, "ms": 1e6, "msecond": 1e6}.get(unit, 1)
    groups = {}
    for rec in per.values():
        g = groups.setdefault(rec["key"], {"bytes": [], "ns": 0.0})
        g["bytes"].append(rec["bytes"])
        g["ns"] += rec["ns"]
    best = {}
    for (name, prec, grid), g in groups.items():
        if (name, prec) not in best or g["ns"] > best[(name, prec)][1]["ns"]:
            best[(name, prec)] = (grid, g)
    out = []
    for (name, prec), (grid, g) in sorted(best.items()):
        tag = prec + ("_" + label if label else "")
        out.append(f"{name} {tag} {statistics.mean(g['bytes']):.4g}  # grid {grid}, {len(g['bytes'])} launches")
    return out


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return float(json.load(open(path))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def nd_legs(qd, torch, flush, reps=2):
    """2-D and 3-D workloads on one GPU: device time per run (graph replay), HBM roofline per step."""
    import numpy as np

    peak, peak_kind = measured_peak()
    cases = [("2d_512sq_3states_2000steps", coupled_harmonic_2d()),
             ("3d_128cube_itp_500steps", anharmonic_3d(500, True)),
             ("3d_128cube_realtime_acf_2000steps", anharmonic_3d(2000, False)),
             ("2d_2048sq_2states_100steps_larger_than_l2", wide_grid_2d())]
    out = {}
    for name, opt in cases:
        leg = {"units_per_run": nd_units(opt)}
        pops = {}
        d, n = len(opt["grid"]["bounds"]), opt["grid"]["npoint"]
        S = len(opt["potential"]["custom"]["matrix"])
        for prec in ("fp32", "fp64"):
            # the library's autotuner for the (dims, points, states, precision) key, outside the timing
            tuned = qd.autotune(d, n, S, prec)
            job = qd.Job(opt, prec)
            job.run()  # captures the run's graph; warm-up
            ts = []
            for _ in range(reps):
                flush.fill_(1.0)
                torch.cuda.synchronize()
                ts.append(job.run())
            ms = statistics.mean(ts)
            c = 16 if prec == "fp64" else 8
            bstep = nd_bytes_per_step(opt, c)
            bmoved = nd_bytes_moved(opt, c)
            achieved = bstep * opt["iterations"] / (ms / 1e3) / 1e9
            moved = bmoved * opt["iterations"] / (ms / 1e3) / 1e9
            leg[prec] = {"value": nd_units(opt) / (ms / 1e3), "unit": UNIT, "ms_per_run": ms,
                         "us_per_step": 1e3 * ms / opt["iterations"],
                         "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                      "frac": achieved / peak, "bytes_per_step": bstep, "peak_kind": peak_kind,
                                      "moved": {"bytes_per_step": bmoved, "achieved": moved, "frac": moved / peak,
                                                "note": "the bytes the kernels read and write per step "
                                                        "(bench.nd_bytes_moved); DRAM traffic is lower where the "
                                                        "working set stays in the 126 MB L2"}},
                         "autotune": {k: tuned[k] for k in ("us_per_step", "default_us_per_step", "candidates",
                                                            "tma_row_block", "tma_tile_lines", "rows_per_cta",
                                                            "tile_lines")}}
            h = job.result(want_wavefunction=False).observables[0].history
            if "population" in h:
                pops[prec] = h["population"]
            job.close()
        leg["fp32_over_fp64"] = leg["fp32"]["value"] / leg["fp64"]["value"]
        if len(pops) == 2:
            leg["pop_err_fp32_vs_fp64"] = float(np.max(np.abs(pops["fp32"] - pops["fp64"])))
        out[name] = leg
    return out


SERVE_JOBS, SERVE_RATE, SERVE_MAX_STEPS = 600, 200.0, 1000


def harmonic_1d():
    """1-D harmonic oscillator, 1024 points on [-16, 16], psi0 ~ exp(-(x-1)^2/2), dt 0.1, 1000 steps."""
    return {"grid": {"bounds": [[-16, 16]], "npoint": 1024},
            "initial_conditions": {"position": [1], "momentum": [0], "gamma": [1], "state": 0},
            "potential": {"harmonic": {"k": [1]}}, "mass": [1], "iterations": 1000, "time_step": 0.1,
            "write": {"norm": "N", "total_energy": "E", "position": "X"}}


def config_table(qd):
    """Per-configuration rates in grid-pt*state*steps/s: the oracle on the host (one thread and all
    threads, bounded samples of each workload) and the GPU forms, for the comparison table."""
    import numpy as np

    from oracle import qd_ref

    nproc = os.cpu_count() or 1

    def rate(opt, **kw):
        d = len(opt["grid"]["bounds"])
        S = 1 if "harmonic" in opt["potential"] else len(opt["potential"]["custom"]["matrix"])
        u = opt["grid"]["npoint"] ** d * S * opt["iterations"] * max(1, (opt.get("imaginary") or {}).get("nstate", 1))
        t0 = time.perf_counter()
        qd_ref.run(opt, want_wavefunction=False, **kw)
        return u / (time.perf_counter() - t0)

    def sample(opt, iters):
        o = dict(opt)
        o["iterations"] = iters
        return o

    cases = [("1_harmonic_1d", harmonic_1d(), 1000), ("2_tanh_crossing_1d_p20", workload()[2], 1000),
             ("3_coupled_2d_512sq", coupled_harmonic_2d(), 10), ("4_anharmonic_3d_128cube_itp", anharmonic_3d(500, True), 6),
             ("4_anharmonic_3d_128cube_rt", anharmonic_3d(2000, False), 6)]
    out = {"host_threads": nproc}
    for name, opt, iters in cases:
        o = sample(opt, iters)
        row = {"cpu_1thread": rate(o, nthreads=1), "cpu_all": rate(o, nthreads=nproc), "cpu_sample_steps": iters}
        for prec in ("fp64", "fp32"):
            job = qd.Job(opt, prec)
            job.run()
            ms = statistics.mean([job.run() for _ in range(2)])
            d = len(opt["grid"]["bounds"])
            S = 1 if "harmonic" in opt["potential"] else len(opt["potential"]["custom"]["matrix"])
            row["gpu_" + prec] = opt["grid"]["npoint"] ** d * S * opt["iterations"] / (ms / 1e3)
            job.close()
        out[name] = row
    # serving: the oracle on a 50-job subset of the stream (steps <= 300), all threads, one job per thread
    sub, _ = qd.serving_stream(50, seed=7, max_steps=300)
    u = sum(o["grid"]["npoint"] ** len(o["grid"]["bounds"]) * len(o["potential"]["custom"]["matrix"]) * o["iterations"]
            for o in sub)
    dt, _ = oracle_sample(sub, nproc)
    out["5_serving_subset_50jobs"] = {"cpu_all": u / dt}
    return out


def serving_leg(qd):
    """The serving stream (seeded generator, Poisson arrivals at 200 jobs/s) through the job server:
    p50/p99 submit-to-completion latency and throughput at that rate, throughput with every job
    submitted at once (capacity, the median of three such bursts), FP32 population error against
    the FP64 form job by job; the same
    for precision "auto" (FP32 unless a job's smallest adiabatic gap is below 1e-3 Hartree)."""
    import numpy as np

    opts, arrivals = qd.serving_stream(SERVE_JOBS, seed=7, rate_per_s=SERVE_RATE, max_steps=SERVE_MAX_STEPS)
    units = sum(o["grid"]["npoint"] ** len(o["grid"]["bounds"]) * len(o["potential"]["custom"]["matrix"]) * o["iterations"]
                for o in opts)
    # the autotuner over the stream's 2-D keys (the 1-D jobs take the single-CTA service kernel or the
    # cluster shapes of their line length), outside the timing; served and plain runs share the table
    keys2d = sorted({(o["grid"]["npoint"], len(o["potential"]["custom"]["matrix"])) for o in opts
                     if len(o["grid"]["bounds"]) == 2})
    for n, S in keys2d:
        for prec in ("fp32", "fp64"):
            qd.autotune(2, n, S, prec)
    w_opts, w_arr = qd.serving_stream(60, seed=8, rate_per_s=2000.0, max_steps=200)
    qd.serve_stream(w_opts, w_arr, "fp32")  # warm-up: module loading, memory pool
    qd.serve_stream(w_opts, w_arr, "fp64")
    out = {"jobs": SERVE_JOBS, "arrival_rate_per_s": SERVE_RATE, "steps": f"100..{SERVE_MAX_STEPS}",
           "autotuned_2d_keys": len(keys2d) * 2,
           "workload": "seeded stream: 1-D 256..16384 pts or 2-D 64^2..512^2, 1-3 states, harmonic or tanh-crossing",
           "units": units}
    pops, forms = {}, {}
    for prec in ("fp32", "fp64", "auto"):
        # the populations are compared; the final wavefunctions are not downloaded
        res, lat, wall, st = qd.serve_stream(opts, arrivals, prec, fetch_wavefunction=False)
        lat = np.asarray(lat)
        # capacity: every job submitted at once, the median of three bursts (one varies by +-15 %)
        walls_b = [qd.serve_stream(opts, [0.0] * len(opts), prec, fetch_wavefunction=False)[2] for _ in range(3)]
        wall_b = statistics.median(walls_b)
        out[prec] = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                     "throughput": units / wall, "unit": UNIT, "wall_s": wall,
                     "burst_throughput": units / wall_b, "burst_wall_s": wall_b, "burst_walls_s": walls_b,
                     "grouped_launches": st["grouped_launches"], "grouped_jobs": st["grouped_jobs"],
                     "joined_jobs": st["joined_jobs"], "service_jobs": st["service_jobs"],
                     "service_launches": st["service_launches"], "peak_device_bytes": st["peak_device_bytes"]}
        out[prec]["failed_jobs"] = len(st["failures"])
        pops[prec] = [r.observables[0].history["population"] if r is not None else None for r in res]
        forms[prec] = [r.precision if r is not None else None for r in res]
    def errs_of(x, y):  # a failed or non-finite job counts as an infinite error, never silently skipped
        e = []
        for a, b in zip(x, y):
            if a is None or b is None or not (np.all(np.isfinite(a)) and np.all(np.isfinite(b))):
                e.append(float("inf"))
            else:
                e.append(float(np.max(np.abs(a - b))))
        return e

    errs = errs_of(pops["fp32"], pops["fp64"])
    out["pop_err_fp32_vs_fp64"] = max(errs)
    out["jobs_over_1e-5"] = sum(e > 1e-5 for e in errs)
    errs_auto = errs_of(pops["auto"], pops["fp64"])
    out["auto"]["pop_err_vs_fp64"] = max(errs_auto)
    out["auto"]["jobs_over_1e-5"] = sum(e > 1e-5 for e in errs_auto)
    out["auto"]["jobs_fp64"] = sum(f == "fp64" for f in forms["auto"])
    out["burst_fp32_over_fp64"] = out["fp32"]["burst_throughput"] / out["fp64"]["burst_throughput"]
    # the plain FP64 form on the same stream: every job alone through zqd_run, one after another
    t0 = time.perf_counter()
    lat_plain = []
    for o in opts:
        t1 = time.perf_counter()
        qd.run(o, precision="fp64", want_wavefunction=False)
        lat_plain.append(1e3 * (time.perf_counter() - t1))
    wall_plain = time.perf_counter() - t0
    out["plain_fp64_sequential"] = {"throughput": units / wall_plain, "unit": UNIT, "wall_s": wall_plain,
                                    "p50_job_ms": float(np.percentile(lat_plain, 50)),
                                    "note": "each job alone through zqd_run (FP64), one after another"}
    out["served_fp32_burst_over_plain_fp64"] = out["fp32"]["burst_throughput"] / out["plain_fp64_sequential"]["throughput"]
    out["served_auto_burst_over_plain_fp64"] = out["auto"]["burst_throughput"] / out["plain_fp64_sequential"]["throughput"]
    return out


def fp32_error_table(qd):
    """north_star (3): per configuration, the FP32 form's error against the FP64 form (which the tests
    hold to the oracle at 1e-10 / 1e-12): relative L2 of the final wavefunction, the largest population
    error over the run, the largest total-energy difference over the run and the energy drift
    |E(T) - E(0)| of each form."""
    import numpy as np

    def with_energy(opt):
        o = dict(opt)
        o["write"] = dict(opt.get("write") or {}, total_energy="E", population="P")
        return o

    cases = [("1_harmonic_1d", with_energy(harmonic_1d()))]
    cases += [(f"2_tanh_crossing_p{int(o['initial_conditions']['momentum'][0])}", with_energy(o)) for o in workload()]
    cases += [("3_coupled_2d_512sq", with_energy(coupled_harmonic_2d())),
              ("4_anharmonic_3d_itp", with_energy(anharmonic_3d(500, True))),
              ("4_anharmonic_3d_realtime", with_energy(anharmonic_3d(2000, False)))]
    out = {}
    for name, opt in cases:
        r = {p: qd.run(opt, precision=p).observables[0] for p in ("fp64", "fp32")}
        a, b = r["fp32"], r["fp64"]
        ea, eb = a.history["total_energy"].ravel(), b.history["total_energy"].ravel()
        out[name] = {
            "psi_rel_l2": float(np.linalg.norm(a.wavefunction - b.wavefunction) / np.linalg.norm(b.wavefunction)),
            "pop_max_err": float(np.max(np.abs(a.history["population"] - b.history["population"]))),
            "energy_max_diff": float(np.max(np.abs(ea - eb))),
            "energy_drift_fp32": float(abs(ea[-1] - ea[0])), "energy_drift_fp64": float(abs(eb[-1] - eb[0])),
        }
    return out


def fft_brackets(qd, torch, reps=20):
    """Transform-only timings at the workloads' sizes (FP64 complex, forward + inverse):
    cuFFT (torch.fft) against the library's FFT seam (zqd_fft_execute) on the same device buffer,
    and on the host pocketfft (scipy.fft, every host thread) against the oracle's own FFT, which
    brackets how far the CPU port's radix-2/4 FFT is from an FFTW-class FFT."""
    import ctypes as C

    import numpy as np
    import scipy.fft

    from oracle import qd_ref
    from zinq_b200 import _abi

    L = _abi.load()
    nproc = os.cpu_count() or 1
    out = {"host_threads": nproc}
    for name, shape in (("1d_8192", (8192,)), ("2d_512sq", (512, 512)), ("3d_128cube", (128, 128, 128)),
                        ("2d_2048sq", (2048, 2048))):
        x = torch.randn(*shape, dtype=torch.complex128, device="cuda")
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        dims = tuple(range(len(shape)))
        for _ in range(3):
            torch.fft.ifftn(torch.fft.fftn(x, dim=dims), dim=dims)
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(reps):
            y = torch.fft.ifftn(torch.fft.fftn(x, dim=dims), dim=dims)
        ev1.record()
        torch.cuda.synchronize()
        cufft_ms = ev0.elapsed_time(ev1) / reps
        plans = []
        for sign in (-1, 1):
            h = C.c_void_p()
            arr = (C.c_int * len(shape))(*shape)
            _abi.check(L.zqd_fft_plan_create(len(shape), arr, sign, 0, C.byref(h)))
            plans.append(h)
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        buf = C.c_void_p(x.data_ptr())
        for _ in range(3):
            for h in plans:
                _abi.check(L.zqd_fft_execute(h, buf, stream))
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(reps):
            for h in plans:
                _abi.check(L.zqd_fft_execute(h, buf, stream))
        ev1.record()
        torch.cuda.synchronize()
        own_ms = ev0.elapsed_time(ev1) / reps
        for h in plans:
            L.zqd_fft_destroy(h)
        del x, y
        hx = np.random.default_rng(1).standard_normal(shape) + 1j * np.random.default_rng(2).standard_normal(shape)
        nrep = max(1, int(2e7 // hx.size))
        t0 = time.perf_counter()
        for _ in range(nrep):
            scipy.fft.ifftn(scipy.fft.fftn(hx, workers=nproc), workers=nproc)
        pocket_ms = 1e3 * (time.perf_counter() - t0) / nrep
        t0 = time.perf_counter()
        for _ in range(nrep):
            scipy.fft.ifftn(scipy.fft.fftn(hx, workers=1), workers=1)
        pocket1_ms = 1e3 * (time.perf_counter() - t0) / nrep
        t0 = time.perf_counter()
        for _ in range(nrep):
            qd_ref.fft(qd_ref.fft(hx, -1), 1)
        port_ms = 1e3 * (time.perf_counter() - t0) / nrep
        out[name] = {"cufft_ms": cufft_ms, "zqd_fft_seam_ms": own_ms, "seam_over_cufft": own_ms / cufft_ms,
                     "host_pocketfft_ms": pocket_ms, "host_pocketfft_1thread_ms": pocket1_ms,
                     "host_oracle_fft_ms": port_ms, "oracle_fft_over_pocketfft_1thread": port_ms / pocket1_ms}
    return out


def line_step_model(n, S, C, lrmax, c):
    """Shared-memory traffic and barriers of one step of the resident 1-D kernel, per CTA: local
    Stockham passes of m = n/C points (largest radix 2^lrmax) forward and inverse, each reading and
    writing S*m values; their twiddles (16-byte table entries, R-1 per R-point butterfly, from the
    second pass on); the propagator R applied twice (upper triangle, 16-byte entries); the cluster
    twiddles and kinetic phase; the exchange across the cluster (DSMEM reads and local writes).
    Barriers: one per pass, three more per step in the CTA, three across the cluster."""
    import math

    m = n // C
    logm = int(math.log2(m))
    P = -(-logm // lrmax)
    R = 2 ** lrmax
    nsym = S * (S + 1) // 2
    passes = 2 * P * 2 * S * m * c
    twiddles = 2 * max(P - 1, 0) * (R - 1) / R * S * m * 16
    rtab = 2 * nsym * m * 16
    phases = (3 if C > 1 else 1) * m * 16
    exchange = 3 * S * m * c if C > 1 else 0
    return {"smem_bytes_per_cta": passes + twiddles + rtab + phases + exchange,
            "cta_barriers": 2 * P + 3, "cluster_barriers": 3 if C > 1 else 0, "m": m, "passes_per_transform": P}


def onchip_roofline(L, step_us, n, S, C, lrmax, c, ctas):
    """roofline_onchip: the resident kernel's shared-memory bytes per step against the measured per-SM
    shared-memory bandwidth, and its barrier-latency floor (barriers x measured latency) against the
    measured step time.  Neither is a DRAM roof: the wavefunction never leaves shared memory."""
    import ctypes as C_

    from zinq_b200 import _abi

    o = _abi.ZqdOnchip()
    _abi.check(L.zqd_measure_onchip(C_.byref(o)))
    mod = line_step_model(n, S, C, lrmax, c)
    per_sm = mod["smem_bytes_per_cta"] / (step_us * 1e-6) / 1e9
    floor_cycles = mod["cta_barriers"] * o.syncthreads_cycles + mod["cluster_barriers"] * o.cluster_barrier_cycles
    floor_us = floor_cycles / (o.sm_clock_mhz)
    return {"bound": "latency", "us_per_step": step_us, "ctas": ctas,
            "smem": {"bytes_per_cta_per_step": mod["smem_bytes_per_cta"], "achieved_gbs_per_sm": per_sm,
                     "peak_gbs_per_sm": o.smem_gbs_per_sm, "peak_bytes_per_cycle_per_sm": o.smem_bytes_per_cycle_per_sm,
                     "frac": per_sm / o.smem_gbs_per_sm, "peak_kind": "measured (zqd_measure_onchip)"},
            "barriers": {"cta_per_step": mod["cta_barriers"], "cluster_per_step": mod["cluster_barriers"],
                         "syncthreads_cycles": o.syncthreads_cycles, "cluster_barrier_cycles": o.cluster_barrier_cycles,
                         "floor_us_per_step": floor_us, "frac": floor_us / step_us},
            "shape": {"npoint": n, "states": S, "cluster_ctas": C, "radix": 2 ** lrmax, "points_per_cta": mod["m"]}}


def max_over_ranks(x, dist, device):
    """The largest of every rank's x (the timed region of the slowest replica); x itself without a group."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank, world, steps, seconds_max):
    """Whole-job throughput of `world` replicas: every rank's units over the slowest rank's time."""
    return world * units_per_rank * steps / seconds_max


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="zinq_b200", choices=["zinq_b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-nd", action="store_true", help="skip the 2-D / 3-D legs")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-stream leg")
    ap.add_argument("--profile-case", choices=["fp64", "fp32"], default=None,
                    help="run a small case of the bench workload (1 job x 200 steps) twice and exit; for ncu captures")
    ap.add_argument("--nd-case", nargs=3, metavar=("WORKLOAD", "PRECISION", "STEPS"), default=None,
                    help="run one 2-D/3-D workload (c3 | c3pop | c3pop1 | c3pop2 | c4 | c4itp | wide) for STEPS steps "
                         "twice and exit; "
                         "for ncu captures")
    ap.add_argument("--table", action="store_true",
                    help="print per-configuration CPU (oracle) and GPU rates as one JSON line and exit")
    ap.add_argument("--clocks-csv", default=None,
                    help="where the nvidia-smi samples of the timed region go (default: the system temp dir)")
    ap.add_argument("--traffic-table", nargs=2, metavar=("NCU_CSV", "LABEL"), default=None,
                    help="print 'kernel LABEL dram_bytes_per_launch' rows from an ncu --csv capture and exit")
    ap.add_argument("--no-extra", action="store_true", help="skip the FP32 error table and the FFT brackets")
    args = ap.parse_args()

    if args.traffic_table:
        print("\n".join(traffic_table(*args.traffic_table)))
        return

    if args.table:
        from zinq_b200 import quantum_dynamics as qd

        print(json.dumps(config_table(qd)), flush=True)
        return

    if args.nd_case:
        from zinq_b200 import quantum_dynamics as qd

        case, prec, steps = args.nd_case[0], args.nd_case[1], int(args.nd_case[2])
        def c3pop(nstate=3):  # the 512^2 grid recording populations only (the serving stream's largest jobs)
            o = coupled_harmonic_2d(iters=steps)
            o["write"] = {"population": "P"}
            m = o["potential"]["custom"]["matrix"]
            o["potential"]["custom"]["matrix"] = [row[:nstate] for row in m[:nstate]]
            return o

        opt = {"c3": lambda: coupled_harmonic_2d(iters=steps), "c3pop": c3pop, "c3pop1": lambda: c3pop(1),
               "c3pop2": lambda: c3pop(2), "c4": lambda: anharmonic_3d(steps, False),
               "c4itp": lambda: anharmonic_3d(steps, True), "wide": lambda: wide_grid_2d(steps)}[case]()
        job = qd.Job(opt, prec)
        for _ in range(2):
            ms = job.run()
        print(json.dumps({"nd_case": case, "precision": prec, "ms": ms, "us_per_step": 1e3 * ms / steps}))
        return

    if args.profile_case:
        from zinq_b200 import quantum_dynamics as qd

        b = qd.Batch(workload(200)[2:3], args.profile_case)
        for _ in range(2):
            ms = b.run()
        print(json.dumps({"profile_case": args.profile_case, "ms": ms, "launches": b.launches}))
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        reference_arm(args, rank)
        return

    import datetime

    import numpy as np
    import torch

    from zinq_b200 import _abi
    from zinq_b200 import quantum_dynamics as qd

    torch.cuda.set_device(local)
    _abi.check(_abi.load().zqd_set_device(local))
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    opts = workload()
    U = units(opts)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed(batch, steps, warm):
        for _ in range(warm):
            batch.run()
        barrier()
        times = []
        for _ in range(steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            times.append(batch.run())
        barrier()
        return times

    # the launch shapes of the workload's key, measured by the library's autotuner (outside the timed region)
    tuned = {p: qd.autotune(1, NPOINT, NSTATE, p) for p in ("fp32", "fp64")}
    fp64 = qd.Batch(opts, "fp64")
    fp32 = qd.Batch(opts, "fp32")
    import tempfile

    clk = Clocks(local, args.clocks_csv or os.path.join(tempfile.gettempdir(), f"zqd_bench_clocks_rank{rank}.csv"))
    t32 = timed(fp32, args.steps, args.warmup)
    t64 = timed(fp64, args.steps, args.warmup)
    clocks = clk.stop()
    launches32 = fp32.launches * args.steps
    launches64 = fp64.launches * args.steps

    # accuracy of the FP32 form against the FP64 form (itself parity-tested against the oracle)
    pop_err = 0.0
    for i in range(len(opts)):
        a = fp32.result(i).observables[0].history["population"]
        b = fp64.result(i).observables[0].history["population"]
        pop_err = max(pop_err, float(np.max(np.abs(a - b))))

    # end to end through the public API, host options -> host results
    def e2e(prec):
        for _ in range(args.warmup):
            qd.run_batch_e2e(opts, prec)
        barrier()
        ts, hb, db = [], 0, 0
        for _ in range(args.steps):
            t0 = time.perf_counter()
            _, hb, db = qd.run_batch_e2e(opts, prec)
            ts.append(time.perf_counter() - t0)
        barrier()
        return ts, hb, db

    e2e_times, h2d, d2h = e2e("fp32")
    e2e64_times, h2d64, d2h64 = e2e("fp64")

    def maxall(x):
        return max_over_ranks(x, dist, "cuda")

    s32 = maxall(sum(t32) / 1e3)
    s64 = maxall(sum(t64) / 1e3)
    se2e = maxall(sum(e2e_times))
    se2e64 = maxall(sum(e2e64_times))
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return

    value = replica_value(U, world, args.steps, s32)
    v64 = replica_value(U, world, args.steps, s64)
    peak, peak_kind = measured_peak()
    per_launch = statistics.mean(t32) / 1e3  # one grouped launch runs the whole batch
    achieved = BYTES_PER_UNIT["fp32"] * U / per_launch / 1e9
    traffic = read_traffic("line_solve_kernel", "fp32")
    lat = sorted(t32)

    def shape_of(p):
        e = tuned[p]
        if e["cluster_ctas"]:
            return e["cluster_ctas"], e["radix_log2"]
        return 16, 2  # the built-in rules for 8192 points: 16 CTAs of 512 points, radix 4
    C32, lr32 = shape_of("fp32")
    onchip = onchip_roofline(_abi.load(), 1e6 * per_launch / ITERS, NPOINT, NSTATE, C32, lr32, 8, C32 * len(opts))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * s32 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config({"precision": "FP32 state/butterflies/phases, FP64 tables split hi+lo, FP64 reductions",
                          "parallelism": f"replicas x{world}"}),
        "fp64": {"value": v64, "unit": UNIT, "ms_per_step": 1e3 * s64 / args.steps, "dtype": "f64",
                 "gpu_launches": launches64},
        "fp32_over_fp64": value / v64,
        "pop_err_fp32_vs_fp64": pop_err, "pop_err_ok": pop_err <= 1e-5,
        "latency_ms": {"p50": statistics.median(lat), "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                       "note": "per job; the 5 jobs of a step complete together in one launch"},
        "e2e": {"value": world * U * args.steps / se2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "e2e_fp64": {"value": world * U * args.steps / se2e64, "unit": UNIT, "h2d_bytes_per_step": int(h2d64),
                     "d2h_bytes_per_step": int(d2h64)},
        "gpu_launches": launches32,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of line_solve_kernel on "
                                       "this workload, tabulated in profiles/traffic.txt by bench.py --traffic-table "
                                       "(an earlier capture, not this run)",
                     "note": "algorithmic bytes per grid-pt*state*step (psi r+w once, R read twice).  Not the "
                             "binding roof: the resident kernel keeps psi in shared memory for the whole solve "
                             "(DRAM sees the tables once per job); see roofline_onchip"},
        "clocks": clocks,
        "roofline_onchip": onchip,
        "autotune": {p: {k: tuned[p][k] for k in ("cluster_ctas", "radix_log2", "us_per_step", "default_us_per_step",
                                                  "candidates")} for p in tuned},
    }
    if not args.no_nd:
        line["nd"] = nd_legs(qd, torch, flush)
    if not args.no_extra:
        line["fp32_errors"] = fp32_error_table(qd)
        line["fft_brackets"] = fft_brackets(qd, torch)
    if not args.no_serve:
        line["serving"] = serving_leg(qd)
    if not args.no_cpu:
        sample = workload(ITERS)[2:4]
        dt, _ = oracle_sample(sample, 1)
        line["cpu_baseline"] = {"value": units(sample) / dt, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"2 of the 5 jobs (p0 = 20, 25) x {ITERS} steps, single thread"}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
