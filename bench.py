#!/usr/bin/env python
"""Benchmark of the path-integral Monte Carlo hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--form compensated|plain|fp64]

Workload (the precision form): N = 256 segments, arclength S = 20, source (0,0,0) with
tangent (0,0,1), receiver (0,0,12) with tangent (0,0,1); Gaussian phase sigma = 0.1
(config eps = sigma^2 = 0.01), mu_s = 10, regulariser mu = 1, no absorption, 8192-bin
table from a 20000-step Simpson rule; 2^26 weighted paths per step, sub-chains of
k ~ U{2..32} segments rotated by U(-0.05, 0.05) rad, Philox seed 1234, 256 unweighted
burn-in steps per chain. Inputs are synthetic (there is no dataset). One step = one full
Monte Carlo pass: every chain replays its proposals from the same initial curve.

Metric: path-segments weighted per second = weighted paths x N / time.
  value  device time of the pass (chain kernel + FP64 reduction), CUDA events on the
         launching stream, L2 flushed between steps, max over ranks;
  e2e    the same metric through the C ABI with host buffers, one experiment per step as the
         reference's callers run one: the experiment's parameters set on the caller's context
         (the table is built again), twisty_run (table built on the device, normaliser, initial
         curve, host-to-device copies, the pass, the result copied back).
The JSON line also carries the FP64 error of the estimate, the plain FP32 drop-in's
throughput on the same workload, the roofline of the chain kernel, and a CPU baseline
(the reference's own chain loop, compiled from its sources, on this host's cores).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W = dict(N=256, S=20.0, start=(0.0, 0.0, 0.0), sdir=(0.0, 0.0, 1.0), end=(0.0, 0.0, 12.0), edir=(0.0, 0.0, 1.0),
         sigma=0.1, eps=0.01, scatter=10.0, mu=1.0, absorption=0.0, num_steps_int=20000, bins=8192,
         paths=2 ** 26, k_max=32, max_angle=0.05, seed=1234, burn_in=256)
WORKLOAD_NAME = ("precision form: N=256 S=20 x1=(0,0,12) tangents (0,0,1), sigma=0.1 mu_s=10, 8192-bin table, "
                 "2^26 paths/step, k~U{2..32}, angle~U(-0.05,0.05), Philox seed 1234")
METRIC = "path-segments weighted/s, 1 B200, chosen vs plain form at <=1e-4 rel err vs FP64"
UNIT = "path-segments/s"
# Algorithmic FP32 instruction count of one path-segment of the full recompute: tangent 9,
# curvature 7, bin index 10, blend+absorption 4, log10 scale + compensated add 5, rotation ~3,
# RNG/sincos ~2 (one path-segment = one weighted path x one segment).
INSTR_PER_SEGMENT = 40.0
SMS = 148
LANES_PER_SM = 128


_FP32_PEAK = {}


def fp32_roof(T, device):
    """The FP32 roof in T lane-instructions/s: the device's FMA issue rate measured by the library
    (twisty_measure_fp32_peak, ~100 ms, once per process), and the nominal 148 SMs x 128 lanes x the
    max SM clock of MEASURED_PEAKS.json beside it. MEASURED_PEAKS.json has no FP32 figure."""
    if device not in _FP32_PEAK:
        sm_max = load_peaks().get("sm_max_mhz", 1965.0)
        nominal = SMS * LANES_PER_SM * sm_max * 1e6 / 1e12
        try:
            measured = T.measure_fp32_peak(device) / 1e12
        except Exception:   # reported as unmeasured, never silently replaced by the nominal figure
            measured = None
        _FP32_PEAK[device] = (measured, nominal, sm_max)
    return _FP32_PEAK[device]


def roofline_fields(T, device, achieved_ti):
    measured, nominal, sm_max = fp32_roof(T, device)
    peak = measured if measured else nominal
    return {"achieved": achieved_ti, "peak": peak, "unit": "Tinstr/s", "frac": achieved_ti / peak,
            "peak_kind": ("measured: FMA issue rate of this B200 (twisty_measure_fp32_peak)" if measured else
                          "nominal (the FMA-rate measurement failed)"),
            "peak_nominal": nominal, "frac_of_nominal": achieved_ti / nominal,
            "peak_nominal_basis": f"{SMS} SMs x {LANES_PER_SM} lanes x {sm_max:g} MHz (max SM clock of MEASURED_PEAKS.json)"}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.th = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# Batching workload: 4096 experiments, N log-uniform in [16, 1024], receivers uniform on spheres
# of radius U(2, 10) around the source at the origin (source tangent (0,0,1)), receiver tangents
# uniform on the sphere, S = r U(1.05, 2.0) (redrawn while S is below the minimum arclength),
# sigma ~ U(0.05, 0.3) (eps = sigma^2), mu_s ~ U(5, 50), a 4096-bin table per experiment, 2^16
# paths each; generator seed 1234.
BATCH = dict(n=4096, paths=1 << 16, bins=4096, num_steps_int=2000, mu=1.0, k_max=32, max_angle=0.05,
             burn_in=64, seed=1234)
BATCH_NAME = ("batching: 4096 experiments, N log-uniform [16,1024], receivers on spheres r~U(2,10), S=r*U(1.05,2), "
              "sigma~U(0.05,0.3), mu_s~U(5,50), 4096-bin table each, 2^16 paths each, k~U{2..32}, "
              "angle~U(-0.05,0.05), Philox seed 1234")
# DRAM bytes of one comp_chain_kernel launch (ncu dram__bytes_read.sum + dram__bytes_write.sum
# on the precision workload at 2^20 paths, 16x16 shape; the traffic is per chain, not per path: the table
# and initial curve are read once per CTA and one record is written per chain, so a launch of
# the full workload, with the same chains, moves the same bytes)
TRAFFIC_PER_LAUNCH = 106496
# the incremental variant's full-recompute period (weighted steps)
INCR_RESYNC = 32
# N of the small-N figures reported beside the headline (same geometry and table, 2^32 / N paths)
SMALL_N = (12, 16, 24, 32, 48, 64)
# paths of the export and re-weighing figures (N = 256: 50 MB of positions)
REWEIGH_PATHS = 1 << 14
# (N, paths) of the M-segment estimator figures (the bootstrapper resolves N - 2 in {64, 256})
MSEGMENT = ((66, 1 << 24), (258, 1 << 22))


def batch_experiments(T, n=None, seed=None):
    n = BATCH["n"] if n is None else n
    rng = np.random.default_rng(BATCH["seed"] if seed is None else seed)
    out = []
    while len(out) < n:
        N = int(round(math.exp(rng.uniform(math.log(16), math.log(1024)))))
        r = rng.uniform(2.0, 10.0)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        t = rng.normal(size=3)
        t /= np.linalg.norm(t)
        S = r * rng.uniform(1.05, 2.0)
        sigma = rng.uniform(0.05, 0.3)
        mus = rng.uniform(5.0, 50.0)
        bc = T.make_bc((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), r * d, t, S)
        if T.min_arclength(bc, N) >= S:
            continue
        out.append(T.make_experiment(bc, N, mus, sigma * sigma, BATCH["paths"]))
    return out


# Image workload: 64 x 64 receivers on the plane z = 10, x, y in [-4, 4], tangent (0, 0, 1),
# source at the origin with tangent (0, 0, 1), N = 512, S = 1.3 x distance, sigma = 0.15,
# mu_s = 20, 2^22 paths per pixel; the pixels share sigma and mu_s, so their tables come from
# one multi-arclength set of 256 tables over the pixels' ds range.
IMAGE = dict(nx=64, ny=64, half=4.0, z=10.0, N=512, sigma=0.15, scatter=20.0, paths=1 << 22, bins=4096,
             num_steps_int=2000, n_ds=256, k_max=32, max_angle=0.05, burn_in=64, seed=1234)
IMAGE_NAME = ("image: 64x64 receivers on z=10, x,y in [-4,4], tangent (0,0,1), N=512, S=1.3*distance, "
              "sigma=0.15, mu_s=20, 2^22 paths per pixel, 256-table multi-arclength set, k~U{2..32}, "
              "angle~U(-0.05,0.05), Philox seed 1234")


def batch_params(T, device=0):
    return T.default_params(num_segments=16, mu=BATCH["mu"], eps=0.01, scatter=10.0, absorption=0.0,
                            num_steps_int=BATCH["num_steps_int"], num_curvature_steps=BATCH["bins"],
                            paths_to_skip=BATCH["burn_in"], perturb_seed=BATCH["seed"], bootstrap_seed=7,
                            max_sub_chain=BATCH["k_max"], max_angle=BATCH["max_angle"], form=T.FORM_COMPENSATED,
                            lut_mode=T.LUT_FP64, device=device)


def workload_params(T, form, num_chains=0, chain_offset=0, device=0):
    return T.default_params(num_segments=W["N"], mu=W["mu"], eps=W["eps"], scatter=W["scatter"],
                            absorption=W["absorption"], num_steps_int=W["num_steps_int"],
                            num_curvature_steps=W["bins"], paths_to_generate=W["paths"], paths_to_skip=W["burn_in"],
                            perturb_seed=W["seed"], bootstrap_seed=7, max_sub_chain=W["k_max"],
                            max_angle=W["max_angle"], form=form, lut_mode=T.LUT_FP64, num_chains=num_chains,
                            chain_offset=chain_offset, device=device)


def workload_bc(T):
    return T.make_bc(W["start"], W["sdir"], W["end"], W["edir"], W["S"])


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def time_passes(T, torch, ctx, steps, warmup, device):
    """Device time of `steps` passes, each bracketed by events on one stream, L2 flushed between."""
    stream = torch.cuda.Stream(device=device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            ctx.launch(stream.cuda_stream)
        torch.cuda.synchronize(device)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        for i in range(steps):
            flush.zero_()
            starts[i].record(stream)
            ctx.launch(stream.cuda_stream)
            ends[i].record(stream)
        torch.cuda.synchronize(device)
    ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    return ms


# The workload's initial curve (N = 256 between the fixed points: the reference's bootstrapper
# resolves only N - 2 in {4, 6, 8, 12, 16, 24, ...}, so this is the arc bootstrapper's curve for
# bootstrap seed 7), committed so that the reference arm reads it without loading this library.
BENCH_CURVE = os.path.join(ROOT, "tests", "golden", "bench_curve_256.npy")


def cpu_reference_run(paths, threads, timeout=600):
    """The reference's own chain loop (GeometryRandom, compiled from its sources into
    oracle/_ref) on this host: returns (path-segments/s, perturb ms, record)."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        return None
    cfg = {"experiment": {
        "basicExperiment": {"startPos": list(W["start"]), "startDir": list(W["sdir"]), "endPos": list(W["end"]),
                            "endDir": list(W["edir"]), "arclength": W["S"]},
        "experimentParams": {"pathsToGenerate": paths, "pathsToSkip": W["burn_in"], "numSegments": W["N"],
                             "name": "bench", "experimentDir": tempfile.gettempdir(), "maxPerturbThreads": threads,
                             "maxWeightThreads": 0, "outputBigFloatWeights": False, "outputPathBatches": False,
                             "perturbMethod": 0, "random": {"bootstrapSeed": 7, "perturbSeed": W["seed"]},
                             "useGpu": False,
                             "weighting": {"weightFunction": 0, "mu": W["mu"], "eps": W["eps"],
                                           "numStepsInt": W["num_steps_int"], "numCurvatureSteps": W["bins"],
                                           "absorption": W["absorption"], "scatter": W["scatter"]}}}}
    with tempfile.TemporaryDirectory() as tmp:
        cf = os.path.join(tmp, "cfg.json")
        with open(cf, "w") as f:
            json.dump(cfg, f)
        np.load(BENCH_CURVE).astype(np.float32).tofile(cf + ".curve")
        r = subprocess.run([harness, "chain", cf, cf + ".curve", str(threads), str(paths), cf + ".out"],
                           capture_output=True, text=True, timeout=timeout, env={**os.environ, "TMPDIR": tmp})
        if r.returncode != 0:
            raise RuntimeError(r.stderr[-2000:])
        rec = json.load(open(cf + ".out"))
    return rec["paths"] * W["N"] / (rec["perturb_ms"] / 1e3), rec["perturb_ms"], rec


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference_arm(args):
    ws, rank, _ = dist_info()
    if rank != 0:
        return 0
    threads = cpu_threads()
    paths = threads * 1_000_000   # one 1e6-path CombinedWeightValues chunk per thread
    for _ in range(args.warmup):
        cpu_reference_run(paths // 4, threads)
    vals = []
    for _ in range(args.steps):
        v, ms, rec = cpu_reference_run(paths, threads)
        vals.append((v, ms))
    value = statistics.median(v for v, _ in vals)
    ms = statistics.median(m for _, m in vals)
    sample = (f"{paths} paths x N=256 per step on {threads} threads (one 1e6-path chunk per thread); the reference "
              f"loop's own proposals: k~U{{2..25}}, angle~U(-pi,pi)")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD_NAME, "paths_per_step": paths, "segments": W["N"], "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_image_workload(args, T, torch, device, ws, rank, pg):
    """The image workload through the receiver-grid driver and twisty_run_batch, tables from a
    multi-arclength set (twisty_multi_ds_tables)."""
    from twisty_b200 import drivers
    I = IMAGE
    paths = args.paths or I["paths"]
    eps = float(np.float32(I["sigma"]) * np.float32(I["sigma"]))
    exps = drivers.image_plane_experiments(I["nx"], I["ny"], I["half"], I["z"], I["N"], I["scatter"], eps, paths)
    ds = [e.bc.arclength / I["N"] for e in exps]
    params = T.default_params(num_segments=I["N"], mu=1.0, eps=eps, scatter=I["scatter"], absorption=0.0,
                              num_steps_int=I["num_steps_int"], num_curvature_steps=I["bins"],
                              paths_to_skip=I["burn_in"], perturb_seed=I["seed"], bootstrap_seed=7,
                              max_sub_chain=I["k_max"], max_angle=I["max_angle"], form=T.FORM_COMPENSATED,
                              lut_mode=T.LUT_MULTI_DS, device=device, chain_offset=rank * 1_000_000)
    ctx = T.Context(params)
    t0 = time.perf_counter()
    ctx.multi_ds_tables(min(ds), max(ds), I["n_ds"])
    tables_ms = (time.perf_counter() - t0) * 1e3
    ctx.run_batch(exps, iterations=max(1, args.warmup))
    with ClockSampler(device) as clk:
        res = ctx.run_batch(exps, iterations=args.steps)
    launches = ctx.kernels_per_launch()
    per_step = res[0].perturb_ms
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    ctx.run_batch(exps, iterations=1)
    e2e_ms = (time.perf_counter() - t0) * 1e3
    adjoint = None
    if not args.no_adjoint:
        # gradients of the image's total log-energy with respect to sigma and mu_s: one forward
        # pass and one batched adjoint replay of every pixel's chains (twisty_adjoint_batch)
        t0 = time.perf_counter()
        _, grad, total, tms = ctx.adjoint_batch(exps)
        adj_ms = (time.perf_counter() - t0) * 1e3
        adjoint = {"call_ms": adj_ms, "derivative_tables_ms": float(tms[0]), "replay_ms": float(tms[1]),
                   "log10_total_energy": float(total[0]), "d_log10_total_d_mu_s": float(total[1]),
                   "d_log10_total_d_sigma": float(total[2]),
                   "replay_path_segments_per_s": sum(r.total_paths * I["N"] for r in res) / (float(tms[1]) / 1e3),
                   "note": "call = forward pass + derivative tables + adjoint replay; replay recomputes every "
                           "curvature (exact blend) and stores nothing per step"}
    if pg:
        t = torch.tensor([per_step, e2e_ms], dtype=torch.float64, device=f"cuda:{device}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        per_step, e2e_ms = t.tolist()
    ctx.close()
    done = sum(r.total_paths * I["N"] for r in res)
    value = done * ws / (per_step / 1e3)
    achieved_ti = INSTR_PER_SEGMENT * done / (per_step / 1e3) / 1e12
    if rank == 0:
        import ctypes
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 (f64 cross-chain)", "data": "synthetic",
                "config": {"workload": IMAGE_NAME, "form": "compensated", "experiments": len(exps),
                           "paths_per_pixel": paths, "path_segments_per_step": done, "multi_ds_tables_ms": tables_ms,
                           "l2": "inputs larger than L2 per step (4096 chains' state per pixel batch, 256 tables)",
                           "parallelism": f"independent chains x{ws}"},
                "e2e": {"value": done * ws / (e2e_ms / 1e3), "unit": UNIT, "ms_per_step": e2e_ms,
                        "h2d_bytes_per_step": ctypes.sizeof(T._abi.Experiment) * len(exps),
                        "d2h_bytes_per_step": ctypes.sizeof(T._abi.Result) * len(exps)},
                "roofline": {"bound": "fp32", "kernel": "batch_kernel", **roofline_fields(T, device, achieved_ti),
                             "traffic": None, "basis": f"{INSTR_PER_SEGMENT:g} FP32 instructions per path-segment"},
                "cpu_baseline": None, "clocks": clk.summary(), "gpu_launches": launches * args.steps}
        if adjoint:
            line["adjoint"] = adjoint
        print(json.dumps(line))
    if pg:
        pg.destroy_process_group()
    return 0


def measure_batch(T, device, steps, warmup, exps=None, first=0, chain_offset=0):
    """The batching workload through twisty_run_batch on one device: device time per replay of
    the captured pass, end-to-end time per whole call (host experiments in, results out), and
    the results. `first` numbers the experiments from that index of the full batch (their
    Philox streams and bootstrap seeds), so that a rank's sub-batch gives the full batch's
    results."""
    if exps is None:
        exps = batch_experiments(T)
    params = batch_params(T, device=device)
    params.experiment_id += first
    params.bootstrap_seed += first
    params.chain_offset = chain_offset
    ctx = T.Context(params)
    ctx.run_batch(exps, iterations=max(1, warmup))
    with ClockSampler(device) as clk:
        res = ctx.run_batch(exps, iterations=steps)
    launches = ctx.kernels_per_launch()
    per_step = res[0].perturb_ms if res else 0.0
    setup_ms = res[0].setup_ms if res else 0.0
    # end to end: `steps` whole calls (host inputs in, results out), averaged
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.run_batch(exps, iterations=1)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / steps
    ctx.close()
    done = sum(r.total_paths * x.num_segments for r, x in zip(res, exps))
    return dict(res=res, exps=exps, per_step=per_step, setup_ms=setup_ms, e2e_ms=e2e_ms, done=done,
                launches=launches, clocks=clk.summary())


def batch_roofline(T, device, done, per_step):
    achieved_ti = INSTR_PER_SEGMENT * done / (per_step / 1e3) / 1e12
    return {"bound": "fp32", "kernel": "batch_kernel", **roofline_fields(T, device, achieved_ti), "traffic": None,
            "basis": f"{INSTR_PER_SEGMENT:g} FP32 instructions per path-segment"}


def run_batch_workload(args, T, torch, device, ws, rank, pg):
    """The batching workload through twisty_run_batch. Over several ranks the experiments are
    split by experiment (a contiguous range per rank with its share of the work, the full
    batch's stream ids) and every experiment's result is gathered on every rank."""
    from twisty_b200 import dist as D
    allx = batch_experiments(T)
    idx = D.partition_experiments(allx, rank, ws) if ws > 1 else list(range(len(allx)))
    mine = [allx[i] for i in idx]
    if pg:
        pg.barrier()
    m = measure_batch(T, device, args.steps, args.warmup, exps=mine, first=idx[0] if idx else 0)
    per_step, e2e_ms = m["per_step"], m["e2e_ms"]
    combined = None
    if pg:
        t = torch.tensor([per_step, e2e_ms], dtype=torch.float64, device=f"cuda:{device}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        per_step, e2e_ms = t.tolist()
        full = D.gather_partitioned(m["res"], idx, len(allx), device=f"cuda:{device}")
        combined = {"experiments": len(full), "total_paths": sum(r["total_paths"] for r in full),
                    "failed_paths": sum(r["failed_paths"] for r in full)}
        dn = torch.tensor([float(m["done"])], dtype=torch.float64, device=f"cuda:{device}")
        pg.all_reduce(dn)
        done_all = dn.item()
    else:
        done_all = m["done"]
    value = done_all / (per_step / 1e3)
    if rank == 0:
        import ctypes
        h2d = ctypes.sizeof(T._abi.Experiment) * len(allx)   # the experiment array; tables are built on the device
        d2h = ctypes.sizeof(T._abi.Result) * len(allx)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": per_step, "higher_is_better": True,
                "scaling": "strong" if ws > 1 else "weak",
                "vs_baseline": None, "dtype": "f32 (f64 cross-chain)", "data": "synthetic",
                "config": {"workload": BATCH_NAME, "form": "compensated", "experiments": len(allx),
                           "path_segments_per_step": sum(x.paths * x.num_segments for x in allx),
                           "l2": "inputs larger than L2 (4096 tables of 4096 bins, 134 MB fixed-point + 134 MB linear)",
                           "parallelism": f"experiments split over {ws} ranks" if ws > 1 else "one GPU"},
                "e2e": {"value": done_all / (e2e_ms / 1e3), "unit": UNIT, "ms_per_step": e2e_ms,
                        "setup_ms": m["setup_ms"], "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "roofline": batch_roofline(T, device, m["done"], m["per_step"]),
                "cpu_baseline": None, "clocks": m["clocks"], "gpu_launches": m["launches"] * args.steps}
        if combined:
            line["combined"] = combined
        print(json.dumps(line))
    if pg:
        pg.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--form", default="compensated", choices=["compensated", "plain", "fp64"])
    ap.add_argument("--no-error", action="store_true", help="skip the FP64 error measurement")
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain FP32 drop-in")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-batch", action="store_true", help="skip timing the batching workload")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint (precision line: the differentiation form; image workload: its batched adjoint)")
    ap.add_argument("--no-small-n", action="store_true", help="skip the small-N figures")
    ap.add_argument("--no-reweigh", action="store_true", help="skip the export and re-weighing figures")
    ap.add_argument("--no-msegment", action="store_true", help="skip the M-segment estimator figures")
    ap.add_argument("--paths", type=int, default=0, help="paths per pass (default 2^26; smaller for profiling)")
    ap.add_argument("--workload", default="precision", choices=["precision", "batch", "image"],
                    help="precision: one N=256 experiment (the headline); batch: 4096 uneven experiments; "
                         "image: 64x64 receiver grid at N=512 from a multi-arclength table set")
    ap.add_argument("--experiments", type=int, default=0, help="batch workload: number of experiments (default 4096)")
    ap.add_argument("--image-pixels", type=int, default=0,
                    help="image workload: pixels per side (default 64; smaller grids for profiling)")
    ap.add_argument("--segments", type=int, default=0,
                    help="precision workload with N segments instead of 256 (per-N figures and profiles; the CPU "
                         "baseline and the reference arm keep N = 256)")
    args = ap.parse_args()
    if args.experiments:
        BATCH["n"] = args.experiments
    if args.image_pixels:
        global IMAGE_NAME
        IMAGE["nx"] = IMAGE["ny"] = args.image_pixels
        IMAGE_NAME = IMAGE_NAME.replace("64x64", f"{args.image_pixels}x{args.image_pixels}")
    if args.paths and args.workload == "precision":
        W["paths"] = args.paths
    if args.segments and args.impl == "b200":
        global WORKLOAD_NAME
        W["N"] = args.segments
        WORKLOAD_NAME = WORKLOAD_NAME.replace("N=256", f"N={args.segments}")
        args.no_cpu = True
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import twisty_b200 as T

    ws, rank, local = dist_info()
    device = local
    torch.cuda.set_device(device)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device(f"cuda:{device}"))
        pg = dist
    if args.workload == "batch":
        return run_batch_workload(args, T, torch, device, ws, rank, pg)
    if args.workload == "image":
        return run_image_workload(args, T, torch, device, ws, rank, pg)
    form = {"compensated": T.FORM_COMPENSATED, "plain": T.FORM_PLAIN_FP32, "fp64": T.FORM_FP64}[args.form]
    bc = workload_bc(T)

    # one chain layout for every rank (the form's default), disjoint chain ids per rank
    with T.Context(workload_params(T, form, device=device)) as probe:
        probe.prepare(bc)
        probe.launch()
        chains = probe.collect().num_chains

    ctx = T.Context(workload_params(T, form, num_chains=chains, chain_offset=rank * chains, device=device))
    ctx.prepare(bc)
    with ClockSampler(device) as clk:
        ms = time_passes(T, torch, ctx, args.steps, args.warmup, device)
    res = ctx.collect()
    kernel_ms = res.perturb_ms
    per_step = sum(ms) / len(ms)
    if pg:
        t = torch.tensor([per_step, kernel_ms], dtype=torch.float64, device=f"cuda:{device}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        per_step, kernel_ms = t.tolist()
    segs = res.total_paths * W["N"]
    value = segs * ws / (per_step / 1e3)

    # End to end through the C ABI with host buffers, one experiment per step as a caller of the
    # reference runs one (Experiments/FullExperiment.cpp:204-230): the context is the caller's
    # runner, kept across experiments; every step sets the experiment's parameters
    # (twisty_update_params, after which the table is built again, as RunExperiment builds its
    # table on every call, FullExperimentRunnerOptimalPerturb.cpp:59-69) and runs it
    # (twisty_run: the table on the device, the initial curve, the uploads, the pass, the result
    # read back).
    e2e_params = workload_params(T, form, num_chains=chains, chain_offset=rank * chains, device=device)
    e2e_ctx = T.Context(e2e_params)
    e2e_ctx.run(bc)   # module load and the context's first allocations, outside the timed region
    reps = max(1, min(args.steps, 5))
    if pg:
        pg.barrier()
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for _ in range(reps):
        e2e_ctx.set_params(e2e_params)
        er = e2e_ctx.run(bc)
    torch.cuda.synchronize(device)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / reps
    e2e_ctx.close()
    if pg:
        t = torch.tensor([e2e_ms], dtype=torch.float64, device=f"cuda:{device}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = t.item()
    N = W["N"]
    # bytes each twisty_run moves: up, the fixed-point and linear tables (float2 per bin each),
    # the initial curve and its segment vectors; down, the table range (3 doubles), the float
    # table, the reduced result (ReduceOut, 48 bytes)
    h2d = 8 * W["bins"] + 8 * W["bins"] + 4 * 3 * (N + 1) + 4 * 3 * N
    d2h = 24 + 4 * W["bins"] + 48

    extra = {}
    if rank == 0 and not args.no_error and form != T.FORM_FP64:
        with T.Context(workload_params(T, T.FORM_FP64, num_chains=chains, device=device)) as c64:
            r64 = c64.run(bc)
        extra["error_vs_fp64"] = {"rel": abs(10 ** (res.log10_weight - r64.log10_weight) - 1),
                                  "log10_weight": res.log10_weight, "log10_weight_fp64": r64.log10_weight,
                                  "fp64_ms": r64.perturb_ms, "rel_std_error": res.rel_std_error}
    if rank == 0 and not args.no_plain and form == T.FORM_COMPENSATED:
        with T.Context(workload_params(T, T.FORM_PLAIN_FP32, device=device)) as cp:
            cp.prepare(bc)
            pms = time_passes(T, torch, cp, max(1, min(args.steps, 3)), 1, device)
            rp = cp.collect()
            plain_v = rp.total_paths * N / (sum(pms) / len(pms) / 1e3)
            pe = None
            if not args.no_error:
                with T.Context(workload_params(T, T.FORM_FP64, num_chains=rp.num_chains, device=device)) as c64:
                    rp64 = c64.run(bc)
                pe = abs(10 ** (rp.log10_weight - rp64.log10_weight) - 1)
        extra["plain_fp32"] = {"value": plain_v, "ms_per_step": sum(pms) / len(pms), "chains": rp.num_chains,
                               "error_vs_fp64": pe, "speedup_of_chosen": value / ws / plain_v}

    if rank == 0 and form == T.FORM_COMPENSATED and not args.no_plain:
        # the O(k) incremental variant on the same workload and chains, reported on its own:
        # an algorithmic shortcut, not the recompute-everything definition the value measures
        ip = workload_params(T, form, num_chains=chains, device=device)
        ip.incremental_resync = INCR_RESYNC
        with T.Context(ip) as ci:
            ci.prepare(bc)
            ims = time_passes(T, torch, ci, max(1, min(args.steps, 5)), 1, device)
            ri = ci.collect()
        iv = ri.total_paths * W["N"] / (sum(ims) / len(ims) / 1e3)
        ie = None
        if "error_vs_fp64" in extra:
            ie = abs(10 ** (ri.log10_weight - extra["error_vs_fp64"]["log10_weight_fp64"]) - 1)
        extra["incremental"] = {"value": iv, "unit": UNIT, "ms_per_step": sum(ims) / len(ims),
                                "resync_every": INCR_RESYNC, "error_vs_fp64": ie, "speedup_over_value": iv / (value / ws),
                                "note": "weights updated from the two curvatures each rotation changes, full "
                                        "recompute every resync_every-th weighted step; not the headline"}

    if rank == 0 and form == T.FORM_COMPENSATED and not args.no_small_n and not args.segments:
        # the same geometry and table at small N, where per-step work that does not scale with N
        # bounds the kernel: 2^32 path-segments per pass (2^32 / N paths, so that the 256 burn-in
        # steps per chain stay a small share), events around each pass, L2 flushed between
        small = {}
        for n_small in SMALL_N:
            sp = workload_params(T, form, device=device)
            sp.num_segments = n_small
            sp.paths_to_generate = (1 << 32) // n_small
            with T.Context(sp) as cs:
                cs.prepare(bc)
                sms = time_passes(T, torch, cs, max(3, min(args.steps, 5)), 1, device)
                rs = cs.collect()
            small[str(n_small)] = {"value": rs.total_paths * n_small / (sum(sms) / len(sms) / 1e3),
                                   "ms_per_step": sum(sms) / len(sms), "chains": rs.num_chains,
                                   "shape": T.default_shape(n_small, W["bins"])}
        extra["small_n"] = {"unit": UNIT, "paths": "2^32 / N", "per_n": small,
                            "note": "the precision workload's geometry and 8192-bin table at N segments; up to "
                                    "N = 48 the kernels (all shapes but 4 x 4) turn the shorter side of each move"}

    if rank == 0 and form == T.FORM_COMPENSATED and not args.no_batch:
        # the batching form on its own workload (4096 uneven experiments), timed in this run
        bm = measure_batch(T, device, max(3, min(args.steps, 10)), 1)
        import ctypes
        extra["batching"] = {
            "workload": BATCH_NAME, "value": bm["done"] / (bm["per_step"] / 1e3), "unit": UNIT,
            "ms_per_step": bm["per_step"], "steps": max(3, min(args.steps, 10)),
            "e2e": {"value": bm["done"] / (bm["e2e_ms"] / 1e3), "unit": UNIT, "ms_per_step": bm["e2e_ms"],
                    "setup_ms": bm["setup_ms"],
                    "h2d_bytes_per_step": ctypes.sizeof(T._abi.Experiment) * len(bm["exps"]),
                    "d2h_bytes_per_step": ctypes.sizeof(T._abi.Result) * len(bm["exps"])},
            "roofline": batch_roofline(T, device, bm["done"], bm["per_step"]), "gpu_launches_per_step": bm["launches"],
            "failed_paths": sum(r.failed_paths for r in bm["res"]), "clocks": bm["clocks"]}

    if rank == 0 and form == T.FORM_COMPENSATED and not args.no_reweigh:
        # the export and re-weighing pipeline (the reference's path-batch output and its batch
        # re-weigher): the workload's first REWEIGH_PATHS weighted paths exported, then weighed
        # again through the C ABI by both weighers (host positions in, weights out, each call
        # uploading the positions), end to end on the host clock
        with T.Context(workload_params(T, form, device=device)) as cx:
            t0 = time.perf_counter()
            pos, w_exp, _ = cx.export_paths(bc, None, REWEIGH_PATHS)
            export_ms = (time.perf_counter() - t0) * 1e3
            cx.weight_paths(bc, pos[:64], T.FORM_COMPENSATED)   # tables and buffers, outside the timing
            rw = {}
            for name, f in (("compensated", T.FORM_COMPENSATED), ("plain_fp32", T.FORM_PLAIN_FP32)):
                ts = []
                for _ in range(3):
                    t0 = time.perf_counter()
                    wr, vr, _ = cx.weight_paths(bc, pos, f)
                    ts.append((time.perf_counter() - t0) * 1e3)
                ok = (vr == 1) & np.isfinite(w_exp)
                rel = np.abs(wr[ok] - w_exp[ok]) / np.abs(w_exp[ok])
                rw[name] = {"value": pos.shape[0] * W["N"] / (min(ts) / 1e3), "ms": min(ts),
                            "median_rel_diff_vs_export": float(np.median(rel)) if rel.size else None}
        extra["reweigh"] = {"unit": UNIT, "paths": int(pos.shape[0]), "export_ms": export_ms,
                            "h2d_bytes_per_call": int(pos.nbytes), "d2h_bytes_per_call": int(pos.shape[0] * 9),
                            **rw, "note": "twisty_export_paths of the workload's first weighted paths, then "
                                          "twisty_weight_paths on them (host clock, positions uploaded per call); "
                                          "the weights compared with the export's own"}

    if rank == 0 and form == T.FORM_COMPENSATED and not args.no_msegment:
        # the independent-sample M-segment estimator on the workload's geometry: every path a
        # fresh bootstrapped curve, weighed by the compensated weigher (device time of the pass)
        msr = {}
        for n_ms, p_ms in MSEGMENT:
            mp = workload_params(T, form, device=device)
            mp.num_segments = n_ms
            mp.paths_to_generate = p_ms
            with T.Context(mp) as cm:
                cm.run_msegment(bc)   # tables and buffers
                rm = cm.run_msegment(bc)
            msr[str(n_ms)] = {"paths": int(rm.total_paths), "failed_paths": int(rm.failed_paths), "ms": rm.perturb_ms,
                              "paths_per_s": rm.total_paths / (rm.perturb_ms / 1e3),
                              "value": rm.total_paths * n_ms / (rm.perturb_ms / 1e3),
                              "log10_weight": rm.log10_weight, "rel_std_error": rm.rel_std_error}
        extra["msegment"] = {"unit": UNIT, "per_n": msr,
                             "note": "twisty_run_msegment: paths generated by the recursive bootstrapper on the device "
                                     "and weighed in the compensated form; the estimate is the mean weight"}

    if rank == 0 and form == T.FORM_COMPENSATED and not args.no_adjoint:
        # the differentiation form at its own configuration (N = 128, S = 16, receiver (8,0,0)
        # along x, 4096-bin tables and derivative tables, 2^22 paths): forward pass, then the
        # adjoint replay of its chains (derivative tables built, curvatures recomputed)
        ap_ = T.default_params(num_segments=128, mu=1.0, eps=0.01, scatter=10.0, num_steps_int=4000,
                               num_curvature_steps=4096, form=T.FORM_COMPENSATED, lut_mode=T.LUT_FP64,
                               perturb_seed=31, num_chains=4096, paths_to_generate=1 << 22, paths_to_skip=2000,
                               max_sub_chain=32, max_angle=0.1, device=device)
        abc = T.make_bc((0, 0, 0), (1, 0, 0), (8, 0, 0), (1, 0, 0), 16.0)
        with T.Context(ap_) as ca:
            f0 = ca.run(abc)
            ca.adjoint(abc, f0)   # warm
            t0 = time.perf_counter()
            f1 = ca.run(abc)
            t1 = time.perf_counter()
            g = ca.adjoint(abc, f1)
            t2 = time.perf_counter()
        segs_a = f1.total_paths * 128
        extra["adjoint"] = {"workload": "differentiation form: N=128 S=16 x1=(8,0,0) tangents (1,0,0), sigma=0.1 "
                                        "mu_s=10, 4096-bin tables and derivative tables, 2^22 paths (4096 chains, "
                                        "2000 burn-in steps), k~U{2..32}, angle~U(-0.1,0.1)",
                            "forward_ms": (t1 - t0) * 1e3, "adjoint_ms": (t2 - t1) * 1e3,
                            "adjoint_path_segments_per_s": segs_a / (t2 - t1),
                            "gradient": {"d_mu_s": g[0], "d_sigma": g[1], "d_receiver": list(g[2:5])},
                            "note": "host wall time of twisty_run and of twisty_adjoint (derivative tables, replay, "
                                    "reduction); the replay runs the burn-in steps again"}

    combined = None
    if pg:
        # the one exchange step: every rank's (log10 sum, relative SE, counts) combined
        from twisty_b200 import dist as D
        combined = D.all_combine(res, device=f"cuda:{device}")

    clocks = clk.summary()
    achieved_ti = INSTR_PER_SEGMENT * segs / (kernel_ms / 1e3) / 1e12
    roofline = {"bound": "fp32", "kernel": "comp_chain_kernel" if form == T.FORM_COMPENSATED else args.form,
                **roofline_fields(T, device, achieved_ti),
                "traffic": TRAFFIC_PER_LAUNCH if form == T.FORM_COMPENSATED else None,
                "basis": f"{INSTR_PER_SEGMENT:g} FP32 instructions per path-segment; traffic = DRAM bytes per launch "
                         "from ncu (per chain, not per path)",
                "segments_per_s_kernel_only": segs / (kernel_ms / 1e3)}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        threads = cpu_threads()
        try:
            r = cpu_reference_run(threads * 1_000_000, threads)
            if r:
                cpu = {"value": r[0], "unit": UNIT, "cores": threads, "kind": "reference",
                       "sample": f"{threads * 1_000_000} paths x N=256, reference GeometryRandom loop on {threads} threads"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": threads, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 (f64 cross-chain)", "data": "synthetic",
                "config": {"workload": WORKLOAD_NAME, "form": args.form, "chains_per_gpu": chains,
                           "steps_per_chain": res.steps_per_chain, "paths_per_gpu": res.total_paths,
                           "l2": "flushed between steps (256 MB write)", "parallelism": f"independent chains x{ws}"},
                "e2e": {"value": segs * ws / (e2e_ms / 1e3), "unit": UNIT, "ms_per_step": e2e_ms,
                        "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "per_step": "twisty_update_params + twisty_run: table build, initial curve, uploads, pass, "
                                    "result read back",
                        "setup_ms": er.setup_ms},
                "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
                "gpu_launches": ctx.kernels_per_launch() * args.steps, **extra}
        if combined:
            line["combined"] = combined
        print(json.dumps(line))
    ctx.close()
    if pg:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
