"""Generate the golden fixtures under tests/golden/ from the reference itself.

    make -C oracle ref && python tests/golden/make_golden.py

Every expected value here comes out of the reference's own code, compiled from its
sources by oracle/Makefile (with the three patches it documents) and driven through
oracle/_ref/ref_harness:
  lut_*.npz        WeightLookupTableIntegral::Initialize tables and their metadata
  paths_*.npz      path batches and, per path, the reference weigher's log10 weight,
                   curvatures and left bin indices (UpdateTangentsFromPos,
                   UpdateCurvaturesFromTangents_RadiativeTransfer, WeightCurveViaCurvatureLog10_CudaSafe)
  rotate.npz       RotateVectorByQuaternion on random inputs
  cw.npz           CombinedWeightValues_C add / combine / extract sequences
  norm.json        log10 Norm(N, ds, bc) for N = 4, 5 and 6 (the N = 5, 6 records take the
                   reference's 1e10-term quadrature, about a minute each; `--only norm`)
  boot_*.npy       reference bootstrap curves (ResolveEvenNumberOfSegments)
  chain_*.json     full runs of the reference's Markov-chain loop (GeometryRandom) for the
                   statistical comparison, with per-1e6-path chunk sums
  msegment_*.json  the reference's independent-sample estimator (MSegmentPathGenerationMC's
                   per-path work through its own functions): mean weight and relative SE
                   (`--msegment-only` regenerates just these)
  lut_D/E, paths_D/E, boot_258, chain_D/E.json
                   the same fixtures at the configurations the benchmark metric is quoted on
                   (`--only baseline`): D is the plain-form configuration (N = 66, S = 10,
                   receiver (8,0,0) along x, 4096-bin table), E the precision-form one (N = 258,
                   S = 20, receiver (0,0,12) along z, 8192-bin table from a 20000-step rule);
                   N = 66 and 258 because the reference's bootstrapper resolves only N - 2 in
                   {4, 6, 8, 12, 16, 24, ...}. Their path batches include chain states under the
                   benchmark's own proposals (k <= 32, angles within +-0.1 and +-0.05) beside the
                   reference's (k <= 25, angles in (-pi, pi)).
The path batches are perturbed with the oracle's chain runner so they cover curved
configurations; their weights still come from the reference weigher. This script reads
the reference tree only through oracle/_ref, and is never run by the tests themselves.
"""
from __future__ import annotations

import json
import math
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import py_oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
H = O.REF_HARNESS
F32 = np.float32

# (name, mu, eps, scatter, absorption, numStepsInt, bins, N, S)
LUTS = [
    ("A", 1.0, 0.01, 10.0, 0.0, 2000, 1024, 66, 10.0),
    ("B", 1.0, 0.01, 10.0, 0.05, 2000, 2048, 34, 12.0),
    ("C", 0.3, 0.0025, 50.0, 0.0, 4000, 512, 18, 6.0),
]
# the benchmark configurations (plain form, precision form)
BASELINE_LUTS = [
    ("D", 1.0, 0.01, 10.0, 0.0, 4000, 4096, 66, 10.0),
    ("E", 1.0, 0.01, 10.0, 0.0, 20000, 8192, 258, 20.0),
]
# the benchmark's proposals per set: (k_max, max_angle)
BASELINE_PROPOSALS = {"D": (32, 0.1), "E": (32, 0.05)}
GEOM = {  # N -> (startPos, startDir, endPos, endDir)
    66: ((0, 0, 0), (1, 0, 0), (8, 0, 0), (1, 0, 0)),
    34: ((0, 0, 0), (0, 0, 1), (0, 0, 7), (0, 0, 1)),
    18: ((0, 0, 0), (1, 0, 0), (2.5, 1.0, 0.5), (0, 1, 0)),
    10: ((0, 0, 0), (1, 0, 0), (3, 0, 0), (1, 0, 0)),
    258: ((0, 0, 0), (0, 0, 1), (0, 0, 12), (0, 0, 1)),
}


def run(args, **kw):
    return subprocess.run([H, *map(str, args)], check=True, capture_output=True, text=True, **kw)


def bc12(n):
    g = GEOM[n]
    return [c for v in g for c in v]


def ref_lut(tmp, mu, eps, scatter, absorption, nsteps, bins, ds):
    f = os.path.join(tmp, "lut.bin")
    run(["lut", repr(mu), repr(eps), repr(scatter), repr(absorption), nsteps, bins, repr(float(ds)), f])
    b = open(f, "rb").read()
    hdr = np.frombuffer(b[:24], F32)
    n = struct.unpack("<I", b[24:28])[0]
    lut = np.frombuffer(b[28:28 + 4 * n], F32).copy()
    return f, hdr, lut


def ref_weigh(tmp, lutfile, N, S, absorption, pos):
    pf = os.path.join(tmp, "paths.bin")
    of = os.path.join(tmp, "wout.bin")
    with open(pf, "wb") as f:
        f.write(struct.pack("<Q", pos.shape[0]))
        f.write(np.ascontiguousarray(pos, F32).tobytes())
    run(["weigh", lutfile, N, repr(float(S)), repr(float(absorption)), pf, of])
    b = open(of, "rb").read()
    rec = 1 + 8 + 8 * (N - 1)
    P = pos.shape[0]
    valid = np.zeros(P, np.uint8)
    w = np.zeros(P)
    curv = np.zeros((P, N - 1), F32)
    bins = np.zeros((P, N - 1), np.int32)
    for p in range(P):
        x = b[p * rec:(p + 1) * rec]
        valid[p] = x[0]
        w[p] = struct.unpack("<d", x[1:9])[0]
        curv[p] = np.frombuffer(x[9:9 + 4 * (N - 1)], F32)
        bins[p] = np.frombuffer(x[9 + 4 * (N - 1):], np.int32)
    return w, valid, curv, bins


def ref_bootstrap(tmp, N, S, seed):
    f = os.path.join(tmp, "boot.bin")
    run(["bootstrap", N, repr(float(S)), *bc12(N), seed, f])
    return np.fromfile(f, F32).reshape(N + 1, 3)


def ref_msegment(tmp, N, S, seed, paths, threads, mu, eps, scatter, absorption, nsteps, bins):
    """The reference's M-segment estimator (harness mode msegment): mean weight and its
    relative standard error from the spread of the independent paths."""
    ds = F32(S) / F32(N)
    ref_lut(tmp, mu, eps, scatter, absorption, nsteps, bins, ds)
    out = os.path.join(tmp, "ms.bin")
    run(["msegment", os.path.join(tmp, "lut.bin"), N, repr(float(S)), *bc12(N), repr(absorption), seed, paths,
         threads, "-", out])
    b = np.fromfile(out, dtype=np.dtype([("v", "u1"), ("w", "<f8")]))
    w = b["w"][b["v"] == 1]
    m = float(w.max())
    x = 10.0 ** (w - m)
    mean = float(x.mean())
    return {"N": N, "S": S, "seed": seed, "paths": paths, "valid": int(w.size), "mu": mu, "eps": eps,
            "scatter": scatter, "absorption": absorption, "num_steps_int": nsteps, "bins": bins,
            "log10_mean": m + math.log10(mean), "rel_se": float(x.std(ddof=1) / math.sqrt(x.size) / mean)}


def make_config(N, S, paths, skip, seed, mu, eps, scatter, absorption, nsteps, bins, threads):
    g = GEOM[N]
    return {"experiment": {
        "basicExperiment": {"startPos": list(g[0]), "startDir": list(g[1]), "endPos": list(g[2]),
                            "endDir": list(g[3]), "arclength": S},
        "experimentParams": {"pathsToGenerate": paths, "pathsToSkip": skip, "numSegments": N, "name": "golden",
                             "experimentDir": "/tmp/twisty_golden", "maxPerturbThreads": threads,
                             "maxWeightThreads": 0, "outputBigFloatWeights": False, "outputPathBatches": False,
                             "perturbMethod": 0, "random": {"bootstrapSeed": 7, "perturbSeed": seed},
                             "useGpu": False,
                             "weighting": {"weightFunction": 0, "mu": mu, "eps": eps, "numStepsInt": nsteps,
                                           "numCurvatureSteps": bins, "absorption": absorption,
                                           "scatter": scatter}}}}


def make_msegment(tmp):
    for N, S in ((10, 5.0), (34, 12.0), (66, 10.0)):
        ms = ref_msegment(tmp, N, S, 12345, 1 << 22, os.cpu_count() or 1, 1.0, 0.01, 10.0, 0.0, 2000, 1024)
        with open(os.path.join(OUT, f"msegment_{N}.json"), "w") as f:
            json.dump(ms, f, indent=1)


def weighed_batch(tmp, name, mu, eps, scatter, absorption, nsteps, bins, N, S, init, proposals=None):
    """Reference table for the set, and a path batch weighed by the reference weigher: the
    initial curve, chain states after a few rotations of U(-pi, pi) (the reference's own
    proposals), after longer runs of the benchmark's proposals when given, and a straight path."""
    ds = F32(S) / F32(N)
    lf, hdr, lut = ref_lut(tmp, mu, eps, scatter, absorption, nsteps, bins, ds)
    np.savez(os.path.join(OUT, f"lut_{name}.npz"), lut=lut, hdr=hdr,
             params=np.array([mu, eps, scatter, absorption, nsteps, bins, N, S], np.float64))
    wp = O.wparams(mu, eps, scatter, absorption, nsteps, bins)
    olut, meta = O.lut_f32(wp, ds)
    pos = [init[None]]
    for seed, steps in ((11, 3), (12, 17), (13, 60)):
        r = O.run_chains(init, N, S, olut, meta, seed=seed, n_chains=20, steps=steps, want_final=True)
        pos.append(r["final_pos"])
    if proposals:
        k_max, angle = proposals
        for seed, steps in ((14, 200), (15, 2000)):
            r = O.run_chains(init, N, S, olut, meta, seed=seed, n_chains=20, steps=steps, want_final=True,
                             k_max=k_max, max_angle=angle)
            pos.append(r["final_pos"])
    st = np.zeros((1, N + 1, 3), F32)
    st[0, :, 0] = np.arange(N + 1, dtype=F32) * ds
    pos.append(st)
    pos = np.concatenate(pos).astype(F32)
    w, valid, curv, rbins = ref_weigh(tmp, lf, N, S, absorption, pos)
    np.savez(os.path.join(OUT, f"paths_{name}.npz"), pos=pos, log10w=w, valid=valid, curv=curv, bins=rbins)
    print(f"lut/paths {name}: {pos.shape[0]} paths, N={N}")


def reference_chain_run(tmp, key, N, S, paths, threads, mu, eps, scatter, absorption, nsteps, bins, curve, skip=1000,
                        repeats=1):
    """The reference's runner loop on `threads` chains (perturbSeed 4321 + thread); with repeats
    > 1, further runs on the next seeds (4321 + r * threads + thread), their 1e6-path chunks
    pooled into one record (the runner uses at most one chain per host core)."""
    recs = []
    for r in range(repeats):
        cfg = make_config(N, S, paths, skip, 4321 + r * threads, mu, eps, scatter, absorption, nsteps, bins, threads)
        cf = os.path.join(tmp, f"chain_{key}.json")
        json.dump(cfg, open(cf, "w"))
        np.asarray(curve, F32).tofile(cf + ".curve")
        run(["chain", cf, cf + ".curve", threads, paths, cf + ".out"])
        res = json.load(open(cf + ".out"))
        res["config"] = cfg
        recs.append(res)
    res = recs[0]
    if repeats > 1:
        res["chunk_log10"] = [x for r in recs for x in r["chunk_log10"]]
        res["chunk_paths"] = [x for r in recs for x in r["chunk_paths"]]
        res["paths"] = sum(r["paths"] for r in recs)
        res["perturb_ms"] = sum(r["perturb_ms"] for r in recs)
        res["runs"] = [{"perturbSeed": r["config"]["experiment"]["experimentParams"]["random"]["perturbSeed"],
                        "log10_weight": r["log10_weight"]} for r in recs]
        x = np.array([v for v, n in zip(res["chunk_log10"], res["chunk_paths"]) if n > 0])
        res["log10_weight"] = float(x.max() + np.log10((10.0 ** (x - x.max())).sum()) + res["log10_normalizer"])
        res["config"]["experiment"]["experimentParams"]["pathsToGenerate"] = res["paths"]
    json.dump(res, open(os.path.join(OUT, f"chain_{key}.json"), "w"))
    print(f"chain {key} N={N}: log10 W = {res['log10_weight']:.6f} in {res['perturb_ms']:.0f} ms")


def make_baseline_sets(tmp):
    """Fixtures at the benchmark configurations: tables, weighed batches and runner runs."""
    threads = os.cpu_count() or 1
    boot66 = ref_bootstrap(tmp, 66, 10.0, 7)
    assert np.array_equal(boot66, np.load(os.path.join(OUT, "boot_66.npy")))
    boot258 = ref_bootstrap(tmp, 258, 20.0, 7)
    np.save(os.path.join(OUT, "boot_258.npy"), boot258)
    boots = {66: boot66, 258: boot258}
    for name, mu, eps, scatter, absorption, nsteps, bins, N, S in BASELINE_LUTS:
        if "--runs-only" not in sys.argv:
            weighed_batch(tmp, name, mu, eps, scatter, absorption, nsteps, bins, N, S, boots[N],
                          BASELINE_PROPOSALS[name])
        # burn-in per chain: at N = 66 the reference's chains forget the initial curve within
        # 1000 steps; at N = 258 (S = 20 on a 12-unit chord) their first million steps still
        # relax (chunk sums 30 decades above the later ones), so that run skips 3e6 steps, and
        # runs 16 chains of one 1e6-path chunk each (its heavy-tailed weights want the standard
        # error from independent chains, not from consecutive chunks of a few: two runs of
        # 8 chains on distinct seeds)
        if N < 200:
            reference_chain_run(tmp, name, N, S, 16_000_000, threads, mu, eps, scatter, absorption, nsteps, bins,
                                boots[N])
        else:
            reference_chain_run(tmp, name, N, S, 8_000_000, 8, mu, eps, scatter, absorption, nsteps, bins, boots[N],
                                skip=3_000_000, repeats=2)


NORM_CASES = [
    (4, 0.25, [0, 0, 0, 0, 0, 1, 0.3, 0.1, 0.4, 0, 0, 1]),
    (4, 0.5, [0, 0, 0, 1, 0, 0, 0.7, 0.2, 0.1, 0, 1, 0]),
    (4, 0.1, [0, 0, 0, 0, 0, 1, 0, 0, 0.25, 0, 0, 1]),
    # N = 5 and 6 run the reference's nested 1e10-term quadrature (K5 and K6 both expand to the
    # same sum over F7, PathWeightUtils.cpp:705); z = 1.83 and 1.87, inside the K4 support
    (5, 0.25, [0, 0, 0, 0, 0, 1, 0.2, 0.1, 0.9, 0, 0, 1]),
    (6, 0.2, [0, 0, 0, 0, 0, 1, 0.1, 0.2, 0.7, 0, 0, 1]),
]


def make_norm():
    norm = []
    for N, ds, bc in NORM_CASES:
        out = run(["norm", N, repr(ds), *bc]).stdout.strip().splitlines()[-1]
        norm.append({"N": N, "ds": ds, "bc": bc, "log10": float(out)})
        print(f"norm N={N} ds={ds}: {float(out)!r}")
    json.dump(norm, open(os.path.join(OUT, "norm.json"), "w"), indent=1)


def main():
    if not os.path.exists(H):
        sys.exit("build the reference first: make -C oracle ref")
    if "--only" in sys.argv:
        what = sys.argv[sys.argv.index("--only") + 1]
        with tempfile.TemporaryDirectory() as tmp:
            if what == "baseline":
                make_baseline_sets(tmp)
            elif what == "norm":
                make_norm()
            else:
                sys.exit(f"unknown --only {what}")
        return
    rng = np.random.default_rng(20261203)
    with tempfile.TemporaryDirectory() as tmp:
        # ---- bootstrap curves
        boots = {}
        for N, S in ((10, 5.0), (18, 6.0), (34, 12.0), (66, 10.0)):
            boots[N] = ref_bootstrap(tmp, N, S, 7)
            np.save(os.path.join(OUT, f"boot_{N}.npy"), boots[N])
        # ---- independent-sample M-segment estimates (2^22 paths each)
        make_msegment(tmp)
        if "--msegment-only" in sys.argv:
            return
        # ---- tables and weighed path batches
        for name, mu, eps, scatter, absorption, nsteps, bins, N, S in LUTS:
            weighed_batch(tmp, name, mu, eps, scatter, absorption, nsteps, bins, N, S, boots[N])
        # ---- rotation
        n = 512
        q = rng.normal(size=(n, 4)).astype(F32)
        q /= np.linalg.norm(q, axis=1, keepdims=True)
        v = (rng.normal(size=(n, 3)) * 3).astype(F32)
        f = os.path.join(tmp, "rot.bin")
        with open(f, "wb") as fh:
            fh.write(struct.pack("<Q", n))
            fh.write(np.concatenate([q, v], 1).astype(F32).tobytes())
        run(["rotate", f, f + ".out"])
        np.savez(os.path.join(OUT, "rotate.npz"), q=q, v=v, out=np.fromfile(f + ".out", F32).reshape(n, 3))
        # ---- combined weights
        seqs = [rng.normal(-300, 20, 4000), np.sort(rng.normal(-50, 5, 1000)), np.full(64, -12.5),
                rng.normal(700, 40, 3000)]
        splits = [1500, 400, 32, 2999]
        recs = []
        for s, sp in zip(seqs, splits):
            f = os.path.join(tmp, "cw.bin")
            with open(f, "wb") as fh:
                fh.write(struct.pack("<QQ", len(s), sp))
                fh.write(np.asarray(s, np.float64).tobytes())
            run(["cw", f, f + ".out"])
            b = open(f + ".out", "rb").read()
            recs.append({"values": np.asarray(s).tolist(), "split": sp,
                         "cw": [list(struct.unpack("<dddII", b[i * 32:(i + 1) * 32])[:4]) for i in range(3)],
                         "extract_log10": list(struct.unpack("<ddd", b[96:120]))})
        json.dump(recs, open(os.path.join(OUT, "cw.json"), "w"))
        # ---- normaliser
        make_norm()
        # ---- reference Markov-chain runs (statistical parity): theta ~ U(-pi, pi), k <= 25
        for N, S, paths, threads in ((10, 5.0, 32_000_000, 8), (18, 6.0, 16_000_000, 8), (66, 10.0, 16_000_000, 8)):
            reference_chain_run(tmp, str(N), N, S, paths, threads, 1.0, 0.01, 10.0, 0.0, 2000, 1024, boots[N])
        # ---- the benchmark configurations
        make_baseline_sets(tmp)


if __name__ == "__main__":
    main()
