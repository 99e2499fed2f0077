"""The oracle's Philox-driven chains against the reference's own Markov-chain runs.

The reference draws its proposals from per-thread mt19937_64 streams, the oracle (and the
CUDA kernels) from Philox; the two runs are therefore compared statistically: the mean
path weight of each must agree within 3 combined standard errors, the standard error of
each coming from the spread of independent chain (or 1e6-path chunk) sums.
"""
import numpy as np
import pytest

from conftest import golden_json

F32 = np.float32


def chunk_stats(log10_sums, paths):
    """log10 of the mean path weight and its relative standard error from chunk sums."""
    x = np.asarray(log10_sums, np.float64)
    m = x.max()
    s = 10.0 ** (x - m)
    tot = s.sum()
    n = len(s)
    se = np.sqrt(n * s.var(ddof=1)) / tot
    return m + np.log10(tot) - np.log10(paths), se


def ref_stats(rec):
    x = [v for v, n in zip(rec["chunk_log10"], rec["chunk_paths"]) if n > 0]
    return chunk_stats(x, rec["paths"])


def oracle_run(oracle, rec, n_chains, steps, f64=False, threads=8):
    cfg = rec["config"]["experiment"]
    ep = cfg["experimentParams"]
    w = ep["weighting"]
    N = ep["numSegments"]
    S = cfg["basicExperiment"]["arclength"]
    init = np.load(f"tests/golden/boot_{N}.npy")
    wp = oracle.wparams(w["mu"], w["eps"], w["scatter"], w["absorption"], w["numStepsInt"], w["numCurvatureSteps"])
    if f64:
        lut, meta = oracle.lut_f64(wp, float(F32(S) / F32(N)))
    else:
        lut, meta = oracle.lut_f32(wp, F32(S) / F32(N))
    r = oracle.run_chains(init, N, S, lut, meta, seed=77, n_chains=n_chains, steps=steps,
                          burn_in=ep["pathsToSkip"], f64=f64, threads=threads)
    return chunk_stats(r["chain_log10"], n_chains * steps), r


@pytest.mark.parametrize("N,chains,steps", [(10, 4000, 500), (18, 2000, 500), (66, 400, 500)])
def test_oracle_chains_match_reference_runner(oracle, N, chains, steps):
    rec = golden_json(f"chain_{N}.json")
    ref_mean, ref_se = ref_stats(rec)
    mean, se, = oracle_run(oracle, rec, chains, steps)[0]
    tol = 3.0 * np.hypot(ref_se, se) / np.log(10.0)   # relative SE -> log10 units
    assert abs(mean - ref_mean) < tol, (mean, ref_mean, se, ref_se)


def test_fp32_chain_tracks_fp64_twin(oracle):
    """Same Philox proposals and small rotation angles: the FP32 reference-semantics chain and
    the FP64 twin follow the same trajectory (per-chain sums within ~1e-6 in log10)."""
    N, S = 18, 6.0
    init = np.load("tests/golden/boot_18.npy")
    wp = oracle.wparams(1.0, 0.01, 10.0, 0.0, 2000, 1024)
    ds = F32(S) / F32(N)
    l32, m32 = oracle.lut_f32(wp, ds)
    l64, m64 = oracle.lut_f64(wp, float(ds))
    kw = dict(seed=5, n_chains=64, steps=300, burn_in=200, max_angle=0.05, k_max=12)
    a = oracle.run_chains(init, N, S, l32, m32, **kw)
    b = oracle.run_chains(init, N, S, l64, m64, f64=True, **kw)
    # A curvature within rounding of a bin edge lands in a neighbouring bin; with the
    # reference's interpolation weight in curvature units (PathWeighters.cpp:79-82) that
    # moves the segment weight by (L_{i+1}-L_i)/L_i ~ 2e-3 here, so single chains may
    # differ by ~1e-4 while typical chains and the total agree to ~1e-6.
    d = np.abs(a["chain_log10"] - b["chain_log10"])
    assert np.median(d) < 1e-5 and d.max() < 1e-3
    assert abs(oracle.log10_sum(a["chain_log10"]) - oracle.log10_sum(b["chain_log10"])) < 2e-5


def test_large_angle_dynamics_decorrelate(oracle):
    """With the reference's U(-pi, pi) angles, rounding differences grow exponentially:
    after ~1000 steps FP32 and FP64 trajectories are unrelated, so such runs can only be
    compared statistically (test_oracle_chains_match_reference_runner)."""
    N, S = 18, 6.0
    init = np.load("tests/golden/boot_18.npy")
    wp = oracle.wparams(1.0, 0.01, 10.0, 0.0, 2000, 1024)
    ds = F32(S) / F32(N)
    l32, m32 = oracle.lut_f32(wp, ds)
    l64, m64 = oracle.lut_f64(wp, float(ds))
    kw = dict(seed=5, n_chains=16, steps=1, want_final=True)
    near = [oracle.run_chains(init, N, S, l, m, burn_in=10, f64=f, **kw)["final_pos"]
            for l, m, f in ((l32, m32, False), (l64, m64, True))]
    far = [oracle.run_chains(init, N, S, l, m, burn_in=1500, f64=f, **kw)["final_pos"]
           for l, m, f in ((l32, m32, False), (l64, m64, True))]
    assert np.abs(near[0] - near[1]).max() < 1e-5
    assert np.median(np.abs(far[0] - far[1]).max(axis=(1, 2))) > 1e-2
