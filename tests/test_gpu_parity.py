"""Parity of the CUDA library (through its C ABI) with the oracle and the reference's own
golden outputs. Every test here needs a B200 (marker `gpu`)."""
import math

import numpy as np
import pytest

from conftest import GEOM, LUT_SETS, golden_json, golden_npz

import twisty_b200 as T
from twisty_b200 import _abi

pytestmark = pytest.mark.gpu
F32 = np.float32


def lut_params(name, **kw):
    mu, eps, sc, ab, nst, bins, N, S = LUT_SETS[name]
    return T.default_params(num_segments=N, mu=mu, eps=eps, scatter=sc, absorption=ab, num_steps_int=nst,
                            num_curvature_steps=bins, **kw), N, S


def geom_bc(N, S):
    g = GEOM[N]
    return T.make_bc(g[0], g[1], g[2], g[3], S)


def golden_lut_info(name):
    g = golden_npz(f"lut_{name}.npz")
    h = g["hdr"]
    info = _abi.LutInfo(float(h[0]), float(h[1]), float(h[2]), float(h[3]), float(h[4]), float(h[5]), g["lut"].size)
    return g["lut"], info


# ------------------------------------------------------------------------------ tables
@pytest.mark.parametrize("name", sorted(LUT_SETS))
def test_faithful_table_bit_exact_with_reference(name):
    p, N, S = lut_params(name, lut_mode=T.LUT_FAITHFUL)
    g = golden_npz(f"lut_{name}.npz")
    with T.Context(p) as ctx:
        lut, info = ctx.build_lut(F32(S) / F32(N))
    assert np.array_equal(lut.view(np.uint32), g["lut"].view(np.uint32))
    h = g["hdr"]
    assert (info.min_curvature, info.max_curvature, info.curvature_step, info.min_segment_weight,
            info.max_segment_weight) == (h[0], h[1], h[2], h[3], h[4])


@pytest.mark.parametrize("name", sorted(LUT_SETS))
def test_fp64_table_matches_oracle_twin(oracle, name):
    p, N, S = lut_params(name, lut_mode=T.LUT_FP64)
    mu, eps, sc, ab, nst, bins, _, _ = LUT_SETS[name]
    ds = F32(S) / F32(N)
    ref, _ = oracle.lut_f64(oracle.wparams(mu, eps, sc, ab, nst, bins), float(ds))
    with T.Context(p) as ctx:
        lut, _ = ctx.build_lut(ds)
    assert np.max(np.abs(lut - ref) / ref) < 1.2e-7


def test_batched_fp64_tables_match_oracle_twin(oracle, tmp_path):
    """The batched builder (one launch for a set of tables, read back from the multi-ds cache
    file) on a narrow-phase set (sigma = 0.05) whose high-curvature tail is replaced by the
    smallest positive entry, and a broad one."""
    for mu, eps, sc, nst, bins, lo, hi, n_ds in ((1.0, 0.0025, 5.0, 2000, 4096, 0.0195, 0.05, 3),
                                                  (1.0, 0.09, 50.0, 2000, 2048, 0.1, 0.3, 3)):
        p = T.default_params(num_segments=64, mu=mu, eps=eps, scatter=sc, num_steps_int=nst, num_curvature_steps=bins,
                             lut_mode=T.LUT_MULTI_DS)
        path = tmp_path / f"set_{eps}.twmd"
        with T.Context(p) as ctx:
            ctx.multi_ds_tables(lo, hi, n_ds, str(path))
        raw = path.read_bytes()
        tabs = np.frombuffer(raw, np.float32, offset=60 + 16 * n_ds).reshape(n_ds, bins)
        step = (F32(hi) - F32(lo)) / F32(n_ds - 1)
        for i in range(n_ds):
            ds = F32(lo) + F32(i) * step
            ref, _ = oracle.lut_f64(oracle.wparams(mu, eps, sc, 0.0, nst, bins), float(ds))
            assert np.max(np.abs(tabs[i] - ref) / ref) < 1.2e-7, (eps, i)


# ------------------------------------------------------------------------ weighting
@pytest.mark.parametrize("name", sorted(LUT_SETS))
def test_plain_weigher_matches_reference(name):
    p, N, S = lut_params(name)
    paths = golden_npz(f"paths_{name}.npz")
    lut, info = golden_lut_info(name)
    with T.Context(p) as ctx:
        ctx.set_lut(lut, info)
        w, v, b = ctx.weight_paths(geom_bc(N, S), paths["pos"], form=T.FORM_PLAIN_FP32, want_bins=True)
    assert np.array_equal(v, paths["valid"])
    assert np.array_equal(b, paths["bins"])                     # bit-exact bins
    assert np.max(np.abs(w - paths["log10w"])) < 1e-12           # FP64 log10 may differ by an ulp


# Edge window of the compensated weigher, in units of 2^-24 (the unit roundoff of the unit
# tangents' coordinates). A curvature is |t_{i+1} - t_i| N/S, a difference of two unit vectors,
# so its rounding error is set by the rounding of the tangent coordinates, not by the ulp of
# the curvature itself; in bins that is 2^-24 * kscale, kscale = (N/S) / step (= (bins - 1) /
# 2.02 for the reference's tables). The compensated weigher normalises with the hardware
# reciprocal square root and scales the tangents to kscale, a few roundings more than the
# reference's 1/sqrtf; its bin may differ from the reference's only where the reference's
# curvature lies within EDGE_ULPS of them of a bin edge (4096 bins: 1.9e-3 of a bin).
EDGE_ULPS = 16


def edge_jumps_log10(lut, step):
    """|log10| of the jump of the reference's segment weight at each bin edge e (between bins
    e-1 and e): the blend reaches L_{e-1} + step (L_e - L_{e-1}) just below the edge (its
    interpolation weight is in curvature units, Twisty/PathWeighters.cpp:79-82) and L_e at it."""
    L = lut.astype(np.float64)
    below = L[:-1] + float(step) * (L[1:] - L[:-1])
    return np.concatenate([[0.0], np.abs(np.log10(L[1:]) - np.log10(below))])


@pytest.mark.parametrize("name", sorted(LUT_SETS))
def test_compensated_weigher_matches_reference(name):
    p, N, S = lut_params(name)
    paths = golden_npz(f"paths_{name}.npz")
    lut, info = golden_lut_info(name)
    with T.Context(p) as ctx:
        ctx.set_lut(lut, info)
        w, v, b = ctx.weight_paths(geom_bc(N, S), paths["pos"], form=T.FORM_COMPENSATED, want_bins=True)
    assert np.array_equal(v, paths["valid"])
    # bins bit-exact except for curvatures within EDGE_ULPS tangent roundings of a bin edge
    step = float(info.curvature_step)
    kscale = float(F32(N) / F32(S)) / step
    r = paths["curv"].astype(np.float64) / step
    edge_dist = np.abs(r - np.round(r))
    mism = b != paths["bins"]
    window = EDGE_ULPS * 2.0 ** -24 * kscale
    assert not np.any(mism & (edge_dist >= window)), (edge_dist[mism].max() / (2.0 ** -24 * kscale), window)
    assert np.abs(b - paths["bins"]).max() <= 1
    # per-path log10 weights within 1e-5 relative; a path with edge flips may move further, by
    # at most the weight jumps at the edges it crossed
    jumps = edge_jumps_log10(lut, step)
    edge = np.maximum(b, paths["bins"])
    allowed = np.where(mism, jumps[np.clip(edge, 0, lut.size - 1)], 0.0).sum(axis=1)
    ref = paths["log10w"]
    dev = np.abs(w - ref)
    assert np.all(dev <= 1e-5 * np.abs(ref) + allowed * (1 + 1e-6)), (dev - allowed).max()
    flip = mism.any(axis=1)
    assert np.all(dev[~flip] < 1e-5 * np.abs(ref[~flip])), (dev[~flip] / np.abs(ref[~flip])).max()


# ---------------------------------------------------------------------------- chains
def chain_ctx(name, form, seed=1234, chains=256, steps=200, burn=50, k_max=25, angle=float(F32(np.pi)), lut_ext=True):
    p, N, S = lut_params(name, form=form, perturb_seed=seed, num_chains=chains, paths_to_generate=chains * steps,
                         paths_to_skip=burn, max_sub_chain=k_max, max_angle=angle)
    ctx = T.Context(p)
    if lut_ext:
        lut, info = golden_lut_info(name)
        ctx.set_lut(lut, info)
    boot = np.load(f"tests/golden/boot_{N}.npy")
    ctx.set_initial_curve(boot)
    return ctx, N, S, boot


@pytest.mark.parametrize("name,angle,k_max", [("A", float(F32(np.pi)), 25), ("C", float(F32(np.pi)), 25), ("B", 0.05, 25),
                                              ("D", 0.1, 32), ("E", 0.05, 32), ("E", float(F32(np.pi)), 25)])
def test_plain_chains_bit_exact_with_oracle(oracle, name, angle, k_max):
    """Plain chains against the oracle's FP32 chains, bit for bit in log10 (FP64 log10 and sums
    may differ in the last place), on the reference's and the benchmark's proposals."""
    ctx, N, S, boot = chain_ctx(name, T.FORM_PLAIN_FP32, angle=angle, k_max=k_max)
    r = ctx.run(geom_bc(N, S))
    ctx.close()
    lut, info = golden_lut_info(name)
    mu, eps, sc, ab, nst, bins, _, _ = LUT_SETS[name]
    olut, meta = oracle.lut_f32(oracle.wparams(mu, eps, sc, ab, nst, bins), F32(S) / F32(N))
    o = oracle.run_chains(boot, N, S, olut, meta, seed=1234, n_chains=256, steps=200, burn_in=50, k_max=k_max,
                          max_angle=angle, absorption=ab)
    ref = oracle.log10_sum(o["chain_log10"])
    assert r.total_paths == int(o["chain_valid"].sum()) == 256 * 200
    assert abs(r.log10_weight - ref) < 1e-11, (r.log10_weight, ref)


def test_fp64_form_matches_oracle_twin(oracle):
    name = "A"
    ctx, N, S, boot = chain_ctx(name, T.FORM_FP64, angle=0.05, lut_ext=False)
    ctx.update(lut_mode=T.LUT_FP64)
    r = ctx.run(geom_bc(N, S))
    ctx.close()
    mu, eps, sc, ab, nst, bins, _, _ = LUT_SETS[name]
    olut, meta = oracle.lut_f64(oracle.wparams(mu, eps, sc, ab, nst, bins), float(F32(S) / F32(N)))
    o = oracle.run_chains(boot, N, S, olut, meta, seed=1234, n_chains=256, steps=200, burn_in=50, k_max=25,
                          max_angle=0.05, f64=True)
    assert abs(r.log10_weight - oracle.log10_sum(o["chain_log10"])) < 1e-9


@pytest.mark.parametrize("name", ["A", "B", "D", "E"])
def test_compensated_within_1e4_of_fp64(name):
    """Small rotation angles keep FP32 and FP64 trajectories together: the compensated
    estimate agrees with the FP64 form on the same proposals to better than 1e-4."""
    res = {}
    for form in (T.FORM_COMPENSATED, T.FORM_FP64):
        p, N, S = lut_params(name, form=form, perturb_seed=99, num_chains=2048, paths_to_generate=2048 * 500,
                             paths_to_skip=100, max_sub_chain=32, max_angle=0.1, lut_mode=T.LUT_FP64)
        with T.Context(p) as ctx:
            ctx.set_initial_curve(np.load(f"tests/golden/boot_{N}.npy"))
            res[form] = ctx.run(geom_bc(N, S))
    a, b = res[T.FORM_COMPENSATED], res[T.FORM_FP64]
    assert a.total_paths == b.total_paths == 2048 * 500
    rel = abs(10 ** (a.log10_weight - b.log10_weight) - 1)
    assert rel < 1e-4, rel


@pytest.mark.parametrize("N", [300, 700, 1024])
def test_long_paths_compensated_within_1e4_of_fp64(N):
    """Long paths: N = 300 keeps 32-bit fixed-point path totals, 700 and 1024 need the wide
    (64-bit total) form; both agree with the FP64 form on the same proposals."""
    res = {}
    for form in (T.FORM_COMPENSATED, T.FORM_FP64):
        p = T.default_params(num_segments=N, mu=1.0, eps=0.01, scatter=10.0, num_steps_int=2000,
                             num_curvature_steps=4096, form=form, perturb_seed=5, num_chains=1024,
                             paths_to_generate=1024 * 200, paths_to_skip=50, max_sub_chain=32, max_angle=0.05,
                             lut_mode=T.LUT_FP64)
        with T.Context(p) as ctx:
            res[form] = ctx.run(T.make_bc((0, 0, 0), (0, 0, 1), (0, 0, 12), (0, 0, 1), 20.0))
    a, b = res[T.FORM_COMPENSATED], res[T.FORM_FP64]
    assert a.total_paths == b.total_paths == 1024 * 200
    assert a.failed_paths == 0
    rel = abs(10 ** (a.log10_weight - b.log10_weight) - 1)
    assert rel < 1e-4, rel


# (reference run, chains, weighted steps per chain) of the GPU side, every chain with the
# reference run's 1000-step burn-in
STAT_RUNS = [("10", 8000, 1000), ("18", 8000, 1000), ("66", 8000, 1000), ("D", 8000, 1000)]


@pytest.mark.parametrize("key,chains,steps", STAT_RUNS)
@pytest.mark.parametrize("form", [T.FORM_COMPENSATED, T.FORM_PLAIN_FP32])
def test_statistics_match_reference_runner(key, chains, steps, form):
    """MC estimate within 3 standard errors of the reference CPU runner's own run (the
    reference's proposals: k <= 25, angles in (-pi, pi)); D and E are the benchmark
    configurations."""
    rec = golden_json(f"chain_{key}.json")
    ep = rec["config"]["experiment"]["experimentParams"]
    w = ep["weighting"]
    N = ep["numSegments"]
    S = rec["config"]["experiment"]["basicExperiment"]["arclength"]
    p = T.default_params(num_segments=N, mu=w["mu"], eps=w["eps"], scatter=w["scatter"], absorption=w["absorption"],
                         num_steps_int=w["numStepsInt"], num_curvature_steps=w["numCurvatureSteps"], form=form,
                         perturb_seed=2024, paths_to_generate=chains * steps, paths_to_skip=ep["pathsToSkip"],
                         num_chains=chains, lut_mode=T.LUT_FAITHFUL)
    with T.Context(p) as ctx:
        ctx.set_initial_curve(np.load(f"tests/golden/boot_{N}.npy"))
        r = ctx.run(geom_bc(N, S))
    x = np.array([v for v, n in zip(rec["chunk_log10"], rec["chunk_paths"]) if n > 0])
    m = x.max()
    s = 10 ** (x - m)
    ref_mean = m + np.log10(s.sum()) - np.log10(rec["paths"])
    ref_se = np.sqrt(len(s) * s.var(ddof=1)) / s.sum()
    got_mean = r.log10_mean_weight
    tol = 3 * np.hypot(ref_se, r.rel_std_error) / np.log(10)
    assert abs(got_mean - ref_mean) < tol, (got_mean, ref_mean, r.rel_std_error, ref_se)


def test_chain_sums_match_reference_runner_n258():
    """The precision-form configuration (N = 258, S = 20, receiver (0,0,12), 8192 bins) under the
    reference's proposals. Its chains need millions of steps to forget the initial curve, and
    their path weights are heavy-tailed: the reference's 16 chains (3e6 burn-in steps, then one
    1e6-path chunk each) have sums spread over 3 decades, and its two runs of 8 chains differ by
    1.5 decades in total. The mean of so few chains, and its standard error, are dominated by the
    largest one or two, so a 3-standard-error test of means is not informative here; the chains
    are compared as distributions instead: 256 chains of the same length and burn-in, their
    log10 sums against the reference's 16 by a two-sided Mann-Whitney test at level 1e-3, and
    their medians within the spread of the reference's. The compensated form runs it; the plain
    form's chains are the oracle's bit for bit at this configuration
    (test_plain_chains_bit_exact_with_oracle), and one plain-form thread per chain would take
    minutes over these 4e6-step chains."""
    form = T.FORM_COMPENSATED
    from scipy.stats import mannwhitneyu
    rec = golden_json("chain_E.json")
    ep = rec["config"]["experiment"]["experimentParams"]
    w = ep["weighting"]
    N = ep["numSegments"]
    S = rec["config"]["experiment"]["basicExperiment"]["arclength"]
    ref = np.array([v for v, n in zip(rec["chunk_log10"], rec["chunk_paths"]) if n == 1_000_000])
    assert ref.size == 16
    chains, steps = 256, 1_000_000
    p = T.default_params(num_segments=N, mu=w["mu"], eps=w["eps"], scatter=w["scatter"], absorption=w["absorption"],
                         num_steps_int=w["numStepsInt"], num_curvature_steps=w["numCurvatureSteps"], form=form,
                         perturb_seed=2024, paths_to_generate=chains * steps, paths_to_skip=ep["pathsToSkip"],
                         num_chains=chains, lut_mode=T.LUT_FAITHFUL)
    with T.Context(p) as ctx:
        ctx.set_initial_curve(np.load("tests/golden/boot_258.npy"))
        r = ctx.run(geom_bc(N, S))
        mine, valid = ctx.chain_results(r.num_chains)
    assert r.num_chains == chains and r.steps_per_chain == steps and np.all(valid == steps)
    pval = mannwhitneyu(mine, ref, alternative="two-sided").pvalue
    assert pval > 1e-3, (pval, np.median(mine), np.median(ref), ref.min(), ref.max())
    assert ref.min() <= np.median(mine) <= ref.max()


def test_results_state_their_error_against_fp64():
    """Every result carries a bound of its arithmetic against FP64 (per path, for the path's own
    curvatures), and with fp64_check_chains the measured relative error of its first chains'
    weight against the FP64 form replaying them: equal to what a separate FP64 run of the same
    chains gives."""
    chains, steps = 512, 200
    kw = dict(perturb_seed=99, num_chains=chains, paths_to_generate=chains * steps, paths_to_skip=100,
              max_sub_chain=32, max_angle=0.1, lut_mode=T.LUT_FP64)
    p, N, S = lut_params("D", form=T.FORM_COMPENSATED, fp64_check_chains=chains, **kw)
    with T.Context(p) as ctx:
        ctx.set_initial_curve(np.load("tests/golden/boot_66.npy"))
        a = ctx.run(geom_bc(N, S))
        assert ctx.kernels_per_launch() == 3
    p64, _, _ = lut_params("D", form=T.FORM_FP64, **kw)
    with T.Context(p64) as ctx:
        ctx.set_initial_curve(np.load("tests/golden/boot_66.npy"))
        b = ctx.run(geom_bc(N, S))
    assert a.fp64_check_chains == chains and math.isnan(b.fp64_rel_error) and b.weight_error_bound == 0.0
    assert a.fp64_rel_error == pytest.approx(abs(10 ** (a.log10_weight - b.log10_weight) - 1), rel=1e-6, abs=1e-12)
    assert a.fp64_rel_error < 1e-4
    assert 0.0 < a.weight_error_bound < 1e-4
    pp, _, _ = lut_params("D", form=T.FORM_PLAIN_FP32, **kw)
    with T.Context(pp) as ctx:
        c = ctx.run(geom_bc(N, S))
    assert math.isnan(c.fp64_rel_error) and c.weight_error_bound == pytest.approx(65 * 2.6e-8)


def test_runs_are_deterministic_and_split_api_matches():
    p, N, S = lut_params("A", perturb_seed=7, paths_to_generate=300_000, paths_to_skip=10)
    bc = geom_bc(N, S)
    with T.Context(p) as ctx:
        a = ctx.run(bc)
        b = ctx.run(bc)
        ctx.prepare(bc)
        ctx.launch()
        c = ctx.collect()
        assert ctx.kernels_per_launch() == 2
    assert a.log10_weight == b.log10_weight == c.log10_weight
    assert a.total_paths == 300_000


def test_runner_mirror_api():
    cfg = golden_json("chain_66.json")["config"]
    cfg["experiment"]["experimentParams"]["pathsToGenerate"] = 100_000
    ep, bc = T.ParseExperimentParamsFromConfig(cfg)
    res = T.FullExperimentRunnerOptimalPerturb(ep).RunExperiment(bc)
    assert res.totalPathsGenerated == 100_000 and np.isfinite(res.experimentWeightLog10)
    res2 = T.FullExperimentRunnerOptimalPerturbOptimized_GPU(ep).RunExperiment(bc)
    assert res2.experimentWeightLog10 == res.experimentWeightLog10


def test_normalizer_k4_matches_reference():
    with T.Context(T.default_params(num_segments=4)) as ctx:
        for rec in golden_json("norm.json"):
            if rec["N"] != 4:
                continue
            b = rec["bc"]
            bc = _abi.BC(_abi.Vec3(*b[0:3]), _abi.Vec3(*b[3:6]), _abi.Vec3(*b[6:9]), _abi.Vec3(*b[9:12]),
                         rec["ds"] * 4)
            assert ctx.normalizer_log10(4, rec["ds"], bc) == pytest.approx(rec["log10"], rel=1e-14, abs=1e-14)


@pytest.mark.parametrize("N", [5, 6])
def test_normalizer_k5_k6_match_reference(N):
    """The device quadrature of K5 / K6 (1e10 K4 terms, FP64 sums) against the reference's own
    Norm (PathWeightUtils.cpp:721-752, accumulated in its big-float type): the node positions and
    K4 terms are the reference's float arithmetic, so only the summation order differs."""
    recs = [r for r in golden_json("norm.json") if r["N"] == N]
    assert recs
    with T.Context(T.default_params(num_segments=N)) as ctx:
        for rec in recs:
            b = rec["bc"]
            bc = _abi.BC(_abi.Vec3(*b[0:3]), _abi.Vec3(*b[3:6]), _abi.Vec3(*b[6:9]), _abi.Vec3(*b[9:12]),
                         rec["ds"] * N)
            got = ctx.normalizer_log10(N, rec["ds"], bc)
            assert abs(got - rec["log10"]) < 1e-9, (got, rec["log10"])


def test_error_statuses():
    p, N, S = lut_params("A", paths_to_generate=1000)
    with T.Context(p) as ctx:
        with pytest.raises(T.TwistyError) as e:
            ctx.run(T.make_bc((0, 0, 0), (1, 0, 0), (20, 0, 0), (1, 0, 0), 10.0))
        assert e.value.status == _abi.ERR_INFEASIBLE_GEOMETRY
        ctx.update(num_steps_int=2001)
        with pytest.raises(T.TwistyError) as e:
            ctx.run(geom_bc(N, S))
        assert e.value.status == _abi.ERR_INVALID_CONFIG
        ctx.update(num_steps_int=2000, perturb_method=1)
        with pytest.raises(T.TwistyError) as e:
            ctx.run(geom_bc(N, S))
        assert e.value.status == _abi.ERR_UNSUPPORTED
        ctx.update(perturb_method=0)
        assert ctx.run(geom_bc(N, S)).total_paths == 1000   # the context stays usable


@pytest.mark.parametrize("form", [T.FORM_PLAIN_FP32, T.FORM_COMPENSATED])
def test_weighers_on_degenerate_and_clamped_paths(oracle, form):
    """Edge cases of the weighers against the oracle (pinned to the reference): a path with a
    zero-length segment, whose tangent is NaN and which the reference marks invalid
    (PathWeighters.cpp:89-92), and curvatures beyond a truncated table's range, clamped to its
    last bin (:45-65)."""
    p, N, S = lut_params("A")
    paths = golden_npz("paths_A.npz")
    pos = paths["pos"].copy()
    pos[5, 11] = pos[5, 10]          # zero-length segment 10 of path 5
    pos[7, 40] = pos[7, 41]          # and segment 40 of path 7
    lut, info = golden_lut_info("A")
    keep = lut.size // 8             # a table covering the lowest eighth of the curvature range
    step = F32(info.curvature_step)
    lut_t = np.ascontiguousarray(lut[:keep])
    max_k = float(F32(step * F32(keep - 1)))
    info_t = _abi.LutInfo(0.0, max_k, float(step), float(lut_t.min()), float(lut_t.max()), info.ds, keep)
    meta = oracle.LutMeta(0.0, max_k, float(step), float(lut_t.min()), float(lut_t.max()), info.ds, keep, 0)
    ow, ov, ob, oc = oracle.weigh_f32(pos, N, S, lut_t, meta, want_bins=True, want_curv=True)
    assert ov[5] == 0 and ov[7] == 0 and ov.sum() == ov.size - 2
    assert np.any(oc[ov == 1] > max_k)   # some curvatures beyond the table, clamped
    with T.Context(p) as ctx:
        ctx.set_lut(lut_t, info_t)
        w, v, b = ctx.weight_paths(geom_bc(N, S), pos, form=form, want_bins=True)
    assert np.array_equal(v, ov)
    ok = ov == 1
    if form == T.FORM_PLAIN_FP32:
        assert np.array_equal(b[ok], ob[ok]) and np.max(np.abs(w[ok] - ow[ok])) < 1e-12
    else:
        assert np.all(np.abs(w[ok] - ow[ok]) < 1e-5 * np.abs(ow[ok]) + edge_jumps_log10(lut_t, step)[
            np.clip(np.maximum(b[ok], ob[ok]), 0, keep - 1)].sum(axis=1) * (b[ok] != ob[ok]).any(axis=1))


def test_empty_passes_and_batches():
    """Zero paths: a run reports no paths and a weight of zero (log10 -inf), weighing no paths
    is a no-op, and an empty batch returns nothing."""
    p, N, S = lut_params("A", paths_to_generate=0)
    with T.Context(p) as ctx:
        r = ctx.run(geom_bc(N, S))
        assert r.total_paths == 0 and r.num_chains == 0 and r.log10_weight == -math.inf
        w, v, b = ctx.weight_paths(geom_bc(N, S), np.zeros((0, N + 1, 3), np.float32), form=T.FORM_PLAIN_FP32)
        assert w.size == 0
        assert ctx.run_batch([]) == []
