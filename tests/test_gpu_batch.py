"""Batched runs (twisty_run_batch): many experiments of uneven N, S, mu_s and eps in one pass.

Each experiment of a batch must give the result of a single-experiment run with the same
chains (same Philox stream id, chain count and steps, initial curve and per-experiment table):
the batch changes only how the chains are scheduled, not what they compute. The tables are
built on the device for the batch and on the host for single runs, so the log10 weights agree
to the rounding of the fixed-point table entries (far below 1e-6).
"""
import math

import numpy as np
import pytest

import twisty_b200 as T

pytestmark = pytest.mark.gpu

BASE = dict(mu=1.0, absorption=0.0, num_steps_int=2000, num_curvature_steps=1024, paths_to_skip=64,
            perturb_seed=4242, bootstrap_seed=11, max_sub_chain=32, max_angle=0.3,
            form=T.FORM_COMPENSATED, lut_mode=T.LUT_FP64, experiment_id=100)


def _experiments():
    rng = np.random.default_rng(7)
    out = []
    for n, paths in [(16, 1 << 13), (40, 1 << 14), (100, 1 << 14), (200, 20000), (300, 1 << 13), (700, 1 << 12)]:
        r = rng.uniform(2.0, 6.0)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        t = rng.normal(size=3)
        t /= np.linalg.norm(t)
        while True:
            S = r * rng.uniform(1.1, 1.8)
            bc = T.make_bc((0, 0, 0), (0, 0, 1), r * d, t, S)
            if T.min_arclength(bc, n) < S:
                break
        sigma = rng.uniform(0.08, 0.25)
        out.append(T.make_experiment(bc, n, rng.uniform(5.0, 30.0), sigma * sigma, paths))
    return out


def _single(e_idx, x, num_chains):
    p = T.default_params(num_segments=x.num_segments, eps=x.eps, scatter=x.scatter,
                         paths_to_generate=x.paths, num_chains=num_chains,
                         **{**BASE, "experiment_id": BASE["experiment_id"] + e_idx,
                            "bootstrap_seed": BASE["bootstrap_seed"] + e_idx})
    with T.Context(p) as ctx:
        return ctx.run(x.bc)


def test_batch_matches_single_runs():
    exps = _experiments()
    with T.Context(T.default_params(num_segments=16, eps=0.01, scatter=10.0, **BASE)) as ctx:
        res = ctx.run_batch(exps)
    assert len(res) == len(exps)
    for i, (x, r) in enumerate(zip(exps, res)):
        assert r.total_paths == x.paths
        assert r.failed_paths == 0
        assert math.isfinite(r.log10_weight)
        s = _single(i, x, r.num_chains)
        assert s.num_chains == r.num_chains and s.steps_per_chain == r.steps_per_chain
        assert s.total_paths == r.total_paths
        assert abs(s.log10_weight - r.log10_weight) < 1e-6, (i, x.num_segments, s.log10_weight, r.log10_weight)
        assert abs(s.log10_normalizer - r.log10_normalizer) < 1e-12


def test_batch_replays_are_identical():
    exps = _experiments()[:3]
    with T.Context(T.default_params(num_segments=16, eps=0.01, scatter=10.0, **BASE)) as ctx:
        a = ctx.run_batch(exps, iterations=1)
        b = ctx.run_batch(exps, iterations=3)
    for x, y in zip(a, b):
        assert x.log10_weight == y.log10_weight
        assert x.total_paths == y.total_paths


def test_batch_rejects_bad_experiment_with_its_index():
    exps = _experiments()[:3]
    bad = T.make_experiment(exps[1].bc, 2, 10.0, 0.01, 100)
    with T.Context(T.default_params(num_segments=16, eps=0.01, scatter=10.0, **BASE)) as ctx:
        with pytest.raises(T.TwistyError) as ei:
            ctx.run_batch([exps[0], bad, exps[2]])
        assert "experiment 1" in str(ei.value)


def test_batch_empty_experiment_and_empty_batch():
    exps = _experiments()[:2]
    exps[1].paths = 0
    with T.Context(T.default_params(num_segments=16, eps=0.01, scatter=10.0, **BASE)) as ctx:
        assert ctx.run_batch([]) == []
        res = ctx.run_batch(exps)
    assert res[1].total_paths == 0 and res[1].num_chains == 0
    assert res[0].total_paths == exps[0].paths


def test_batch_matches_oracle_fp64_twin(oracle):
    """Each experiment of a batch of uneven N against the oracle's FP64 twin chains on the same
    proposals (Philox stream of the experiment, chain ids, burn-in), the same initial curve and
    its own FP64 table (mu_s, eps, maxBound = 10/eps per experiment): within 1e-4 relative.
    Small rotation angles keep the FP32 and FP64 trajectories together."""
    base = {**BASE, "max_angle": 0.1}
    chains, steps = 256, 64
    exps = _experiments()[:5]
    for x in exps:
        x.paths = chains * steps
    with T.Context(T.default_params(num_segments=16, eps=0.01, scatter=10.0, num_chains=chains, **base)) as ctx:
        res = ctx.run_batch(exps)
    for i, (x, r) in enumerate(zip(exps, res)):
        assert r.num_chains == chains and r.steps_per_chain == steps and r.total_paths == chains * steps
        N = x.num_segments
        p = T.default_params(num_segments=N, **{**base, "bootstrap_seed": base["bootstrap_seed"] + i})
        init = T.bootstrap_curve(p, x.bc)
        ds = float(np.float32(x.bc.arclength) / np.float32(N))
        lut, meta = oracle.lut_f64(oracle.wparams(base["mu"], x.eps, x.scatter, 0.0, base["num_steps_int"],
                                                  base["num_curvature_steps"]), ds)
        o = oracle.run_chains(init, N, x.bc.arclength, lut, meta, seed=base["perturb_seed"], n_chains=chains,
                              steps=steps, burn_in=base["paths_to_skip"], k_max=base["max_sub_chain"],
                              max_angle=base["max_angle"], experiment=base["experiment_id"] + i, f64=True)
        ref = oracle.log10_sum(o["chain_log10"])
        rel = abs(10 ** (r.log10_weight - ref) - 1)
        assert rel < 1e-4, (i, N, r.log10_weight, ref, rel)
