"""Receiver-grid drivers (twisty_b200.drivers): geometry of the reference's drivers, the
BeamSpread draws reproduced from std::mt19937, and (GPU) a batched pass per grid."""
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

import twisty_b200 as T
from twisty_b200 import drivers as D

F32 = np.float32


def test_ring_geometry():
    ex = D.ring_experiments((0, 0, 0), (0, 0, 1), 2.0, 1.0, 15.0, 8, 64, 20.0, 0.0225, 1000)
    assert len(ex) == 8
    for i, e in enumerate(ex):
        z = 1.0 + i * 2.0
        assert (e.bc.end_pos.x, e.bc.end_pos.y) == (2.0, 0.0) and abs(e.bc.end_pos.z - z) < 1e-6
        d = math.hypot(2.0, z)
        assert abs(e.bc.arclength - max(1.1 * d, 3.0)) < 1e-5
        t = (e.bc.end_dir.x, e.bc.end_dir.y, e.bc.end_dir.z)
        assert np.allclose(t, (2.0 / d, 0.0, z / d), atol=1e-6)


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_beam_spread_draws_match_std_mt19937(tmp_path):
    """std::uniform_real_distribution<float>(0, 1) over std::mt19937(seed), as the reference draws."""
    src = tmp_path / "d.cpp"
    src.write_text('#include <random>\n#include <cstdio>\nint main(){std::mt19937 g(42);'
                   'std::uniform_real_distribution<float> u(0.0f,1.0f);'
                   'for(int i=0;i<64;++i) printf("%.9g\\n",(double)u(g)); return 0;}\n')
    exe = tmp_path / "d"
    subprocess.run(["g++", "-O2", "-o", str(exe), str(src)], check=True)
    want = np.array([float(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()],
                    F32)
    got = D._mt19937_uniform_floats(42, 64)
    assert np.array_equal(got, want)


def test_beam_spread_and_image_geometry():
    b = D.beam_spread_experiments((0, 0, 0), (0, 0, 1), 5.0, 16, 42, 64, 20.0, 0.0225, 1000)
    for e in b:
        p = np.array([e.bc.end_pos.x, e.bc.end_pos.y, e.bc.end_pos.z])
        assert abs(np.linalg.norm(p) - 5.0) < 1e-5
        assert e.bc.arclength > T.min_arclength(e.bc, 64)
    im = D.image_plane_experiments(8, 4, 4.0, 10.0, 512, 20.0, 0.0225, 1000)
    assert len(im) == 32
    xs = sorted({round(e.bc.end_pos.x, 6) for e in im})
    assert xs[0] == -3.5 and xs[-1] == 3.5 and all(e.bc.end_pos.z == 10.0 for e in im)


@pytest.mark.gpu
def test_ring_sweep_as_one_batch_matches_single_runs():
    ex = D.ring_experiments((0, 0, 0), (0, 0, 1), 1.5, 4.0, 8.0, 3, 64, 20.0, 0.0225, 20000)
    base = dict(num_segments=64, mu=1.0, eps=0.0225, scatter=20.0, num_steps_int=2000, num_curvature_steps=1024,
                form=T.FORM_COMPENSATED, lut_mode=T.LUT_FP64, perturb_seed=5, paths_to_skip=16, max_sub_chain=32,
                max_angle=0.1)
    with T.Context(T.default_params(**base)) as ctx:
        res = D.run(ctx, ex)
    for i, (e, r) in enumerate(zip(ex, res)):
        assert r.total_paths == 20000 and math.isfinite(r.log10_weight)
        p = T.default_params(**dict(base, paths_to_generate=20000, num_chains=r.num_chains, experiment_id=i,
                                    bootstrap_seed=i))
        with T.Context(p) as c:
            s = c.run(e.bc)
        assert abs(s.log10_weight - r.log10_weight) < 1e-6


@pytest.mark.gpu
def test_beam_spread_batch_matches_oracle_fp64_twin(oracle):
    """The BeamSpread receivers (the reference's own draws) as one batch, each experiment against
    the oracle's FP64 twin chains on the same proposals, initial curve and its own FP64 table:
    within 1e-4 relative (small rotation angles keep FP32 and FP64 trajectories together)."""
    chains, steps = 256, 64
    ex = D.beam_spread_experiments((0, 0, 0), (0, 0, 1), 3.0, 4, 42, 48, 20.0, 0.0225, chains * steps)
    base = dict(num_segments=48, mu=1.0, eps=0.0225, scatter=20.0, num_steps_int=2000, num_curvature_steps=1024,
                form=T.FORM_COMPENSATED, lut_mode=T.LUT_FP64, perturb_seed=9, paths_to_skip=32, max_sub_chain=32,
                max_angle=0.1, num_chains=chains, bootstrap_seed=21, experiment_id=3)
    with T.Context(T.default_params(**base)) as ctx:
        res = D.run(ctx, ex)
    for i, (e, r) in enumerate(zip(ex, res)):
        assert r.num_chains == chains and r.steps_per_chain == steps
        init = T.bootstrap_curve(T.default_params(**dict(base, bootstrap_seed=21 + i)), e.bc)
        ds = float(F32(e.bc.arclength) / F32(48))
        lut, meta = oracle.lut_f64(oracle.wparams(1.0, e.eps, e.scatter, 0.0, 2000, 1024), ds)
        o = oracle.run_chains(init, 48, e.bc.arclength, lut, meta, seed=9, n_chains=chains, steps=steps, burn_in=32,
                              k_max=32, max_angle=0.1, experiment=3 + i, f64=True)
        ref = oracle.log10_sum(o["chain_log10"])
        assert abs(10 ** (r.log10_weight - ref) - 1) < 1e-4, (i, r.log10_weight, ref)
