"""twisty_autotune: times the compensated kernel shapes for one N and records the fastest."""
import math

import pytest

import twisty_b200 as T

pytestmark = pytest.mark.gpu


def _params(N, **kw):
    base = dict(num_segments=N, mu=1.0, eps=0.01, scatter=10.0, num_steps_int=2000, num_curvature_steps=2048,
                form=T.FORM_COMPENSATED, lut_mode=T.LUT_FP64, perturb_seed=3, paths_to_generate=1 << 20,
                paths_to_skip=16, max_sub_chain=32, max_angle=0.05)
    base.update(kw)
    return T.default_params(**base)


def test_autotune_records_a_shape_that_later_runs_use(tmp_path):
    N = 100
    bc = T.make_bc((0, 0, 0), (0, 0, 1), (0, 0, 6), (0, 0, 1), 10.0)
    with T.Context(_params(N)) as ctx:
        best = ctx.autotune(bc, 1 << 19)
        assert best["num_segments"] == N and best["bins"] == 2048
        assert best["group"] * best["spl"] >= N and best["path_segments_per_s"] > 1e9
        r = ctx.run(bc)   # knobs at zero: the recorded shape, default chain count for it
    requested = 148 * best["warps"] * (32 // best["group"])   # the shape's default chain count
    steps = -(-(1 << 20) // requested)
    assert r.num_chains == -(-(1 << 20) // steps)
    assert r.total_paths == 1 << 20 and r.failed_paths == 0 and math.isfinite(r.log10_weight)
    out = tmp_path / "tune.json"
    T.tuning_cache_save(str(out))
    assert '"n": 100' in out.read_text()


def test_autotune_rejects_other_forms():
    bc = T.make_bc((0, 0, 0), (0, 0, 1), (0, 0, 6), (0, 0, 1), 10.0)
    with T.Context(_params(100, form=T.FORM_PLAIN_FP32)) as ctx:
        with pytest.raises(T.TwistyError):
            ctx.autotune(bc, 1 << 16)


def test_batch_keeps_the_default_for_a_tuned_shape_it_has_no_kernel_for(tmp_path):
    """A tuning-cache entry for a single-run-only shape (8 x 32) is used by single runs of its
    N and table size; batched runs of that N keep the default shape instead of failing."""
    import torch
    N, bins, paths = 222, 768, 1 << 14
    f = tmp_path / "tune.json"
    f.write_text('{"entries": [{"device": "%s", "n": %d, "bins": %d, "group": 8, "spl": 32, "warps": 16, '
                 '"path_segments_per_s": 1.0}]}' % (torch.cuda.get_device_name(0), N, bins))
    T.tuning_cache_load(str(f))
    bc = T.make_bc((0, 0, 0), (0, 0, 1), (0, 0, 15), (0, 0, 1), 30.0)
    with T.Context(_params(N, num_curvature_steps=bins, paths_to_generate=paths)) as ctx:
        res = ctx.run_batch([T.make_experiment(bc, N, 10.0, 0.01, paths)])
        r = ctx.run(bc)
    assert len(res) == 1 and res[0].total_paths == paths and res[0].failed_paths == 0
    assert math.isfinite(res[0].log10_weight)
    assert r.total_paths == paths and r.failed_paths == 0 and math.isfinite(r.log10_weight)


def test_measured_fp32_peak_is_near_the_nominal_rate():
    """twisty_measure_fp32_peak, the roofline's denominator: independent FMA chains in every lane
    reach the FP32 pipe's rate, 128 lanes x SMs x the SM clock (at most the 1965 MHz maximum)."""
    v = T.measure_fp32_peak(0)
    assert 0.5 * 148 * 128 * 1965e6 < v < 1.05 * 148 * 128 * 1965e6, v
