"""Incremental weight updates (incremental_resync = R > 1): the same chains as the full
recompute, each weighted path's total updated from the two curvatures its rotation changed
and recomputed in full every R-th weighted step. Estimates agree with the full recompute and
with the FP64 form on the same proposals."""
import pytest

import twisty_b200 as T

pytestmark = pytest.mark.gpu


def _run(N, S, resync, form=T.FORM_COMPENSATED, bins=4096):
    p = T.default_params(num_segments=N, mu=1.0, eps=0.01, scatter=10.0, num_steps_int=2000,
                         num_curvature_steps=bins, form=form, lut_mode=T.LUT_FP64, perturb_seed=17, num_chains=2048,
                         paths_to_generate=2048 * 400, paths_to_skip=64, max_sub_chain=32, max_angle=0.05,
                         incremental_resync=resync)
    with T.Context(p) as ctx:
        return ctx.run(T.make_bc((0, 0, 0), (0, 0, 1), (0, 0, 12), (0, 0, 1), S))


@pytest.mark.parametrize("N,S", [(64, 14.0), (256, 20.0), (700, 40.0)])
def test_incremental_matches_full_recompute_and_fp64(N, S):
    full = _run(N, S, 0)
    inc = _run(N, S, 32)
    f64 = _run(N, S, 0, form=T.FORM_FP64)
    assert inc.total_paths == full.total_paths == 2048 * 400
    assert inc.failed_paths == 0
    rel_full = abs(10 ** (inc.log10_weight - full.log10_weight) - 1)
    rel_f64 = abs(10 ** (inc.log10_weight - f64.log10_weight) - 1)
    assert rel_full < 1e-5, rel_full
    assert rel_f64 < 1e-4, rel_f64


def test_resync_every_step_is_the_full_recompute():
    """R = 1 (and 0) means every weighted step is recomputed in full: identical results."""
    a = _run(256, 20.0, 0)
    b = _run(256, 20.0, 1)
    assert a.log10_weight == b.log10_weight
