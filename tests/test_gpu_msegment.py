"""Independent-sample M-segment Monte Carlo (twisty_run_msegment) against the reference's own
estimator (golden fixtures from MSegmentPathGenerationMC's per-path work run through the
reference's functions): the mean weights agree within 3 combined standard errors."""
import json
import math
import os

import pytest

from conftest import GEOM, ROOT

import twisty_b200 as T

pytestmark = pytest.mark.gpu


def _fixture(N):
    with open(os.path.join(ROOT, "tests", "golden", f"msegment_{N}.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("form", [T.FORM_PLAIN_FP32, T.FORM_COMPENSATED])
@pytest.mark.parametrize("N", [10, 34, 66])
def test_msegment_matches_reference_estimator(N, form):
    ref = _fixture(N)
    g = GEOM[N]
    bc = T.make_bc(g[0], g[1], g[2], g[3], ref["S"])
    p = T.default_params(num_segments=N, mu=ref["mu"], eps=ref["eps"], scatter=ref["scatter"],
                         absorption=ref["absorption"], num_steps_int=ref["num_steps_int"],
                         num_curvature_steps=ref["bins"], paths_to_generate=1 << 22, perturb_seed=99,
                         form=form, lut_mode=T.LUT_FAITHFUL)
    with T.Context(p) as ctx:
        r = ctx.run_msegment(bc)
    assert r.total_paths + r.failed_paths == 1 << 22
    assert r.failed_paths < 1e-4 * (1 << 22)
    rel = abs(10 ** (r.log10_weight - ref["log10_mean"]) - 1)
    se = math.hypot(ref["rel_se"], r.rel_std_error)
    assert rel < 3 * se, (rel, se, r.log10_weight, ref["log10_mean"])


def test_msegment_refusals():
    bc = T.make_bc((0, 0, 0), (1, 0, 0), (8, 0, 0), (1, 0, 0), 10.0)
    with T.Context(T.default_params(num_segments=64, paths_to_generate=1000)) as ctx:   # N-2 = 62
        with pytest.raises(T.TwistyError):
            ctx.run_msegment(bc)
    with T.Context(T.default_params(num_segments=66, paths_to_generate=1000, form=T.FORM_FP64)) as ctx:
        with pytest.raises(T.TwistyError):
            ctx.run_msegment(bc)
