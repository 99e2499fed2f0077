"""Multi-arclength table sets (twisty_multi_ds_tables, lut_mode LUT_MULTI_DS): the reference's
CachedMultiArclengthWeightLookupTable built in one batched device quadrature, cached on disk,
and the closest table taken per run (single and batched)."""
import numpy as np
import pytest

import twisty_b200 as T

pytestmark = pytest.mark.gpu

F32 = np.float32
N = 64
W = dict(mu=1.0, eps=0.01, scatter=10.0, num_steps_int=2000, num_curvature_steps=1024)
RUN = dict(num_segments=N, form=T.FORM_COMPENSATED, perturb_seed=8, num_chains=512, paths_to_generate=512 * 200,
           paths_to_skip=32, max_sub_chain=32, max_angle=0.05)
MIN_DS, MAX_DS, NDS = 0.1, 0.3, 21


def _bc(S):
    return T.make_bc((0, 0, 0), (1, 0, 0), (0.5 * S, 0, 0), (1, 0, 0), S)


def _grid(i):
    step = (F32(MAX_DS) - F32(MIN_DS)) / F32(NDS - 1)
    return float(F32(MIN_DS) + F32(i) * step)


def test_multi_ds_run_on_a_grid_point_equals_the_exact_table(tmp_path):
    ds = _grid(7)
    S = float(F32(ds) * F32(N))
    assert float(F32(S) / F32(N)) == ds
    with T.Context(T.default_params(lut_mode=T.LUT_MULTI_DS, **W, **RUN)) as ctx:
        ctx.multi_ds_tables(MIN_DS, MAX_DS, NDS, str(tmp_path / "set.twmd"))
        a = ctx.run(_bc(S))
    with T.Context(T.default_params(lut_mode=T.LUT_FP64, **W, **RUN)) as ctx:
        b = ctx.run(_bc(S))
    assert a.log10_weight == b.log10_weight
    # a second context reads the same set from the cache file
    with T.Context(T.default_params(lut_mode=T.LUT_MULTI_DS, **W, **RUN)) as ctx:
        ctx.multi_ds_tables(MIN_DS, MAX_DS, NDS, str(tmp_path / "set.twmd"))
        c = ctx.run(_bc(S))
    assert c.log10_weight == a.log10_weight


def test_multi_ds_batch_takes_the_closest_table_per_experiment():
    Ss = [N * d for d in (0.115, 0.183, 0.2, 0.271)]
    exps = [T.make_experiment(_bc(S), N, W["scatter"], W["eps"], 512 * 100) for S in Ss]
    base = dict(RUN, paths_to_generate=512 * 100)
    with T.Context(T.default_params(lut_mode=T.LUT_MULTI_DS, **W, **base)) as ctx:
        ctx.multi_ds_tables(MIN_DS, MAX_DS, NDS)
        res = ctx.run_batch(exps)
        for i, (S, r) in enumerate(zip(Ss, res)):
            ctx.update(experiment_id=i, bootstrap_seed=base.get("bootstrap_seed", 0) + i, num_chains=r.num_chains)
            s = ctx.run(_bc(S))
            assert abs(s.log10_weight - r.log10_weight) < 1e-6, (i, s.log10_weight, r.log10_weight)
        ctx.update(experiment_id=0, bootstrap_seed=0, num_chains=512)


def test_multi_ds_refusals():
    with T.Context(T.default_params(lut_mode=T.LUT_MULTI_DS, **W, **RUN)) as ctx:
        with pytest.raises(T.TwistyError):
            ctx.run(_bc(12.0))                       # no set built
        ctx.multi_ds_tables(MIN_DS, MAX_DS, NDS)
        bad = T.make_experiment(_bc(12.0), N, 20.0, W["eps"], 1000)
        with pytest.raises(T.TwistyError) as ei:
            ctx.run_batch([T.make_experiment(_bc(12.0), N, W["scatter"], W["eps"], 1000), bad])
        assert "experiment 1" in str(ei.value)
        with pytest.raises(T.TwistyError):
            ctx.multi_ds_tables(0.3, 0.1, NDS)       # empty range
