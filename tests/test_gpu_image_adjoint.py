"""The batched adjoint (twisty_adjoint_batch) on a receiver grid: the image drivers' pixel loop
(Experiments/BeamSpreadExperiment.cpp:240-269, NoisyCircleExperiment.cpp:259-361) differentiated
in one forward pass of the batch and one persistent adjoint replay. Needs a B200.

Each pixel's gradient must be the single-experiment adjoint of the same chains (same Philox
stream, chain layout, initial curve and table), and the gradient of the image's total
log-energy, log10 sum_pixels W_p, with respect to the mu_s and sigma all pixels share must match
central finite differences of that total (common random numbers, h = 1e-3 relative).
"""
import math

import numpy as np
import pytest

import twisty_b200 as T
from twisty_b200 import drivers as D

pytestmark = pytest.mark.gpu

N, SCATTER, SIGMA = 66, 20.0, 0.15
CHAINS, STEPS = 1024, 64
BASE = dict(mu=1.0, absorption=0.0, num_steps_int=2000, num_curvature_steps=2048, paths_to_skip=200,
            perturb_seed=777, bootstrap_seed=3, max_sub_chain=32, max_angle=0.1, form=T.FORM_COMPENSATED,
            lut_mode=T.LUT_FP64, experiment_id=40, num_chains=CHAINS)


def _grid(scatter=SCATTER, sigma=SIGMA):
    eps = float(np.float32(sigma) * np.float32(sigma))
    return D.image_plane_experiments(4, 4, 4.0, 10.0, N, scatter, eps, CHAINS * STEPS)


def _ctx():
    return T.Context(T.default_params(num_segments=N, eps=0.0225, scatter=SCATTER, **BASE))


def test_pixel_gradients_equal_single_experiment_adjoints():
    exps = _grid()
    with _ctx() as ctx:
        res, grad, total, timing = ctx.adjoint_batch(exps)
        fwd = ctx.run_batch(exps)
    assert np.all(np.isfinite(grad)) and timing[1] > 0
    for i, (x, r) in enumerate(zip(exps, res)):
        assert r.total_paths == CHAINS * STEPS and r.log10_weight == fwd[i].log10_weight
        p = T.default_params(num_segments=N, eps=x.eps, scatter=x.scatter, paths_to_generate=x.paths,
                             **{**BASE, "experiment_id": BASE["experiment_id"] + i,
                                "bootstrap_seed": BASE["bootstrap_seed"] + i})
        with T.Context(p) as c:
            s = c.run(x.bc)
            g = c.adjoint(x.bc, s)
        assert abs(s.log10_weight - r.log10_weight) < 1e-6
        scale = np.abs(g).max()
        assert np.all(np.abs(grad[i] - g) < 1e-5 * scale), (i, grad[i], g)
    # the total: log-sum of the pixels, its gradient the weighted mean of theirs
    L = np.array([r.log10_weight for r in res])
    m = L.max()
    w = 10.0 ** (L - m)
    assert total[0] == pytest.approx(m + math.log10(w.sum()), abs=1e-12)
    assert total[1] == pytest.approx((w * grad[:, 0]).sum() / w.sum(), rel=1e-12)
    assert total[2] == pytest.approx((w * grad[:, 1]).sum() / w.sum(), rel=1e-12)


def _total_log10(scatter=SCATTER, sigma=SIGMA):
    with _ctx() as ctx:
        res = ctx.run_batch(_grid(scatter, sigma))
    L = np.array([r.log10_weight for r in res])
    m = L.max()
    return m + math.log10((10.0 ** (L - m)).sum())


def test_image_log_energy_gradient_matches_central_differences():
    with _ctx() as ctx:
        _, _, total, _ = ctx.adjoint_batch(_grid())
    h = 1e-3
    fd_mu = (_total_log10(scatter=SCATTER * (1 + h)) - _total_log10(scatter=SCATTER * (1 - h))) / (2 * h * SCATTER)
    fd_sig = (_total_log10(sigma=SIGMA * (1 + h)) - _total_log10(sigma=SIGMA * (1 - h))) / (2 * h * SIGMA)
    assert abs(total[1] - fd_mu) < 1e-3 * abs(fd_mu), (total[1], fd_mu)
    assert abs(total[2] - fd_sig) < 1e-3 * abs(fd_sig), (total[2], fd_sig)


def test_adjoint_batch_rejects_tables_it_cannot_differentiate():
    with T.Context(T.default_params(num_segments=N, eps=0.0225, scatter=SCATTER,
                                    **{**BASE, "lut_mode": T.LUT_FAITHFUL})) as ctx:
        with pytest.raises(T.TwistyError) as e:
            ctx.adjoint_batch(_grid()[:2])
        assert e.value.status == 8
