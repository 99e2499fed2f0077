"""torch.autograd binding (twisty_b200.autograd): forward = RunExperiment's log10 weight,
backward = the library's adjoint of the same chains."""
import numpy as np
import pytest
import torch

from conftest import GEOM

import twisty_b200 as T
from twisty_b200.autograd import _moved, _with, experiment_log10_weight

pytestmark = pytest.mark.gpu

N, S = 66, 10.0


def _setup():
    g = GEOM[N]
    bc = T.make_bc(g[0], g[1], g[2], g[3], S)
    p = T.default_params(num_segments=N, mu=1.0, eps=0.01, scatter=10.0, num_steps_int=4000,
                         num_curvature_steps=4096, form=T.FORM_COMPENSATED, lut_mode=T.LUT_FP64, perturb_seed=31,
                         num_chains=4096, paths_to_generate=4096 * 300, paths_to_skip=100, max_sub_chain=32,
                         max_angle=0.1)
    return p, bc, np.array(g[2], dtype=np.float64)


def test_autograd_matches_the_adjoint_of_the_same_run():
    p, bc, rx = _setup()
    mu = torch.tensor(10.0, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(0.1, dtype=torch.float64, requires_grad=True)
    rec = torch.tensor(rx, dtype=torch.float64, requires_grad=True)
    y = experiment_log10_weight(mu, sig, rec, p, bc)
    y.backward()
    p2, bc2 = _with(p, 10.0, 0.1), _moved(bc, rx)   # the parameters the binding runs with
    with T.Context(p2) as ctx:
        fwd = ctx.run(bc2)
        g = ctx.adjoint(bc2, fwd)
    assert y.item() == fwd.log10_weight
    assert mu.grad.item() == pytest.approx(g[0], rel=1e-12)
    assert sig.grad.item() == pytest.approx(g[1], rel=1e-12)
    assert np.allclose(rec.grad.numpy(), g[2:], rtol=1e-12, atol=0)


def test_autograd_chain_rule_and_fd():
    """Gradients flow through an outer expression; d/d(mu_s) agrees with a central difference
    of the forward (common random numbers, h = 1e-3 relative)."""
    p, bc, rx = _setup()
    a = torch.tensor(2.0, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(0.1, dtype=torch.float64)
    rec = torch.tensor(rx, dtype=torch.float64)
    y = 3.0 * experiment_log10_weight(a * 5.0, sig, rec, p, bc)
    y.backward()
    h = 1e-3
    with torch.no_grad():
        yp = experiment_log10_weight(torch.tensor(10.0 * (1 + h), dtype=torch.float64), sig, rec, p, bc)
        ym = experiment_log10_weight(torch.tensor(10.0 * (1 - h), dtype=torch.float64), sig, rec, p, bc)
    fd = 3.0 * 5.0 * (yp.item() - ym.item()) / (2 * h * 10.0)
    assert abs(a.grad.item() - fd) < 1e-3 * abs(fd), (a.grad.item(), fd)


def test_autograd_rejects_forms_without_an_adjoint():
    p, bc, rx = _setup()
    p.form = T.FORM_PLAIN_FP32
    with pytest.raises(T.TwistyError):
        experiment_log10_weight(torch.tensor(10.0, dtype=torch.float64), torch.tensor(0.1, dtype=torch.float64),
                                torch.tensor(rx), p, bc)
