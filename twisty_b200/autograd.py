"""torch.autograd binding of the experiment estimate and its adjoint.

``experiment_log10_weight(mu_s, sigma, receiver, params, bc)`` returns log10 experimentWeight
(the reference's RunExperiment result, Twisty/ExperimentRunner.h:73-82, in log10) as a 0-d
float64 tensor whose backward calls the library's adjoint pass (twisty_adjoint): gradients
with respect to the scattering coefficient mu_s, the phase width sigma (eps = sigma^2) and
the receiver position (the fixed end points N-1 and N move together, the interior is held).
The adjoint replays exactly the chains of the forward pass (same Philox streams), so the
gradient is that of the estimate the forward returned, not of a fresh one.

The forward and the adjoint both run on the GPU in the compensated form with FP64-built
tables (lut_mode FP64, which also builds the derivative tables); torch supplies only the
graph bookkeeping.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _abi
from . import FORM_COMPENSATED, LUT_FP64, Context, TwistyError


def _with(params: _abi.Params, mu_s: float, sigma: float) -> _abi.Params:
    p = _abi.Params()
    C.pointer(p)[0] = params
    p.scatter = float(mu_s)
    eps = np.float32(sigma) * np.float32(sigma)
    p.eps = float(eps)
    p.max_bound = float(np.float32(10.0) / eps)   # maxBound = 10/eps (Twisty/ExperimentRunner.cpp:169-171)
    return p


def _moved(bc: _abi.BC, receiver) -> _abi.BC:
    b = _abi.BC()
    C.pointer(b)[0] = bc
    b.end_pos = _abi.Vec3(*(float(v) for v in receiver))
    return b


class ExperimentLog10Weight(torch.autograd.Function):
    """log10 experimentWeight as a function of (mu_s, sigma, receiver position)."""

    @staticmethod
    def forward(fctx, mu_s, sigma, receiver, params, bc):
        if params.form != FORM_COMPENSATED or params.lut_mode != LUT_FP64:
            raise TwistyError(8, "the adjoint replays the compensated form with lut_mode FP64")
        p = _with(params, mu_s.item(), sigma.item())
        b = _moved(bc, receiver.detach().cpu().numpy())
        run = Context(p)
        res = run.run(b)
        fctx.run, fctx.bc, fctx.res = run, b, res
        fctx.dtypes = (mu_s.dtype, sigma.dtype, receiver.dtype)
        return torch.tensor(res.log10_weight, dtype=torch.float64, device=mu_s.device)

    @staticmethod
    def backward(fctx, grad_out):
        g = fctx.run.adjoint(fctx.bc, fctx.res)   # d/d(mu_s), d/d(sigma), d/d(receiver x, y, z)
        fctx.run.close()
        go = grad_out.to(torch.float64)
        dm, ds, dr = fctx.dtypes
        d_mu = (go * float(g[0])).to(dm)
        d_sigma = (go * float(g[1])).to(ds)
        d_rx = (go * torch.tensor(g[2:5], dtype=torch.float64, device=grad_out.device)).to(dr)
        return d_mu, d_sigma, d_rx, None, None


def experiment_log10_weight(mu_s: torch.Tensor, sigma: torch.Tensor, receiver: torch.Tensor,
                            params: _abi.Params, bc: _abi.BC) -> torch.Tensor:
    """One RunExperiment with mu_s, sigma and the receiver position taken from tensors.

    params: the context parameters (form COMPENSATED, lut_mode FP64); its scatter, eps and
    max_bound are replaced by mu_s, sigma^2 and 10/sigma^2. bc: the boundary conditions; its
    end position is replaced by receiver (3 values)."""
    return ExperimentLog10Weight.apply(mu_s, sigma, receiver, params, bc)
