"""Small N against the oracle's FP64 twin chains, through the C ABI. Needs a B200.

Below N = 49 the compensated form runs code paths of its own: forward passes turn the
complement of a sub-chain longer than half the path (the moved path up to one rotation of the
whole path, with the path's end-to-end chord carried through those moves); groups of 1 and 4
lanes apply each rotation as v + (R - I) v; long passes at N = 13..24 take the one-lane shapes
1 x 16 and 1 x 24; N = 37..48 take 4 x 12, which turns the shorter side as well. Every chain
here is compared, as a whole run, with the oracle's FP64 chains (oracle/twisty_oracle.c,
which turns the sub-chain itself by the reference's quaternion rotation) on the same
proposals (Philox stream, chain ids, burn-in), initial curve and FP64 table. Small rotation
angles keep the FP32 and FP64 trajectories together, so the estimates agree to the FP32
trajectory's rounding: 1.5e-7 of |log10 W| plus 1e-5.
"""
import numpy as np
import pytest

import twisty_b200 as T

pytestmark = pytest.mark.gpu

BASE = dict(mu=1.0, eps=0.01, scatter=10.0, num_steps_int=2000, num_curvature_steps=2048, perturb_seed=4321,
            max_sub_chain=32, max_angle=0.05, bootstrap_seed=7)
CHAINS, STEPS = 256, 2000


def _bc(N):
    S = max(0.12 * N, 1.0)
    return T.make_bc((0, 0, 0), (1, 0, 0), (0.55 * S, 0.1 * S, 0), (1, 0, 0), S)


# (N, burn-in, forced shape or None, the shape the run must take)
CASES = [
    (10, 4, None, (1, 12)),
    (12, 4, None, (1, 12)),
    (16, 4, None, (1, 16)),        # 512000 paths >= 60000 x 4 burn-in steps: one lane
    (16, 2, None, (1, 16)),        # >= 210000 x 2: one lane at 24 warps
    (16, 16, None, (4, 4)),        # a short pass against its burn-in: 4 lanes
    (20, 2, None, (1, 24)),        # 512000 >= 130000 x 2
    (24, 2, None, (1, 24)),
    (24, 8, None, (4, 8)),
    (32, 4, None, (4, 8)),
    (36, 4, None, (4, 9)),
    (40, 4, None, (4, 12)),
    (48, 4, None, (4, 12)),
    (20, 4, (4, 5, 32), (4, 5)),
]


@pytest.mark.parametrize("N,burn,force,shape", CASES)
def test_small_n_matches_oracle_fp64_chains(oracle, N, burn, force, shape):
    kw = dict(BASE, num_segments=N, form=T.FORM_COMPENSATED, lut_mode=T.LUT_FP64, num_chains=CHAINS,
              paths_to_generate=CHAINS * STEPS, paths_to_skip=burn)
    if force:
        kw.update(comp_group=force[0], comp_spl=force[1], comp_warps=force[2])
    p = T.default_params(**kw)
    bc = _bc(N)
    with T.Context(p) as ctx:
        r = ctx.run(bc)
    assert (r.kernel_shape >> 8, r.kernel_shape & 0xFF) == shape, hex(r.kernel_shape)
    assert r.total_paths == CHAINS * STEPS and r.failed_paths == 0 and r.steps_per_chain == STEPS
    init = T.bootstrap_curve(p, bc)
    ds = float(np.float32(bc.arclength) / np.float32(N))
    lut, meta = oracle.lut_f64(oracle.wparams(BASE["mu"], BASE["eps"], BASE["scatter"], 0.0, BASE["num_steps_int"],
                                              BASE["num_curvature_steps"]), ds)
    o = oracle.run_chains(init, N, bc.arclength, lut, meta, seed=BASE["perturb_seed"], n_chains=CHAINS, steps=STEPS,
                          burn_in=burn, k_max=BASE["max_sub_chain"], max_angle=BASE["max_angle"], f64=True)
    ref = oracle.log10_sum(o["chain_log10"])
    assert abs(r.log10_weight - ref) < 1.5e-7 * abs(ref) + 1e-5, (N, shape, r.log10_weight, ref)
