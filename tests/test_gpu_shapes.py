"""Every kernel shape of the compensated form against the FP64 form, through the C ABI.
Needs a B200.

The default shape depends on N (4, 8, 16 or 32 lanes per chain x 2..32 segments per lane), so
a sweep of N, powers of two, 2^k + 2 (the reference's own configurations) and the N just
past them (only the group's last slots padded, or most of them), covers every shape and both
the full and the padded curvature loops. Small
rotation angles keep the FP32 and FP64 trajectories together, so the two estimates of
log10(experimentWeight) agree to ~1e-7 of its magnitude (the per-segment rounding of the
FP32 trajectory adds up along the path: at N = 384, |log10 w| = 430, that is 5e-5) on the
same proposals; a wrong mask or padded slot would move it by whole segment weights.
"""
import pytest

import twisty_b200 as T

pytestmark = pytest.mark.gpu

NS = [4, 5, 6, 7, 8, 9, 10, 12, 13, 14, 16, 17, 18, 20, 31, 32, 33, 34, 36, 40, 48, 64, 65, 66, 72, 76, 80, 96, 100, 128, 129, 130,
      136, 150, 160, 170, 192, 200, 256, 257, 258, 272, 300, 320, 350, 384, 400, 420, 448, 512, 513, 514, 544, 600, 640, 768, 800, 850, 896,
      1000, 1024]


def _params(N, form, **kw):
    base = dict(num_segments=N, mu=1.0, eps=0.01, scatter=10.0, num_steps_int=2000, num_curvature_steps=2048,
                form=form, lut_mode=T.LUT_FP64, perturb_seed=4321, num_chains=512, paths_to_generate=512 * 64,
                paths_to_skip=16, max_sub_chain=32, max_angle=0.05)
    base.update(kw)
    return T.default_params(**base)


def _bc(N):
    S = max(0.12 * N, 1.0)
    return T.make_bc((0, 0, 0), (1, 0, 0), (0.55 * S, 0.1 * S, 0), (1, 0, 0), S)


@pytest.mark.parametrize("N", NS)
def test_default_shape_matches_fp64(N):
    res = {}
    for form in (T.FORM_COMPENSATED, T.FORM_FP64):
        with T.Context(_params(N, form)) as ctx:
            res[form] = ctx.run(_bc(N))
    a, b = res[T.FORM_COMPENSATED], res[T.FORM_FP64]
    assert a.total_paths == b.total_paths == 512 * 64
    assert a.failed_paths == 0
    assert abs(a.log10_weight - b.log10_weight) < 1.5e-7 * abs(b.log10_weight) + 1e-5, (a.log10_weight, b.log10_weight)


@pytest.mark.parametrize("N,shapes", [(24, [(4, 8, 32), (8, 4, 32), (16, 4, 16), (32, 4, 16)]),
                                      (150, [(16, 12, 16), (8, 32, 8), (16, 16, 16), (32, 8, 16)]),
                                      (170, [(8, 24, 16), (16, 12, 16), (16, 16, 16)]),
                                      (300, [(16, 20, 16), (32, 12, 16)]),
                                      (440, [(16, 28, 16), (32, 16, 16)]),
                                      (600, [(32, 20, 16), (32, 24, 16)]),
                                      (700, [(32, 24, 8), (32, 32, 8)]),
                                      (850, [(32, 28, 8), (32, 32, 8)])])
def test_shapes_agree_on_the_same_chains(N, shapes):
    """The same chains under different shapes: the proposals and the fixed-point path totals
    are the same; only the float reduction order of the rotation axis differs."""
    out = []
    for g, spl, w in shapes:
        with T.Context(_params(N, T.FORM_COMPENSATED, comp_group=g, comp_spl=spl, comp_warps=w)) as ctx:
            r = ctx.run(_bc(N))
        assert r.total_paths == 512 * 64 and r.failed_paths == 0
        out.append(r.log10_weight)
    assert max(out) - min(out) < 1e-5 * abs(out[0]) + 1e-6, out


@pytest.mark.parametrize("N,shape", [(80, (4, 20, 24)), (90, (4, 24, 20)), (96, (4, 24, 24)), (112, (4, 28, 16)),
                                     (100, (4, 28, 20)), (128, (4, 32, 12)), (120, (4, 32, 16)),
                                     (16, (4, 4, 32)), (16, (1, 16, 16)), (13, (1, 16, 24)), (24, (1, 24, 16)),
                                     (20, (1, 24, 12)), (18, (1, 24, 16))])
def test_explicit_shape_matches_fp64(N, shape):
    """Shapes the defaults do not pick at these N (the autotuner's candidates, among them the
    one-lane 1 x 16 and 1 x 24 that long passes take at N = 13..24), full and padded, with the
    table staged and through L1, against the FP64 form on the same proposals."""
    g, spl, w = shape
    with T.Context(_params(N, T.FORM_COMPENSATED, comp_group=g, comp_spl=spl, comp_warps=w)) as ctx:
        a = ctx.run(_bc(N))
    with T.Context(_params(N, T.FORM_FP64)) as ctx:
        b = ctx.run(_bc(N))
    assert a.total_paths == b.total_paths == 512 * 64
    assert a.failed_paths == 0
    assert abs(a.log10_weight - b.log10_weight) < 1.5e-7 * abs(b.log10_weight) + 1e-5, (a.log10_weight, b.log10_weight)


@pytest.mark.parametrize("N,angle", [(10, 0.05), (12, 0.05), (24, 0.05), (32, 0.05), (36, 0.05), (48, 0.05), (24, 0.3),
                                     (36, 0.3), (48, 0.3)])
def test_long_chains_turning_the_shorter_side_match_fp64(N, angle):
    """Below N = 49 the forward kernels turn the complement of a sub-chain that is longer than
    half the path (by -theta about the same chord: the moved path up to one rotation of the
    whole path) and carry the path's end-to-end chord d through those moves, re-summed every
    16 steps. The FP64 form always turns the sub-chain itself. Few chains with many steps each
    (16384) would show a drift of d as a drift of the weights; they agree as short chains do.
    (At N <= 12 with 0.3 rad moves the FP32 and FP64 trajectories of such long chains part by
    3e-5 to 2e-3 in log10 whichever side is turned, as they did before complements were turned;
    0.05 rad keeps them together there.)"""
    kw = dict(num_chains=64, paths_to_generate=64 * 16384, max_angle=angle)
    res = {}
    for form in (T.FORM_COMPENSATED, T.FORM_FP64):
        with T.Context(_params(N, form, **kw)) as ctx:
            res[form] = ctx.run(_bc(N))
    a, b = res[T.FORM_COMPENSATED], res[T.FORM_FP64]
    assert a.total_paths == b.total_paths == 64 * 16384
    assert a.failed_paths == 0
    assert abs(a.log10_weight - b.log10_weight) < 1.5e-7 * abs(b.log10_weight) + 1e-5, (a.log10_weight, b.log10_weight)
