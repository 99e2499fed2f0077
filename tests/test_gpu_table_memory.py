"""Where the compensated form keeps the weight table (twisty_params.comp_table_memory), through
the C ABI. Needs a B200.

The reference's own configurations mostly use 20000-bin tables (160 KB): staged in shared
memory beside the chain state they would leave a CTA a quarter of its warps, so forward passes
read them through L1 instead. The 20- and 24-segment shapes, whose 24 warps leave little room
beside the chain state, stage a table at 20 warps where it fits there (8192 bins in the
20-segment shapes). Both placements run the same arithmetic on the same table values, so with
the same chain layout their results are identical.
"""
import pytest

import twisty_b200 as T
from twisty_b200 import _abi

pytestmark = pytest.mark.gpu


def _params(N, bins, **kw):
    base = dict(num_segments=N, mu=1.0, eps=0.01, scatter=10.0, num_steps_int=2000, num_curvature_steps=bins,
                form=T.FORM_COMPENSATED, lut_mode=T.LUT_FP64, perturb_seed=99, num_chains=1024,
                paths_to_generate=1024 * 100, paths_to_skip=20, max_sub_chain=32, max_angle=0.05)
    base.update(kw)
    return T.default_params(**base)


def _bc(N):
    S = 0.08 * N
    return T.make_bc((0, 0, 0), (0, 0, 1), (0, 0, 0.6 * S), (0, 0, 1), S)


@pytest.mark.parametrize("N", [64, 256, 700])
def test_l1_and_shared_tables_give_identical_results(N):
    out = []
    for mem in (1, 2):
        with T.Context(_params(N, 20000, comp_table_memory=mem, comp_warps=4)) as ctx:
            out.append(ctx.run(_bc(N)))
    assert out[0].total_paths == out[1].total_paths == 1024 * 100
    assert out[0].log10_weight == out[1].log10_weight


@pytest.mark.parametrize("N", [64, 256, 1024])
def test_table_too_large_for_shared_memory_runs_through_l1(N):
    """100000 bins (800 KB) cannot be staged at all: the default placement reads it through L1
    and agrees with the FP64 form on the same proposals."""
    res = {}
    for form in (T.FORM_COMPENSATED, T.FORM_FP64):
        with T.Context(_params(N, 100000, form=form)) as ctx:
            res[form] = ctx.run(_bc(N))
    a, b = res[T.FORM_COMPENSATED], res[T.FORM_FP64]
    assert a.total_paths == b.total_paths and a.failed_paths == 0
    assert abs(a.log10_weight - b.log10_weight) < 1.5e-7 * abs(b.log10_weight) + 1e-5, (a.log10_weight, b.log10_weight)
    # forcing shared memory is refused with a clear status
    with T.Context(_params(N, 100000, comp_table_memory=1)) as ctx:
        with pytest.raises(T.TwistyError) as ei:
            ctx.run(_bc(N))
    assert "too large" in str(ei.value)


def test_invalid_table_memory_is_rejected():
    with T.Context(_params(64, 4096, comp_table_memory=3)) as ctx:
        with pytest.raises(T.TwistyError) as ei:
            ctx.run(_bc(64))
    assert ei.value.status == _abi.ERR_INVALID_CONFIG and "comp_table_memory" in str(ei.value)


@pytest.mark.parametrize("N,group", [(80, 4), (160, 8), (320, 16), (640, 32)])
def test_twenty_segment_shapes_stage_8192_bin_tables_at_20_warps(N, group):
    """An 8192-bin table (64 KB) does not fit beside 24 warps of a 20-segment shape's chain
    state; the default placement stages it at 20 warps instead of reading it through L1 at 24.
    Same chains as the L1 placement at 20 warps (identical result) and as the FP64 form."""
    s = T.default_shape(N, 8192)
    assert (s["group"], s["spl"], s["warps"], s["table_in_l1"]) == (group, 20, 20, 0), s
    chains = 148 * 20 * (32 // group)
    kw = dict(num_chains=chains, paths_to_generate=chains * 40)
    res = {}
    for key, extra in (("staged", {}), ("l1", dict(comp_warps=20, comp_table_memory=2)),
                       ("fp64", dict(form=T.FORM_FP64))):
        with T.Context(_params(N, 8192, **kw, **extra)) as ctx:
            res[key] = ctx.run(_bc(N))
    a, b, c = res["staged"], res["l1"], res["fp64"]
    assert a.kernel_shape == b.kernel_shape == (group << 8) | 20
    assert a.total_paths == b.total_paths == c.total_paths == chains * 40 and a.failed_paths == 0
    assert a.log10_weight == b.log10_weight
    assert abs(a.log10_weight - c.log10_weight) < 1.5e-7 * abs(c.log10_weight) + 1e-5, (a.log10_weight, c.log10_weight)
