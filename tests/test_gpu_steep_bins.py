"""Fixed-point tables with steep bins, through the C ABI. Needs a B200.

The compensated form's fixed-point table interpolates log10 of the reference's linear blend
by a secant; in a bin where that secant would err by more than 1e-7 per segment the table
stores a NaN slope, and a path that crosses such a bin is weighed again with the exact blend
through the linear table. Narrow phase functions (sigma = 0.05) give tables with a few steep
bins just below the replaced high-curvature tail; rotations of up to pi drive paths there.
"""
import math

import numpy as np
import pytest

import twisty_b200 as T

pytestmark = pytest.mark.gpu
F32 = np.float32

N, S = 24, 3.0
ANGLE = float(F32(np.pi))
W = dict(mu=1.0, eps=0.0025, scatter=40.0, num_steps_int=2000, num_curvature_steps=4096, lut_mode=T.LUT_FP64)


def _bc():
    return T.make_bc((0, 0, 0), (1, 0, 0), (2.0, 0, 0), (1, 0, 0), S)


def _params(**kw):
    base = dict(num_segments=N, form=T.FORM_COMPENSATED, perturb_seed=5, num_chains=1024,
                paths_to_generate=1024 * 400, paths_to_skip=50, max_sub_chain=25, max_angle=ANGLE, **W)
    base.update(kw)
    return T.default_params(**base)


def _steep_bins(lut, step):
    L = lut.astype(np.float64)
    r = L[1:] / L[:-1] - 1.0
    return np.nonzero((step * r) ** 2 / (8.0 * math.log(10.0)) > 1e-7)[0]


def test_run_keeps_the_fixed_point_table_and_loses_no_path():
    with T.Context(_params()) as ctx:
        lut, info = ctx.build_lut(F32(S) / F32(N))
        r = ctx.run(_bc())
    steep = _steep_bins(lut, float(info.curvature_step))
    assert len(steep) >= 1
    assert r.table_form == T.TABLE_FIXED_NARROW and r.steep_bins == len(steep)
    assert r.total_paths == 1024 * 400 and r.failed_paths == 0


def test_exported_weights_match_the_reference_weigher_on_steep_paths():
    """Per-path weights of the chain kernel (fixed-point table with the linear-table
    fallback) against the reference-semantics weigher on the exported geometry."""
    n_out = 20000
    with T.Context(_params(num_chains=256, paths_to_generate=256 * 200)) as ctx:
        lut, info = ctx.build_lut(F32(S) / F32(N))
        pos, w, _ = ctx.export_paths(_bc(), None, n_out)
        ref, valid, bins = ctx.weight_paths(_bc(), pos, form=T.FORM_PLAIN_FP32, want_bins=True)
        wc, vc, bc_ = ctx.weight_paths(_bc(), pos, form=T.FORM_COMPENSATED, want_bins=True)
    steep = _steep_bins(lut, float(info.curvature_step))
    hits = np.isin(bins, steep).any(axis=1)
    assert hits.sum() >= 10, hits.sum()                      # the case under test occurs
    assert np.all(valid == 1) and np.all(vc == 1) and np.all(np.isfinite(w))
    # The compensated weigher sees the same positions as the reference weigher: edge flips (a
    # curvature within rounding of a bin edge lands in the neighbour bin) aside, every path
    # agrees to 1e-5 relative, steep-bin paths included.
    same_bins = np.all(bc_ == bins, axis=1)
    rel_c = np.abs(wc - ref) / np.abs(ref)
    assert np.all(rel_c[same_bins & hits] < 1e-5), rel_c[same_bins & hits].max()
    assert np.median(rel_c) < 1e-6 and np.mean(rel_c < 1e-5) > 0.95
    # The chain kernel weighs its own tangents, of which the exported float positions are a
    # rounded image, so its bins near an edge can differ from the weigher's (unseen here; in
    # a steep bin the reference's blend jumps there by up to a few 1e-2 in log10). Most
    # steep-bin paths still agree to 1e-6, and none is lost or far off.
    rel_w = np.abs(w - ref) / np.abs(ref)
    assert np.median(rel_w) < 1e-6 and np.mean(rel_w < 1e-5) > 0.95
    assert np.median(rel_w[hits]) < 1e-6 and rel_w[hits].max() < 1e-2, rel_w[hits].max()


def test_incremental_and_batched_agree_with_the_full_recompute():
    bc = _bc()
    with T.Context(_params()) as ctx:
        full = ctx.run(bc)
    with T.Context(_params(incremental_resync=8)) as ctx:
        incr = ctx.run(bc)
    assert incr.failed_paths == 0 and incr.total_paths == full.total_paths
    assert abs(incr.log10_weight - full.log10_weight) < 1e-6, (incr.log10_weight, full.log10_weight)
    exp = T.make_experiment(bc, N, W["scatter"], W["eps"], 1024 * 400)
    with T.Context(_params()) as ctx:
        (b,) = ctx.run_batch([exp])
    assert b.table_form == T.TABLE_FIXED_NARROW and b.steep_bins == full.steep_bins
    assert b.failed_paths == 0
    assert abs(b.log10_weight - full.log10_weight) < 1e-6, (b.log10_weight, full.log10_weight)
