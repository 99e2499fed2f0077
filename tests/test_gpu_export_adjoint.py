"""Path export (the reference's .pbd/.bdt/.pmd/.bcf/index.json set) and the adjoint,
through the C ABI. Needs a B200."""
import os

import numpy as np
import pytest

from conftest import GEOM, LUT_SETS, golden_npz

import twisty_b200 as T
from twisty_b200 import _abi

pytestmark = pytest.mark.gpu
F32 = np.float32


def bc_for(N, S):
    g = GEOM[N]
    return T.make_bc(g[0], g[1], g[2], g[3], S)


def golden_lut(name):
    g = golden_npz(f"lut_{name}.npz")
    h = g["hdr"]
    return g["lut"], _abi.LutInfo(*map(float, h[:6]), g["lut"].size)


def test_plain_export_matches_oracle_paths(oracle, tmp_path):
    mu, eps, sc, ab, nst, bins, N, S = LUT_SETS["A"]
    chains, steps, burn = 64, 20, 5
    p = T.default_params(num_segments=N, form=T.FORM_PLAIN_FP32, perturb_seed=55, num_chains=chains,
                         paths_to_generate=chains * steps, paths_to_skip=burn, mu=mu, eps=eps, scatter=sc,
                         num_steps_int=nst, num_curvature_steps=bins)
    boot = np.load("tests/golden/boot_66.npy")
    lut, info = golden_lut("A")
    with T.Context(p) as ctx:
        ctx.set_lut(lut, info)
        ctx.set_initial_curve(boot)
        pos, w, r = ctx.export_paths(bc_for(N, S), str(tmp_path), 200)
    assert pos.shape == (200, N + 1, 3) and r.total_paths == chains * steps
    olut, meta = oracle.lut_f32(oracle.wparams(mu, eps, sc, ab, nst, bins), F32(S) / F32(N))
    o = oracle.run_chains(boot, N, S, olut, meta, seed=55, n_chains=10, steps=steps, burn_in=burn, want_paths=True)
    assert np.max(np.abs(w - o["path_log10"][:200])) < 1e-11
    # exported positions re-weighed by the reference-semantics oracle give the same weights
    ow, ov, _, _ = oracle.weigh_f32(pos, N, S, olut, meta, want_bins=False)
    assert np.all(ov == 1) and np.max(np.abs(ow - w)) < 1e-11
    out = tmp_path / "GeneratedCurves"
    assert os.path.getsize(out / "BoundaryConditions.bcf") == 56
    assert os.path.getsize(out / "Paths_Binary.pbd") == 200 * (N + 1) * 12
    lin = np.fromfile(out / "Log10PathWeights_Binary.bdt", np.float64)
    assert np.allclose(np.log10(lin), w + r.log10_normalizer, rtol=0, atol=1e-9)
    meta_lines = (out / "Paths_Metadata.pmd").read_text().split("\n")
    assert meta_lines[0] == f"0 0 {steps}"
    assert (out / "index.json").exists() and os.path.getsize(out / "FiveSegment_Binary.bdt") == 200 * 12


def test_compensated_export_geometry_and_weights(oracle, tmp_path):
    mu, eps, sc, ab, nst, bins, N, S = LUT_SETS["B"]
    p = T.default_params(num_segments=N, form=T.FORM_COMPENSATED, perturb_seed=3, num_chains=256,
                         paths_to_generate=256 * 50, paths_to_skip=20, mu=mu, eps=eps, scatter=sc, absorption=ab,
                         num_steps_int=nst, num_curvature_steps=bins, max_sub_chain=16, max_angle=0.1)
    bc = bc_for(N, S)
    with T.Context(p) as ctx:
        pos, w, r = ctx.export_paths(bc, None, 500)
    pos64 = pos.astype(np.float64)
    seg = np.linalg.norm(np.diff(pos64, axis=1), axis=2)
    # rotations preserve segment lengths: every exported path keeps the initial curve's (the
    # reference bootstrapper, used for this N, places its points to within 1e-3 of ds, as the
    # reference's own curves do; the arc to ~1e-7)
    init = T.bootstrap_curve(p, bc).astype(np.float64)
    seg0 = np.linalg.norm(np.diff(init, axis=0), axis=1)
    assert np.allclose(seg, seg0[None, :], rtol=2e-6)
    assert np.allclose(seg0, float(F32(S) / F32(N)), rtol=1e-3)
    assert np.allclose(pos64[:, 0], (0, 0, 0)) and np.allclose(pos64[:, -1], (0, 0, 7), atol=2e-5)
    # the reference weigher on the exported geometry: every path within 1e-5 relative, plus the
    # weight jumps at the bin edges its curvatures lie near. The exported positions are the
    # chain's tangents times lengths summed in double and rounded to float (2^-24 of |x| <= 7
    # each), so the reference's curvatures from them differ from the chain's by up to ~5e-3 of a
    # bin here (a segment's two rounded ends move its unit tangent by up to 2 x 7 x 2^-24 / ds =
    # 2.4e-6, a curvature takes two tangents, and kscale = (bins - 1) / 2.02 ~ 1000 bins per
    # unit): an edge within 1e-2 bins of a curvature may flip.
    olut, meta = oracle.lut_f32(oracle.wparams(mu, eps, sc, ab, nst, bins), F32(S) / F32(N))
    ow, ov, ob, oc = oracle.weigh_f32(pos, N, S, olut, meta, absorption=ab, want_bins=True, want_curv=True)
    assert np.all(ov == 1)
    r_ = oc.astype(np.float64) / float(meta.step)
    near = np.abs(r_ - np.round(r_)) < 1e-2
    Lr = olut.astype(np.float64)
    below = Lr[:-1] + float(meta.step) * (Lr[1:] - Lr[:-1])
    jumps = np.concatenate([[0.0], np.abs(np.log10(Lr[1:]) - np.log10(below))])
    edge = np.clip(np.round(r_).astype(np.int64), 0, bins - 1)
    allowed = np.where(near, jumps[edge], 0.0).sum(axis=1)
    dev = np.abs(ow - w)
    assert np.all(dev <= 1e-5 * np.abs(ow) + allowed * (1 + 1e-6)), (dev - 1e-5 * np.abs(ow) - allowed).max()
    assert np.median(dev / np.abs(ow)) < 1e-6


# The differentiation configuration: N = 128 (and 130, the N the reference's bootstrapper
# resolves), S = 16, source (0,0,0) and receiver (8,0,0) with tangents (1,0,0), sigma = 0.1,
# mu_s = 10, 4096-bin tables and derivative tables, 2^22 paths (4096 chains x 1024 steps), sub-chains of
# k <= 32 rotated by U(-0.1, 0.1). The burn-in of 2000 steps lets the segments next to the
# receiver wander over many table bins (a segment there moves only when a rotated sub-chain
# ends at point N-1, about once in N - 33 steps): with the chains still near the initial
# curve, every path's last two curvatures sit at nearly the same place in the table and a
# finite difference of the estimate depends on where the bin edges fall (measured on the
# FP64 oracle: 0.5 % swings with the step), not on the derivative.
C4_RECEIVER = (8.0, 0.0, 0.0)
C4 = dict(mu=1.0, eps=0.01, scatter=10.0, num_steps_int=4000, num_curvature_steps=4096, lut_mode=T.LUT_FP64,
          perturb_seed=31, num_chains=4096, paths_to_generate=4096 * 1024, paths_to_skip=2000, max_sub_chain=32,
          max_angle=0.1)
# finite-difference steps: 1e-3 relative for mu_s and sigma; for the receiver 1e-3 of the
# source-receiver distance (0.064 ds)
H_REL = 1e-3
H_RECEIVER = 1e-3 * 8.0


def adjoint_setup(form=T.FORM_COMPENSATED, N=128, **kw):
    S = 16.0
    base = dict(C4, num_segments=N, form=form)
    base.update(kw)
    return T.default_params(**base), T.make_bc((0, 0, 0), (1, 0, 0), C4_RECEIVER, (1, 0, 0), S)


def run_log10(form, N=128, **kw):
    p, bc = adjoint_setup(form, N, **kw)
    with T.Context(p) as ctx:
        return ctx.run(bc).log10_weight


def richardson(f, step):
    """Central difference extrapolated from steps h and 2h: (4 D(h) - D(2h)) / 3."""
    d1 = (f(step) - f(-step)) / (2 * step)
    d2 = (f(2 * step) - f(-2 * step)) / (4 * step)
    return (4 * d1 - d2) / 3


def gpu_adjoint(N):
    p, bc = adjoint_setup(N=N)
    with T.Context(p) as ctx:
        fwd = ctx.run(bc)
        g = ctx.adjoint(bc, fwd)
    assert fwd.total_paths == 4096 * 1024 and fwd.failed_paths == 0
    return np.asarray(g), fwd


@pytest.mark.parametrize("N", [128, 130])
@pytest.mark.parametrize("form", [T.FORM_COMPENSATED, T.FORM_FP64])
def test_adjoint_mu_sigma_match_central_differences(form, N):
    g, _ = gpu_adjoint(N)
    mus, sigma = 10.0, 0.1
    fd_mu = (run_log10(form, N, scatter=mus * (1 + H_REL)) - run_log10(form, N, scatter=mus * (1 - H_REL))) / \
        (2 * H_REL * mus)
    fd_sig = (run_log10(form, N, eps=(sigma * (1 + H_REL)) ** 2) - run_log10(form, N, eps=(sigma * (1 - H_REL)) ** 2)) / \
        (2 * H_REL * sigma)
    assert abs(g[0] - fd_mu) < 1e-3 * abs(fd_mu), (g[0], fd_mu)
    assert abs(g[1] - fd_sig) < 1e-3 * abs(fd_sig), (g[1], fd_sig)


@pytest.mark.parametrize("N", [128, 130])
def test_adjoint_receiver_matches_central_differences(N):
    """d log10 W / d receiver against central differences of the FP64 form with the receiver
    moved when weighing (the chains held: the pathwise estimator's definition), common random
    numbers, within 1e-3 of the gradient's largest component."""
    g, _ = gpu_adjoint(N)
    fd = []
    for axis in range(3):
        def f(t, axis=axis):
            e = [0.0, 0.0, 0.0]
            e[axis] = t
            return run_log10(T.FORM_FP64, N, eval_end_shift=tuple(e))
        fd.append(richardson(f, H_RECEIVER))
    fd = np.array(fd)
    scale = np.abs(fd).max()
    assert np.all(np.abs(g[2:] - fd) < 1e-3 * scale), (g[2:], fd)


def test_adjoint_matches_fp64_cpu_finite_differences_of_the_reference_weighters(oracle):
    """All five gradient components against the oracle's FP64 CPU finite differences: the FP64
    twin of the reference's table build and weigher, rebuilt for mu_s and sigma +-h and
    re-weighed with the receiver moved, on the same Philox proposals, chain for chain."""
    N = 128
    g, fwd = gpu_adjoint(N)
    p, bc = adjoint_setup(N=N)
    init = T.bootstrap_curve(p, bc)
    fd = oracle.fd_gradient_f64(init, N, 16.0, C4["mu"], C4["eps"], C4["scatter"], 0.0, C4["num_steps_int"],
                                C4["num_curvature_steps"], seed=C4["perturb_seed"], n_chains=C4["num_chains"],
                                steps=1024, burn_in=C4["paths_to_skip"], k_max=C4["max_sub_chain"],
                                max_angle=C4["max_angle"], h=H_REL, h_receiver=H_RECEIVER)
    assert abs(g[0] - fd[0]) < 1e-3 * abs(fd[0]), (g[0], fd[0])
    assert abs(g[1] - fd[1]) < 1e-3 * abs(fd[1]), (g[1], fd[1])
    scale = np.abs(fd[2:]).max()
    assert np.all(np.abs(g[2:] - fd[2:]) < 1e-3 * scale), (g[2:], fd[2:])


@pytest.mark.parametrize("form", [T.FORM_COMPENSATED, T.FORM_PLAIN_FP32])
def test_weight_histogram_counts_the_exported_paths(form):
    """twisty_weight_histogram (the reference's histogram.txt) against the same pass's exported
    path weights binned on the host by the reference's rule (linear weight incl. normaliser,
    equal buckets, out-of-range weights in the end buckets)."""
    mu, eps, sc, ab, nst, bins, N, S = LUT_SETS["B"]
    chains, steps = 128, 40
    p = T.default_params(num_segments=N, form=form, perturb_seed=8, num_chains=chains, paths_to_generate=chains * steps,
                         paths_to_skip=10, mu=mu, eps=eps, scatter=sc, absorption=ab, num_steps_int=nst,
                         num_curvature_steps=bins, max_sub_chain=16, max_angle=0.3)
    bc = bc_for(N, S)
    with T.Context(p) as ctx:
        pos, w, r = ctx.export_paths(bc, None, chains * steps)
        lin = 10.0 ** (w + r.log10_normalizer)
        lo, hi = np.quantile(lin, 0.05), np.quantile(lin, 0.9)
        counts = ctx.weight_histogram(bc, lo, hi, 64)
    expect = np.zeros(64, np.uint64)
    for v in lin:
        b = 0 if v < lo else 63 if v > hi else min(int((v - lo) / (hi - lo) * 64), 63)
        expect[b] += 1
    assert counts.sum() == r.total_paths == w.size
    # bucket edges: a weight within rounding of an edge may land on either side of it
    assert np.abs(counts.astype(np.int64) - expect.astype(np.int64)).sum() <= 2
