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
    # the reference weigher on the exported geometry agrees to 1e-5 (edge flips aside)
    olut, meta = oracle.lut_f32(oracle.wparams(mu, eps, sc, ab, nst, bins), F32(S) / F32(N))
    ow, ov, _, _ = oracle.weigh_f32(pos, N, S, olut, meta, absorption=ab, want_bins=False)
    rel = np.abs(ow - w) / np.abs(ow)
    assert np.median(rel) < 1e-6 and np.mean(rel < 1e-5) > 0.95


def adjoint_setup(form=T.FORM_COMPENSATED, **kw):
    N, S = 66, 10.0
    base = dict(num_segments=N, mu=1.0, eps=0.01, scatter=10.0, num_steps_int=4000, num_curvature_steps=4096,
                form=form, lut_mode=T.LUT_FP64, perturb_seed=31, num_chains=4096,
                paths_to_generate=4096 * 300, paths_to_skip=100, max_sub_chain=32, max_angle=0.1)
    base.update(kw)
    return T.default_params(**base), bc_for(N, S)


def run_log10(form, **kw):
    p, bc = adjoint_setup(form, **kw)
    with T.Context(p) as ctx:
        return ctx.run(bc).log10_weight


@pytest.mark.parametrize("form", [T.FORM_COMPENSATED, T.FORM_FP64])
def test_adjoint_mu_sigma_match_central_differences(form):
    p, bc = adjoint_setup()
    with T.Context(p) as ctx:
        fwd = ctx.run(bc)
        g = ctx.adjoint(bc, fwd)
    h = 1e-3
    mus, sigma = 10.0, 0.1
    fd_mu = (run_log10(form, scatter=mus * (1 + h)) - run_log10(form, scatter=mus * (1 - h))) / (2 * h * mus)
    fd_sig = (run_log10(form, eps=(sigma * (1 + h)) ** 2) - run_log10(form, eps=(sigma * (1 - h)) ** 2)) / (2 * h * sigma)
    assert abs(g[0] - fd_mu) < 1e-3 * abs(fd_mu), (g[0], fd_mu)
    assert abs(g[1] - fd_sig) < 1e-3 * abs(fd_sig), (g[1], fd_sig)


def test_adjoint_receiver_matches_central_differences():
    p, bc = adjoint_setup()
    with T.Context(p) as ctx:
        fwd = ctx.run(bc)
        g = ctx.adjoint(bc, fwd)
    ds = 10.0 / 66
    h = 1e-2 * ds
    fd = []
    for axis in range(3):
        e = np.zeros(3)
        e[axis] = h
        fd.append((run_log10(T.FORM_FP64, eval_end_shift=tuple(e)) - run_log10(T.FORM_FP64, eval_end_shift=tuple(-e)))
                  / (2 * h))
    fd = np.array(fd)
    scale = np.abs(fd).max()
    assert np.all(np.abs(g[2:] - fd) < 2e-2 * scale), (g[2:], fd)
