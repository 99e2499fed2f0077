"""The CPU oracle against the reference's own outputs (golden fixtures, tests/golden)."""
import numpy as np
import pytest

from conftest import LUT_SETS, golden_json, golden_npz

F32 = np.float32


def test_philox_known_answers(oracle):
    # Random123 known-answer vectors for philox4x32-10
    assert oracle.philox([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert oracle.philox([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert oracle.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_sincos_half_accuracy(oracle):
    for a in np.linspace(-np.pi, np.pi, 997).astype(F32):
        s, c = oracle.sincos_half(float(a))
        assert abs(s - np.sin(np.float64(a) / 2)) < 1.5e-7
        assert abs(c - np.cos(np.float64(a) / 2)) < 1.5e-7


def test_draw_step_ranges(oracle):
    N, kmax = 20, 25
    ks, lefts, angs = [], [], []
    for s in range(4000):
        k, left, ang = oracle.draw_step(99, 0, 3, s, N, kmax, float(F32(np.pi)))
        ks.append(k)
        lefts.append(left)
        angs.append(ang)
        assert 2 <= k <= N - 2 and 1 <= left <= N - k - 1
        assert -np.pi < ang < np.pi
    assert set(ks) == set(range(2, N - 1))            # every k in U{2..min(k_max, N-2)}
    assert min(lefts) == 1


@pytest.mark.parametrize("name", sorted(LUT_SETS))
def test_lut_bit_exact(oracle, name):
    g = golden_npz(f"lut_{name}.npz")
    mu, eps, sc, ab, nst, bins, N, S = LUT_SETS[name]
    lut, meta = oracle.lut_f32(oracle.wparams(mu, eps, sc, ab, nst, bins), F32(S) / F32(N))
    assert np.array_equal(lut.view(np.uint32), g["lut"].view(np.uint32))
    hdr = np.array([meta.min_k, meta.max_k, meta.step, meta.min_w, meta.max_w, meta.ds], F32)
    assert np.array_equal(hdr.view(np.uint32), g["hdr"].view(np.uint32))


@pytest.mark.parametrize("name", sorted(LUT_SETS))
def test_weigher_bit_exact(oracle, name):
    g = golden_npz(f"lut_{name}.npz")
    p = golden_npz(f"paths_{name}.npz")
    mu, eps, sc, ab, nst, bins, N, S = LUT_SETS[name]
    lut, meta = oracle.lut_f32(oracle.wparams(mu, eps, sc, ab, nst, bins), F32(S) / F32(N))
    w, valid, b, curv = oracle.weigh_f32(p["pos"], N, S, lut, meta, absorption=ab, want_curv=True)
    assert np.array_equal(valid, p["valid"])
    assert np.array_equal(w, p["log10w"])
    assert np.array_equal(curv.view(np.uint32), p["curv"].view(np.uint32))
    assert np.array_equal(b, p["bins"])
    # the straight path (last) has every curvature 0 up to the rounding of its unit tangents
    # (x (1/sqrtf(x x)) need not be exactly 1), and bin 0
    assert np.all(p["curv"][-1] < 1e-5) and np.all(p["bins"][-1] == 0)


def test_rotation_bit_exact(oracle):
    g = golden_npz("rotate.npz")
    out = np.stack([oracle.rotate(q, v) for q, v in zip(g["q"], g["v"])])
    assert np.array_equal(out.view(np.uint32), g["out"].view(np.uint32))


def test_combined_weights_bit_exact(oracle):
    for rec in golden_json("cw.json"):
        a, b, c, ex = oracle.cw_run(rec["values"], rec["split"])
        for mine, ref in zip((a, b, c), rec["cw"]):
            assert [mine.max_log10, mine.total, mine.offset, mine.n] == ref
        assert ex == rec["extract_log10"]


def test_normalizer_k4(oracle):
    for rec in golden_json("norm.json"):
        if rec["N"] != 4:
            continue
        got = oracle.norm_log10(4, rec["ds"], np.array(rec["bc"], F32))
        assert got == pytest.approx(rec["log10"], rel=1e-15, abs=1e-15)
