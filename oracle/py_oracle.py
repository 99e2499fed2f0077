"""ctypes loader for the CPU oracle (oracle/twisty_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py, as the checker. The product
package (twisty_b200) never imports this module.

Also wraps the reference harness (oracle/_ref/ref_harness, built from the reference's own
sources by oracle/Makefile) for the golden-vector generator.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_HARNESS = os.path.join(HERE, "_ref", "ref_harness")
REF_FULLEXPERIMENT = os.path.join(HERE, "_ref", "FullExperiment")


class WParams(C.Structure):
    _fields_ = [("mu", C.c_float), ("eps", C.c_float), ("scatter", C.c_float),
                ("absorption", C.c_float), ("min_bound", C.c_float), ("max_bound", C.c_float),
                ("bias", C.c_float), ("num_steps_int", C.c_uint32),
                ("num_curvature_steps", C.c_uint32)]


class LutMeta(C.Structure):
    _fields_ = [("min_k", C.c_float), ("max_k", C.c_float), ("step", C.c_float),
                ("min_w", C.c_float), ("max_w", C.c_float), ("ds", C.c_float),
                ("bins", C.c_uint32), ("pad", C.c_uint32)]


class LutMeta64(C.Structure):
    _fields_ = [("min_k", C.c_double), ("max_k", C.c_double), ("step", C.c_double),
                ("min_w", C.c_double), ("max_w", C.c_double), ("ds", C.c_double),
                ("bins", C.c_uint32), ("pad", C.c_uint32)]


class ChainOpts(C.Structure):
    _fields_ = [("has_shift", C.c_int), ("eval_shift", C.c_double * 3), ("ref_log10", C.c_double),
                ("grad_chains", C.c_void_p)]


class CW(C.Structure):
    _fields_ = [("max_log10", C.c_double), ("total", C.c_double), ("offset", C.c_double),
                ("n", C.c_uint32), ("pad", C.c_uint32)]


def build(force: bool = False) -> str:
    """Compile the oracle library with the committed recipe (gcc, no GPU needed)."""
    src = os.path.join(HERE, "twisty_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return LIB_PATH


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        L.tor_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.tor_draw_step.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.c_uint32, C.c_float, C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint32), C.POINTER(C.c_float)]
        L.tor_sincos_half.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.tor_wparams_default.argtypes = [C.POINTER(WParams), C.c_float, C.c_float, C.c_float,
                                          C.c_float, C.c_uint32, C.c_uint32]
        L.tor_lut_build_f32.argtypes = [C.POINTER(WParams), C.c_float, f32p, C.POINTER(LutMeta), C.c_int]
        L.tor_lut_build_f64.argtypes = [C.POINTER(WParams), C.c_double, f64p, C.POINTER(LutMeta64), C.c_int]
        L.tor_rotate_by_quat_f32.argtypes = [f32p, f32p]
        L.tor_weigh_paths_f32.argtypes = [f32p, C.c_uint64, C.c_uint32, C.c_float, f32p,
                                          C.POINTER(LutMeta), C.c_float, f64p, C.c_void_p,
                                          C.c_void_p, C.c_void_p]
        L.tor_weigh_paths_f64.argtypes = [f64p, C.c_uint64, C.c_uint32, C.c_double, f64p,
                                          C.POINTER(LutMeta64), C.c_double, f64p, C.c_void_p,
                                          C.c_void_p, C.c_void_p]
        L.tor_cw_reset.argtypes = [C.POINTER(CW)]
        L.tor_cw_add.argtypes = [C.POINTER(CW), C.c_double]
        L.tor_cw_combine.argtypes = [C.POINTER(CW), C.POINTER(CW), C.POINTER(CW)]
        L.tor_cw_extract_log10.argtypes = [C.POINTER(CW)]
        L.tor_cw_extract_log10.restype = C.c_double
        L.tor_log10_sum.argtypes = [f64p, C.c_uint64]
        L.tor_log10_sum.restype = C.c_double
        L.tor_norm_log10.argtypes = [C.c_int, C.c_float, f32p]
        L.tor_norm_log10.restype = C.c_double
        L.tor_run_chains_f32.argtypes = [f32p, C.c_uint32, C.c_float, f32p, C.POINTER(LutMeta),
                                         C.c_float, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                                         C.c_uint32, C.c_uint32, C.c_uint32, C.c_float,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_int]
        L.tor_run_chains_f64.argtypes = [f32p, C.c_uint32, C.c_double, f64p, C.POINTER(LutMeta64),
                                         C.c_double, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                                         C.c_uint32, C.c_uint32, C.c_uint32, C.c_float,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_int]
        L.tor_run_chains_f64_opts.argtypes = [f32p, C.c_uint32, C.c_double, f64p, C.POINTER(LutMeta64),
                                              C.c_double, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                                              C.c_uint32, C.c_uint32, C.c_uint32, C.c_float,
                                              C.c_void_p, C.c_void_p, C.POINTER(ChainOpts), C.c_int]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def philox(ctr, key):
    L = lib()
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    L.tor_philox4x32_10(c, k, o)
    return list(o)


def draw_step(seed, experiment, chain, step, n_segments, k_max, max_angle):
    k, left, ang = C.c_uint32(), C.c_uint32(), C.c_float()
    lib().tor_draw_step(seed, experiment, chain, step, n_segments, k_max, max_angle,
                        C.byref(k), C.byref(left), C.byref(ang))
    return k.value, left.value, ang.value


def sincos_half(angle):
    s, c = C.c_float(), C.c_float()
    lib().tor_sincos_half(angle, C.byref(s), C.byref(c))
    return s.value, c.value


def wparams(mu, eps, scatter, absorption, num_steps_int, bins) -> WParams:
    wp = WParams()
    lib().tor_wparams_default(C.byref(wp), mu, eps, scatter, absorption, num_steps_int, bins)
    return wp


def lut_f32(wp: WParams, ds: float, threads: int = os.cpu_count() or 1):
    lut = np.zeros(wp.num_curvature_steps, np.float32)
    meta = LutMeta()
    rc = lib().tor_lut_build_f32(C.byref(wp), ds, lut, C.byref(meta), threads)
    if rc != 0:
        raise ValueError("invalid LUT parameters")
    return lut, meta


def lut_f64(wp: WParams, ds: float, threads: int = os.cpu_count() or 1):
    lut = np.zeros(wp.num_curvature_steps, np.float64)
    meta = LutMeta64()
    rc = lib().tor_lut_build_f64(C.byref(wp), float(ds), lut, C.byref(meta), threads)
    if rc != 0:
        raise ValueError("invalid LUT parameters")
    return lut, meta


def rotate(q, v):
    q = np.ascontiguousarray(q, np.float32)
    v = np.array(v, np.float32)
    lib().tor_rotate_by_quat_f32(q, v)
    return v


def weigh_f32(pos, n_segments, arclength, lut, meta, absorption=0.0, want_bins=True, want_curv=False):
    pos = np.ascontiguousarray(pos, np.float32)
    P = pos.shape[0]
    w = np.zeros(P, np.float64)
    valid = np.zeros(P, np.uint8)
    bins = np.zeros((P, n_segments - 1), np.int32) if want_bins else None
    curv = np.zeros((P, n_segments - 1), np.float32) if want_curv else None
    lib().tor_weigh_paths_f32(pos, P, n_segments, arclength, lut, C.byref(meta), absorption, w,
                              _ptr(valid), _ptr(bins), _ptr(curv))
    return w, valid, bins, curv


def weigh_f64(pos, n_segments, arclength, lut, meta, absorption=0.0, want_bins=False):
    pos = np.ascontiguousarray(pos, np.float64)
    P = pos.shape[0]
    w = np.zeros(P, np.float64)
    valid = np.zeros(P, np.uint8)
    bins = np.zeros((P, n_segments - 1), np.int32) if want_bins else None
    lib().tor_weigh_paths_f64(pos, P, n_segments, arclength, lut, C.byref(meta), absorption, w,
                              _ptr(valid), _ptr(bins), None)
    return w, valid, bins


def cw_run(values, split):
    L = lib()
    a, b, c = CW(), CW(), CW()
    L.tor_cw_reset(C.byref(a))
    L.tor_cw_reset(C.byref(b))
    for i, v in enumerate(values):
        L.tor_cw_add(C.byref(a if i < split else b), float(v))
    L.tor_cw_combine(C.byref(a), C.byref(b), C.byref(c))
    return a, b, c, [L.tor_cw_extract_log10(C.byref(x)) for x in (a, b, c)]


def log10_sum(v):
    v = np.ascontiguousarray(v, np.float64)
    return lib().tor_log10_sum(v, v.size)


def norm_log10(n_segments, ds, bc12):
    return lib().tor_norm_log10(n_segments, ds, np.ascontiguousarray(bc12, np.float32))


def run_chains(init_pos, n_segments, arclength, lut, meta, *, seed, n_chains, steps, burn_in=0,
               k_max=25, max_angle=float(np.float32(np.pi)), experiment=0, chain0=0,
               absorption=0.0, want_paths=False, want_final=False, f64=False,
               threads=os.cpu_count() or 1):
    """Run Philox-driven chains in reference FP32 semantics (or the FP64 twin)."""
    init_pos = np.ascontiguousarray(init_pos, np.float32).reshape(-1)
    npath = n_chains * steps
    pl = np.zeros(npath, np.float64) if want_paths else None
    pv = np.zeros(npath, np.uint8) if want_paths else None
    cl = np.zeros(n_chains, np.float64)
    cv = np.zeros(n_chains, np.uint64)
    fp = (np.zeros((n_chains, n_segments + 1, 3), np.float64 if f64 else np.float32)
          if want_final else None)
    fn = lib().tor_run_chains_f64 if f64 else lib().tor_run_chains_f32
    rc = fn(init_pos, n_segments, arclength, lut, C.byref(meta), absorption, seed, experiment,
            chain0, n_chains, steps, burn_in, k_max, max_angle, _ptr(pl), _ptr(pv), _ptr(cl),
            _ptr(cv), _ptr(fp), threads)
    if rc != 0:
        raise ValueError("invalid chain parameters")
    return {"path_log10": pl, "path_valid": pv, "chain_log10": cl, "chain_valid": cv,
            "final_pos": fp}


def run_chains_f64_opts(init_pos, n_segments, arclength, lut, meta, *, seed, n_chains, steps, burn_in=0, k_max=25,
                        max_angle=float(np.float32(np.pi)), experiment=0, chain0=0, absorption=0.0,
                        eval_shift=None, grad_ref_log10=None, threads=os.cpu_count() or 1):
    """FP64 twin chains with the receiver moved when weighing (eval_shift) and/or the pathwise
    receiver gradient (grad_ref_log10: the reference the path weights are scaled by).
    Returns log10 of the summed weights and, with a gradient, d log10 W / d receiver (3)."""
    init_pos = np.ascontiguousarray(init_pos, np.float32).reshape(-1)
    cl = np.zeros(n_chains, np.float64)
    cv = np.zeros(n_chains, np.uint64)
    o = ChainOpts()
    if eval_shift is not None:
        o.has_shift = 1
        for q in range(3):
            o.eval_shift[q] = float(eval_shift[q])
    g = None
    if grad_ref_log10 is not None:
        g = np.zeros((n_chains, 4), np.float64)
        o.ref_log10 = float(grad_ref_log10)
        o.grad_chains = g.ctypes.data_as(C.c_void_p).value
    rc = lib().tor_run_chains_f64_opts(init_pos, n_segments, arclength, lut, C.byref(meta), absorption, seed,
                                       experiment, chain0, n_chains, steps, burn_in, k_max, max_angle,
                                       _ptr(cl), _ptr(cv), C.byref(o), threads)
    if rc != 0:
        raise ValueError("invalid chain parameters")
    out = {"log10": log10_sum(cl), "valid": int(cv.sum())}
    if g is not None:
        tot = g.sum(axis=0)
        out["grad_receiver"] = tot[:3] / tot[3]
    return out


def fd_gradient_f64(init_pos, n_segments, arclength, mu, eps, scatter, absorption, num_steps_int, bins, *, seed,
                    n_chains, steps, burn_in, k_max, max_angle, h=1e-3, h_receiver=None, richardson=True,
                    threads=os.cpu_count() or 1):
    """FP64 CPU central finite differences of log10 experimentWeight with respect to
    (mu_s, sigma, receiver x, y, z): the FP64 twin of the reference's table build
    (PathWeightUtils.cpp:281-433, maxBound = 10/eps) and weigher (PathWeighters.cpp:27-104)
    re-run with common random numbers (the same Philox proposals). mu_s and sigma = sqrt(eps)
    move by h relative; the receiver by h_receiver (absolute) along each axis, the chain held.
    With richardson, each difference is extrapolated from steps h and 2h,
    (4 D(h) - D(2h)) / 3, which cancels the O(h^2) term of the central difference."""
    ds = float(np.float32(arclength) / np.float32(n_segments))

    def table(mus, e):
        wp = wparams(mu, e, mus, absorption, num_steps_int, bins)
        return lut_f64(wp, ds, threads)

    def run(tab, shift=None):
        lut, meta = tab
        return run_chains_f64_opts(init_pos, n_segments, arclength, lut, meta, seed=seed, n_chains=n_chains,
                                   steps=steps, burn_in=burn_in, k_max=k_max, max_angle=max_angle,
                                   absorption=absorption, eval_shift=shift, threads=threads)["log10"]

    def central(f, x, step):
        d1 = (f(x + step) - f(x - step)) / (2 * step)
        if not richardson:
            return d1
        d2 = (f(x + 2 * step) - f(x - 2 * step)) / (4 * step)
        return (4 * d1 - d2) / 3

    sigma = float(np.sqrt(np.float64(np.float32(eps))))
    base = table(scatter, eps)
    g_mu = central(lambda m: run(table(float(np.float32(m)), eps)), scatter, h * scatter)
    g_sig = central(lambda sg: run(table(scatter, float(np.float32(sg) * np.float32(sg)))), sigma, h * sigma)
    hr = h_receiver if h_receiver is not None else 1e-2 * ds
    g_rx = []
    for axis in range(3):
        def f(t, axis=axis):
            e = np.zeros(3)
            e[axis] = t
            return run(base, e)
        g_rx.append(central(f, 0.0, hr))
    return np.array([g_mu, g_sig, *g_rx])
