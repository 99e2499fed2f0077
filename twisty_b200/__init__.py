"""twisty_b200 -- B200-native path-integral Monte Carlo runner (Python binding of the C ABI).

The product is the CUDA library ``libtwisty_b200.so`` behind the C ABI in
``include/twisty_b200.h``; this package binds it with ctypes for Python callers, tests and
the benchmark. The runner classes mirror the reference's experiment-runner API
(Twisty/ExperimentRunner.h:29-131): ``ExperimentParameters``, ``BoundaryConditions``,
``ParseExperimentParamsFromConfig``, ``FullExperimentRunnerOptimalPerturb`` (and the
``_GPU`` name of the reference's CUDA runner) with ``RunExperiment(bc)`` returning
``ExperimentResults`` -- weights as log10 values, since they overflow double.

There is no CPU fallback: every call goes to the device through the library, and a
missing library or device raises.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _abi
from ._abi import (FORM_COMPENSATED, FORM_FP64, FORM_PLAIN_FP32, LUT_EXTERNAL, LUT_FAITHFUL, LUT_MULTI_DS,
                   LUT_FP64, TABLE_EXACT_BLEND, TABLE_FIXED_NARROW, TABLE_FIXED_WIDE, TABLE_NONE)

__all__ = [
    "TwistyError", "Context", "ExperimentParameters", "BoundaryConditions", "ExperimentResults",
    "ParseExperimentParamsFromConfig", "FullExperimentRunnerOptimalPerturb",
    "FullExperimentRunnerOptimalPerturbOptimized_GPU", "FORM_PLAIN_FP32", "FORM_COMPENSATED",
    "FORM_FP64", "LUT_FAITHFUL", "LUT_FP64", "LUT_EXTERNAL", "TABLE_FIXED_NARROW", "TABLE_FIXED_WIDE",
    "TABLE_EXACT_BLEND", "TABLE_NONE", "default_params", "make_bc",
]


class TwistyError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        name = _abi.load().twisty_status_string(status).decode()
        super().__init__(f"{name}: {message}" if message else name)


def _lib():
    return _abi.load()


def _check(status: int, ctx=None):
    if status != _abi.OK:
        msg = _lib().twisty_last_error(ctx)
        raise TwistyError(status, msg.decode() if msg else "")


def _fptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def default_params(**kw) -> _abi.Params:
    """twisty_params with the reference defaults, then the given fields set."""
    p = _abi.Params()
    _lib().twisty_params_init(C.byref(p))
    for k, v in kw.items():
        if k == "eval_end_shift":
            p.eval_end_shift = _abi.Vec3(*v)
        else:
            setattr(p, k, v)
    if "eps" in kw and "max_bound" not in kw:
        p.max_bound = float(np.float32(10.0) / np.float32(kw["eps"]))
    return p


def make_bc(start_pos, start_dir, end_pos, end_dir, arclength) -> _abi.BC:
    def unit(v):
        v = np.asarray(v, np.float32)
        return v * (np.float32(1.0) / np.sqrt(np.float32(v @ v)))
    return _abi.BC(_abi.Vec3(*map(float, start_pos)), _abi.Vec3(*map(float, unit(start_dir))),
                   _abi.Vec3(*map(float, end_pos)), _abi.Vec3(*map(float, unit(end_dir))), float(arclength))


def make_experiment(bc: _abi.BC, num_segments: int, scatter: float, eps: float, paths: int) -> _abi.Experiment:
    """One entry of a batch (twisty_experiment): its own geometry, N, mu_s and phase eps."""
    return _abi.Experiment(bc, int(num_segments), float(scatter), float(eps), int(paths))


class Context:
    """One runner context (twisty_create / twisty_destroy)."""

    def __init__(self, params: _abi.Params):
        self.params = params
        h = C.c_void_p()
        _check(_lib().twisty_create(C.byref(params), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib().twisty_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def update(self, **kw):
        for k, v in kw.items():
            if k == "eval_end_shift":
                self.params.eval_end_shift = _abi.Vec3(*v)
            else:
                setattr(self.params, k, v)
        if "eps" in kw and "max_bound" not in kw:
            self.params.max_bound = float(np.float32(10.0) / np.float32(kw["eps"]))
        _check(_lib().twisty_update_params(self._h, C.byref(self.params)), self._h)

    def set_params(self, params: _abi.Params):
        """Replace the parameters (twisty_update_params); the next run builds its tables again."""
        self.params = params
        _check(_lib().twisty_update_params(self._h, C.byref(self.params)), self._h)

    def run(self, bc: _abi.BC) -> _abi.Result:
        r = _abi.Result()
        _check(_lib().twisty_run(self._h, C.byref(bc), C.byref(r)), self._h)
        return r

    def chain_results(self, n_chains: int):
        """Per-chain log10 sums (normaliser applied) and valid-path counts of the last pass."""
        lw = np.zeros(n_chains, np.float64)
        v = np.zeros(n_chains, np.uint64)
        _check(_lib().twisty_chain_results(self._h, _fptr(lw), _fptr(v), n_chains), self._h)
        return lw, v

    def weight_histogram(self, bc: _abi.BC, min_weight: float = 4.69653e-16, max_weight: float = 1.17517e-13,
                         n_buckets: int = 500) -> np.ndarray:
        """The reference's path-weight histogram (its defaults: 500 buckets over the range of
        five-segment paths); counts per bucket."""
        c = np.zeros(n_buckets, np.uint64)
        _check(_lib().twisty_weight_histogram(self._h, C.byref(bc), float(min_weight), float(max_weight), n_buckets,
                                              _fptr(c)), self._h)
        return c

    def run_msegment(self, bc: _abi.BC) -> _abi.Result:
        """Independent-sample M-segment MC: paths_to_generate fresh bootstrap curves, mean weight."""
        r = _abi.Result()
        _check(_lib().twisty_run_msegment(self._h, C.byref(bc), C.byref(r)), self._h)
        return r

    def prepare(self, bc: _abi.BC):
        _check(_lib().twisty_prepare(self._h, C.byref(bc)), self._h)

    def launch(self, stream: int = 0):
        _check(_lib().twisty_launch(self._h, C.c_void_p(stream) if stream else None), self._h)

    def collect(self) -> _abi.Result:
        r = _abi.Result()
        _check(_lib().twisty_collect(self._h, C.byref(r)), self._h)
        return r

    def kernels_per_launch(self) -> int:
        return int(_lib().twisty_launch_kernel_count(self._h))

    def weight_paths(self, bc: _abi.BC, pos: np.ndarray, form: int = FORM_PLAIN_FP32, want_bins: bool = False):
        pos = np.ascontiguousarray(pos, np.float32)
        P = pos.shape[0]
        N = self.params.num_segments
        assert pos.shape[1:] == (N + 1, 3)
        w = np.zeros(P, np.float64)
        v = np.zeros(P, np.uint8)
        b = np.zeros((P, N - 1), np.int32) if want_bins else None
        _check(_lib().twisty_weight_paths(self._h, C.byref(bc), _fptr(pos), P, form, _fptr(w), _fptr(v), _fptr(b)),
               self._h)
        return w, v, b

    def build_lut(self, ds: float):
        n = self.params.num_curvature_steps
        lut = np.zeros(n, np.float32)
        info = _abi.LutInfo()
        _check(_lib().twisty_build_lut(self._h, float(ds), _fptr(lut), C.byref(info)), self._h)
        return lut, info

    def set_lut(self, lut: np.ndarray, info: _abi.LutInfo):
        lut = np.ascontiguousarray(lut, np.float32)
        info.bins = lut.size
        _check(_lib().twisty_set_lut(self._h, _fptr(lut), C.byref(info)), self._h)
        self.params.lut_mode = LUT_EXTERNAL
        self.params.num_curvature_steps = lut.size

    def normalizer_log10(self, n: int, ds: float, bc: _abi.BC) -> float:
        out = C.c_double()
        _check(_lib().twisty_normalizer_log10(self._h, n, float(ds), C.byref(bc), C.byref(out)), self._h)
        return out.value

    def set_initial_curve(self, pos: Optional[np.ndarray]):
        if pos is None:
            _check(_lib().twisty_set_initial_curve(self._h, None, 0), self._h)
            return
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        self._curve = pos
        _check(_lib().twisty_set_initial_curve(self._h, _fptr(pos), pos.shape[0]), self._h)

    def export_paths(self, bc: _abi.BC, directory: Optional[str], max_paths: int):
        N = self.params.num_segments
        pos = np.zeros((max_paths, N + 1, 3), np.float32)
        w = np.zeros(max_paths, np.float64)
        n = C.c_uint64()
        r = _abi.Result()
        d = directory.encode() if directory else None
        _check(_lib().twisty_export_paths(self._h, C.byref(bc), d, max_paths, _fptr(pos), _fptr(w), C.byref(n),
                                          C.byref(r)), self._h)
        return pos[: n.value], w[: n.value], r

    def adjoint(self, bc: _abi.BC, fwd: _abi.Result) -> np.ndarray:
        g = (C.c_double * 5)()
        _check(_lib().twisty_adjoint(self._h, C.byref(bc), C.byref(fwd), g), self._h)
        return np.array(list(g))

    def multi_ds_tables(self, min_ds: float, max_ds: float, n_ds: int, cache_path: Optional[str] = None):
        """Build (or load from cache_path) the multi-arclength table set used by lut_mode LUT_MULTI_DS."""
        _check(_lib().twisty_multi_ds_tables(self._h, float(min_ds), float(max_ds), int(n_ds),
                                             cache_path.encode() if cache_path else None), self._h)

    def autotune(self, bc: _abi.BC, trial_paths: int = 0) -> dict:
        """Time every compensated-form kernel shape for this context's N; the fastest is
        recorded in the process-wide tuning cache and used by later passes."""
        t = _abi.Tuning()
        _check(_lib().twisty_autotune(self._h, C.byref(bc), int(trial_paths), C.byref(t)), self._h)
        return {f: getattr(t, f) for f, _ in _abi.Tuning._fields_}

    def adjoint_batch(self, experiments: Sequence[_abi.Experiment]):
        """Forward pass of the batch and the adjoint replay of its chains (twisty_adjoint_batch):
        (results, grad[n, 5] = d log10 W_e / d (mu_s, sigma, receiver xyz), total[3] =
        (log10 sum W_e, d/d mu_s, d/d sigma of it for a shared mu_s and sigma), timing_ms[2])."""
        n = len(experiments)
        arr = (_abi.Experiment * n)(*experiments)
        res = (_abi.Result * n)()
        grad = np.zeros((n, 5), np.float64)
        total = (C.c_double * 3)()
        timing = (C.c_double * 2)()
        _check(_lib().twisty_adjoint_batch(self._h, arr, n, res, grad.ctypes.data_as(C.POINTER(C.c_double)), total,
                                           timing), self._h)
        return list(res), grad, np.array(list(total)), np.array(list(timing))

    def run_batch(self, experiments: Sequence[_abi.Experiment], iterations: int = 1):
        n = len(experiments)
        arr = (_abi.Experiment * n)(*experiments)
        res = (_abi.Result * n)()
        _check(_lib().twisty_run_batch(self._h, arr, n, iterations, res), self._h)
        return list(res)


def tuning_cache_save(path: str):
    """Write the process-wide tuning cache (shapes found by Context.autotune) as JSON."""
    _check(_lib().twisty_tuning_cache_save(path.encode()))


def tuning_cache_load(path: str):
    """Merge a JSON tuning cache into the process-wide one."""
    _check(_lib().twisty_tuning_cache_load(path.encode()))


def default_shape(num_segments: int, bins: int) -> dict:
    """The kernel shape and table placement a compensated forward pass of N segments with a
    bins-bin table takes with the shape knobs at zero (twisty_default_shape; no device needed)."""
    s = _abi.Shape()
    _check(_lib().twisty_default_shape(int(num_segments), int(bins), C.byref(s)))
    return {k: int(getattr(s, k)) for k, _ in _abi.Shape._fields_}


def bootstrap_curve(params: _abi.Params, bc: _abi.BC) -> np.ndarray:
    pos = np.zeros((params.num_segments + 1, 3), np.float32)
    _check(_lib().twisty_bootstrap_curve(C.byref(params), C.byref(bc), _fptr(pos)))
    return pos


def min_arclength(bc: _abi.BC, n: int) -> float:
    return float(_lib().twisty_min_arclength(C.byref(bc), n))


# --------------------------------------------------------------------------------------
# Mirror of the reference's runner API (Twisty/ExperimentRunner.h)
# --------------------------------------------------------------------------------------
@dataclass
class WeightingParameters:
    """Twisty/PathWeightUtils.h:35-48."""
    mu: float = 0.1
    numStepsInt: int = 2000
    minBound: float = 0.0
    maxBound: float = 100.0
    eps: float = 0.01
    bias: float = 1.0
    scatter: float = 0.0
    absorption: float = 0.0
    numCurvatureSteps: int = 10000
    weightingMethod: int = 0


@dataclass
class ExperimentParameters:
    """Twisty/ExperimentRunner.h:42-68 (plus the B200 knobs)."""
    numPathsInExperiment: int = 0
    numPathsToSkip: int = 0
    numSegmentsPerCurve: int = 4
    bootstrapSeed: int = 0
    curvePurturbSeed: int = 0
    weightingParameters: WeightingParameters = field(default_factory=WeightingParameters)
    perturbMethod: int = 0
    maxPerturbThreads: int = 0
    useGpu: bool = True
    experimentName: str = "Default_Experiment"
    experimentDirPath: str = "./Default_Experiment/"
    # B200
    form: int = FORM_COMPENSATED
    lutMode: int = LUT_FP64
    maxSubChain: int = 25
    maxAngle: float = float(np.float32(math.pi))
    numChains: int = 0
    device: int = 0

    def to_c(self) -> _abi.Params:
        w = self.weightingParameters
        return default_params(
            paths_to_generate=int(self.numPathsInExperiment), paths_to_skip=int(self.numPathsToSkip),
            num_segments=int(self.numSegmentsPerCurve), bootstrap_seed=int(self.bootstrapSeed) & 0xFFFFFFFF,
            perturb_seed=int(self.curvePurturbSeed) & 0xFFFFFFFF, weight_function=int(w.weightingMethod),
            perturb_method=int(self.perturbMethod), mu=w.mu, eps=w.eps, scatter=w.scatter,
            absorption=w.absorption, num_steps_int=int(w.numStepsInt),
            num_curvature_steps=int(w.numCurvatureSteps), min_bound=w.minBound, max_bound=w.maxBound,
            bias=w.bias, form=int(self.form), lut_mode=int(self.lutMode),
            max_sub_chain=int(self.maxSubChain), max_angle=float(self.maxAngle),
            num_chains=int(self.numChains), device=int(self.device))


@dataclass
class BoundaryConditions:
    """PerturbUtils::BoundaryConditions (Twisty/CurvePerturbUtils.h:62-68)."""
    m_startPos: Sequence[float] = (0.0, 0.0, 0.0)
    m_startDir: Sequence[float] = (1.0, 0.0, 0.0)
    m_endPos: Sequence[float] = (0.0, 0.0, 0.0)
    m_endDir: Sequence[float] = (1.0, 0.0, 0.0)
    arclength: float = 0.0

    def to_c(self) -> _abi.BC:
        return make_bc(self.m_startPos, self.m_startDir, self.m_endPos, self.m_endDir, self.arclength)


@dataclass
class ExperimentResults:
    """ExperimentRunner::ExperimentResults (Twisty/ExperimentRunner.h:73-82), weights in log10."""
    experimentWeightLog10: float
    totalPathsGenerated: int
    numFailedPaths: int
    totalExperimentMs: float
    setupExperimentMs: float
    perturbExperimentMs: float
    weightingExperimentMs: float
    normalizerLog10: float = 0.0
    relStdError: float = float("nan")
    clampedCurvatures: int = 0
    weightErrorBoundLog10: float = 0.0    # per-path log10 error bound of the arithmetic vs FP64
    fp64RelError: float = float("nan")     # measured on the fp64_check_chains chains (NaN: off)

    @property
    def avgPathWeightLog10(self) -> float:
        return self.experimentWeightLog10 - math.log10(max(self.totalPathsGenerated, 1))


def ParseExperimentParamsFromConfig(config, yaml: bool = False):
    """ExperimentRunner::ParseExperimentParamsFromConfig (Twisty/ExperimentRunner.cpp:48-177).

    `config` is JSON (or YAML) text or a dict; returns (ExperimentParameters, BoundaryConditions).
    """
    import json as _json
    text = config if isinstance(config, str) else _json.dumps(config)
    p = _abi.Params()
    bc = _abi.BC()
    status = _lib().twisty_params_from_config(text.encode(), 1 if yaml else 0, C.byref(p), C.byref(bc))
    _check(status)
    w = WeightingParameters(mu=p.mu, numStepsInt=p.num_steps_int, minBound=p.min_bound, maxBound=p.max_bound,
                            eps=p.eps, bias=p.bias, scatter=p.scatter, absorption=p.absorption,
                            numCurvatureSteps=p.num_curvature_steps, weightingMethod=p.weight_function)
    ep = ExperimentParameters(numPathsInExperiment=p.paths_to_generate, numPathsToSkip=p.paths_to_skip,
                              numSegmentsPerCurve=p.num_segments, bootstrapSeed=p.bootstrap_seed,
                              curvePurturbSeed=p.perturb_seed, weightingParameters=w,
                              perturbMethod=p.perturb_method, form=p.form, lutMode=p.lut_mode,
                              maxSubChain=p.max_sub_chain, maxAngle=p.max_angle, numChains=p.num_chains,
                              device=p.device)
    b = BoundaryConditions((bc.start_pos.x, bc.start_pos.y, bc.start_pos.z),
                           (bc.start_dir.x, bc.start_dir.y, bc.start_dir.z),
                           (bc.end_pos.x, bc.end_pos.y, bc.end_pos.z),
                           (bc.end_dir.x, bc.end_dir.y, bc.end_dir.z), bc.arclength)
    return ep, b


class FullExperimentRunnerOptimalPerturb:
    """Drop-in for the reference's runner (Twisty/FullExperimentRunnerOptimalPerturb.h:26-74)."""

    default_form = FORM_COMPENSATED

    def __init__(self, experimentParams: ExperimentParameters):
        self.m_experimentParams = experimentParams
        self._ctx: Optional[Context] = None

    def _context(self) -> Context:
        p = self.m_experimentParams.to_c()
        if self._ctx is None:
            self._ctx = Context(p)
        else:
            self._ctx.params = p
            _check(_lib().twisty_update_params(self._ctx.handle, C.byref(p)), self._ctx.handle)
        return self._ctx

    def RunExperiment(self, boundaryConditions: BoundaryConditions) -> Optional[ExperimentResults]:
        r = self._context().run(boundaryConditions.to_c())
        return ExperimentResults(r.log10_weight, r.total_paths, r.failed_paths, r.total_ms, r.setup_ms,
                                 r.perturb_ms, r.weighting_ms, r.log10_normalizer, r.rel_std_error,
                                 r.clamped_curvatures, r.weight_error_bound, r.fp64_rel_error)

    run_experiment = RunExperiment


class FullExperimentRunnerOptimalPerturbOptimized_GPU(FullExperimentRunnerOptimalPerturb):
    """The reference's CUDA runner name; the same B200 runner."""


def measure_fp32_peak(device: int = 0) -> float:
    """The device's FP32 issue rate, lane-level FMA instructions per second
    (twisty_measure_fp32_peak): the denominator of the chain kernels' roofline."""
    v = C.c_double()
    _check(_lib().twisty_measure_fp32_peak(int(device), C.byref(v)))
    return float(v.value)
