"""Host-side checks of the C ABI that need no GPU: the library loads and exports every
entry point include/twisty_b200.h declares, config parsing follows the reference schema,
the bootstrapper and geometry checks, and the no-device error path."""
import ctypes as C
import json
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

import twisty_b200 as T
from twisty_b200 import _abi

HEADER = os.path.join(ROOT, "include", "twisty_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(twisty_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _abi.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    nm = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (twisty_\w+)", nm))
    assert set(names) <= exported
    # every ctypes signature matches a declared function and vice versa
    assert sorted(n for n, _, _ in _abi.SIGNATURES) == names


def test_struct_sizes_match_header(tmp_path):
    # compile a probe against the header and compare struct sizes with the ctypes mirror
    src = str(tmp_path / "abi_probe.c")
    with open(src, "w") as f:
        f.write('#include "twisty_b200.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(twisty_params), sizeof(twisty_bc),'
                ' sizeof(twisty_result), sizeof(twisty_lut_info), sizeof(twisty_experiment),'
                ' offsetof(twisty_params, eval_end_shift), offsetof(twisty_result, total_ms),'
                ' offsetof(twisty_params, fp64_check_chains), offsetof(twisty_result, fp64_rel_error)); return 0;}\n')
    exe = src[:-2]
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
    sizes = list(map(int, subprocess.run([exe], capture_output=True, text=True).stdout.split()))
    assert sizes == [C.sizeof(_abi.Params), C.sizeof(_abi.BC), C.sizeof(_abi.Result), C.sizeof(_abi.LutInfo),
                     C.sizeof(_abi.Experiment), _abi.Params.eval_end_shift.offset, _abi.Result.total_ms.offset,
                     _abi.Params.fp64_check_chains.offset, _abi.Result.fp64_rel_error.offset]


def test_params_init_reference_defaults():
    p = T.default_params()
    assert p.struct_size == C.sizeof(_abi.Params)
    # WeightingParameters member initialisers (Twisty/PathWeightUtils.h:35-48)
    assert (p.mu, p.num_steps_int, p.min_bound, p.max_bound, p.eps, p.bias, p.num_curvature_steps) == \
        (pytest.approx(0.1), 2000, 0.0, 100.0, pytest.approx(0.01), 1.0, 10000)
    assert p.max_sub_chain == 25 and p.max_angle == pytest.approx(np.pi)


def reference_config(**over):
    cfg = json.load(open(os.path.join(ROOT, "tests", "golden", "chain_66.json")))["config"]
    cfg["experiment"]["experimentParams"].update(over)
    return cfg


def test_config_json_and_yaml_agree():
    cfg = reference_config()
    ep, bc = T.ParseExperimentParamsFromConfig(json.dumps(cfg))
    assert ep.numSegmentsPerCurve == 66 and ep.numPathsToSkip == 1000
    assert ep.weightingParameters.maxBound == pytest.approx(10.0 / np.float32(0.01))
    lines = []

    def emit(d, ind):
        for k, v in d.items():
            if isinstance(v, dict):
                lines.append(" " * ind + f"{k}:")
                emit(v, ind + 2)
            elif isinstance(v, list):
                lines.append(" " * ind + f"{k}: [{', '.join(map(str, v))}]")
            else:
                lines.append(" " * ind + f"{k}: {json.dumps(v)}  # comment")
    emit(cfg, 0)
    ep2, bc2 = T.ParseExperimentParamsFromConfig("\n".join(lines), yaml=True)
    assert ep2 == ep and bc2 == bc


def test_config_normalises_directions_and_rejects_missing_keys():
    cfg = reference_config()
    cfg["experiment"]["basicExperiment"]["startDir"] = [2.0, 0.0, 0.0]
    ep, bc = T.ParseExperimentParamsFromConfig(cfg)
    assert bc.m_startDir == pytest.approx((1.0, 0.0, 0.0))
    del cfg["experiment"]["experimentParams"]["weighting"]["eps"]
    with pytest.raises(T.TwistyError) as e:
        T.ParseExperimentParamsFromConfig(cfg)
    assert e.value.status == _abi.ERR_INVALID_CONFIG
    with pytest.raises(T.TwistyError):
        T.ParseExperimentParamsFromConfig("{not json")


def test_config_b200_block():
    cfg = reference_config(b200={"form": 0, "maxSubChain": 32, "maxAngle": 0.05, "numChains": 4096})
    ep, _ = T.ParseExperimentParamsFromConfig(cfg)
    assert (ep.form, ep.maxSubChain, ep.numChains) == (0, 32, 4096) and ep.maxAngle == pytest.approx(0.05)


@pytest.mark.parametrize("N,S,end", [(4, 5.0, (3, 0, 0)), (64, 10.0, (8, 0, 0)), (256, 20.0, (0, 0, 12)),
                                     (257, 20.0, (0, 0, 12)), (1024, 40.0, (5, 5, 5)), (13, 3.0, (0, 0, 0))])
def test_bootstrap_any_n(N, S, end):
    d = (0, 0, 1) if end == (0, 0, 12) else (1, 0, 0)
    bc = T.make_bc((0, 0, 0), d, end, d, S)
    pos = T.bootstrap_curve(T.default_params(num_segments=N), bc).astype(np.float64)
    seg = np.linalg.norm(np.diff(pos, axis=0), axis=1)
    ds = np.float32(S) / np.float32(N)
    # positions are stored in float: each length is exact up to the rounding of its end points
    tol = 4 * np.abs(pos).max() * 2.0 ** -24
    assert np.all(np.abs(seg - ds) <= tol + 2e-7 * ds)
    assert np.allclose(pos[0], 0) and np.allclose(pos[-1], end, atol=1e-6)
    assert np.allclose(pos[1], np.array(d) * ds, atol=1e-6)


def test_bootstrap_infeasible():
    bc = T.make_bc((0, 0, 0), (1, 0, 0), (11, 0, 0), (1, 0, 0), 10.0)
    with pytest.raises(T.TwistyError) as e:
        T.bootstrap_curve(T.default_params(num_segments=64), bc)
    assert e.value.status == _abi.ERR_INFEASIBLE_GEOMETRY


def test_min_arclength_formula():
    # CalculateMinimumArclength (Twisty/PathGeneration.cpp:12-43) for straight ends
    bc = T.make_bc((0, 0, 0), (1, 0, 0), (8, 0, 0), (1, 0, 0), 10.0)
    assert T.min_arclength(bc, 64) == pytest.approx(8.0, rel=1e-6)


def test_no_device_is_an_error_not_a_fallback():
    if os.path.exists("/dev/nvidia0"):
        pytest.skip("a GPU is present")
    with pytest.raises(T.TwistyError) as e:
        T.Context(T.default_params(num_segments=8))
    assert e.value.status == _abi.ERR_NO_DEVICE


def test_autograd_binding_imports_without_a_gpu():
    """The torch binding is importable on a CPU host (it calls the library only when run)."""
    from twisty_b200 import autograd
    assert callable(autograd.experiment_log10_weight)
    assert issubclass(autograd.ExperimentLog10Weight, __import__("torch").autograd.Function)


def test_tuning_cache_roundtrip_and_rejects_bad_files(tmp_path):
    """The tuning cache file is host-side JSON: save, reload, and refuse malformed input."""
    import twisty_b200 as T
    good = tmp_path / "tune.json"
    good.write_text('{"entries": [{"device": "X", "n": 256, "bins": 8192, "group": 32, "spl": 8, '
                    '"warps": 32, "path_segments_per_s": 6.6e11}]}')
    T.tuning_cache_load(str(good))
    out = tmp_path / "out.json"
    T.tuning_cache_save(str(out))
    import json
    e = [x for x in json.loads(out.read_text())["entries"] if x["device"] == "X"]
    assert e == [{"device": "X", "n": 256, "bins": 8192, "group": 32, "spl": 8, "warps": 32,
                  "path_segments_per_s": 6.6e11}]
    bad_shape = tmp_path / "bad1.json"
    bad_shape.write_text('{"entries": [{"device": "X", "n": 256, "bins": 8192, "group": 7, "spl": 8, "warps": 32}]}')
    bad_json = tmp_path / "bad2.json"
    bad_json.write_text('{"entries": [ {"device": "X", "n": ')
    for f in (bad_shape, bad_json, tmp_path / "missing.json"):
        with pytest.raises(T.TwistyError):
            T.tuning_cache_load(str(f))


@pytest.mark.parametrize("N,S", [(10, 5.0), (18, 6.0), (34, 12.0), (66, 10.0)])
def test_reference_bootstrapper_bit_exact_with_reference(N, S):
    """bootstrap_kind 1 reproduces the reference's ResolveEvenNumberOfSegments curves (golden
    fixtures from the reference build, bootstrapSeed 7) bit for bit."""
    from conftest import GEOM
    g = GEOM[N]
    bc = T.make_bc(g[0], g[1], g[2], g[3], S)
    ref = np.load(os.path.join(ROOT, "tests", "golden", f"boot_{N}.npy"))
    for kind in (1, 0):   # auto picks the reference's bootstrapper for these N
        pos = T.bootstrap_curve(T.default_params(num_segments=N, bootstrap_seed=7, bootstrap_kind=kind), bc)
        assert pos.shape == ref.shape
        assert np.array_equal(pos.view(np.uint32), ref.view(np.uint32)), (kind, np.abs(pos - ref).max())


def test_reference_bootstrapper_refuses_other_n():
    bc = T.make_bc((0, 0, 0), (1, 0, 0), (8, 0, 0), (1, 0, 0), 10.0)
    with pytest.raises(T.TwistyError):
        T.bootstrap_curve(T.default_params(num_segments=64, bootstrap_kind=1), bc)   # N-2 = 62
    pos = T.bootstrap_curve(T.default_params(num_segments=64, bootstrap_kind=0), bc)   # auto: the arc
    seg = np.linalg.norm(np.diff(pos.astype(np.float64), axis=0), axis=1)
    assert np.allclose(seg, 10.0 / 64, rtol=1e-5)


def test_default_shape_covers_every_n_and_table_size():
    """twisty_default_shape (host-only): every N from 4 to 1024 has a shape that covers it, fits
    in shared memory with its table staged or through L1, and has a batched kernel except the
    one-lane 1 x 16 and 1 x 24 of long passes at N = 13..24 and 4 x 12 at N = 37..48 (batched
    runs take other 4-lane shapes there); tables of up to 4096 bins are staged, 100000-bin tables go through L1."""
    import twisty_b200 as T
    for bins in (256, 2048, 4096, 8192, 20000, 100000):
        for n in range(4, 1025):
            s = T.default_shape(n, bins)
            assert s["group"] * s["spl"] >= n, (n, bins, s)
            assert 1 <= s["warps"] and s["warps"] * 32 <= 1024, (n, bins, s)
            assert s["smem_bytes"] <= 227 * 1024, (n, bins, s)
            if 13 <= n <= 24:
                assert (s["group"], s["spl"], s["batched"]) == (1, 16 if n <= 16 else 24, 0), (n, bins, s)
            elif 37 <= n <= 48:
                assert (s["group"], s["spl"], s["batched"]) == (4, 12, 0), (n, bins, s)
            else:
                assert s["batched"] == 1, (n, bins, s)
            if bins <= 4096:
                assert s["table_in_l1"] == 0, (n, bins, s)
            if bins == 100000:
                assert s["table_in_l1"] == 1, (n, bins, s)
    # the benchmark's shape, and a shape that stages below its full warps
    s = T.default_shape(256, 8192)
    assert (s["group"], s["spl"], s["warps"], s["table_in_l1"]) == (16, 16, 24, 0)
    assert (T.default_shape(768, 4096)["warps"], T.default_shape(768, 4096)["table_in_l1"]) == (20, 0)
    assert (T.default_shape(768, 20000)["warps"], T.default_shape(768, 20000)["table_in_l1"]) == (24, 1)
    for n, bins in ((3, 4096), (1025, 4096), (256, 1)):
        with pytest.raises(T.TwistyError):
            T.default_shape(n, bins)


def test_benchmark_curve_fixture_is_the_bootstrappers():
    """bench.py's reference arm reads the N = 256 initial curve of the precision workload from a
    committed fixture (so that it never loads this library); it must be the curve this library's
    bootstrapper gives for that workload (arc bootstrapper, bootstrap seed 7)."""
    import bench
    pos = T.bootstrap_curve(T.default_params(num_segments=256, bootstrap_seed=7), bench.workload_bc(T))
    fix = np.load(bench.BENCH_CURVE)
    assert np.array_equal(pos.view(np.uint32), fix.view(np.uint32))


CALLER = r'''
// A caller of the reference's runner API, compiled against the drop-in header unchanged.
#include "twisty_b200_runner.hpp"
#include <cstdio>
#include <fstream>
#include <sstream>
using namespace twisty::b200;
int main(int, char **argv)
{
    std::ifstream f(argv[1]);
    std::stringstream buf;
    buf << f.rdbuf();
    BoundaryConditions bc;
    std::string err;
    ExperimentRunner::ExperimentParameters params = ExperimentRunner::ParseExperimentParamsFromConfig(buf.str(), false, &bc, &err);
    if (!err.empty()) { std::printf("parse error %s\n", err.c_str()); return 2; }
    std::printf("segments %u paths %llu skip %llu scatter %g eps %g bins %u end %g %g %g arclength %g\n",
                params.numSegmentsPerCurve, (unsigned long long)params.numPathsInExperiment,
                (unsigned long long)params.numPathsToSkip, params.weightingParameters.scatter,
                params.weightingParameters.eps, params.weightingParameters.numCurvatureSteps,
                bc.m_endPos.x, bc.m_endPos.y, bc.m_endPos.z, bc.arclength);
    FullExperimentRunnerOptimalPerturb runner(params);
    std::optional<ExperimentRunner::ExperimentResults> r = runner.RunExperiment(bc);
    if (!r) { std::printf("no results: %s\n", runner.lastError().c_str()); return 3; }
    std::printf("log10 %.17g paths %llu\n", r->experimentWeightLog10, (unsigned long long)r->totalPathsGenerated);
    return 0;
}
'''


def test_cpp_runner_header_compiles_for_a_reference_style_caller(tmp_path):
    """include/twisty_b200_runner.hpp, the C++ face of the drop-in: a caller written against the
    reference's runner API (ParseExperimentParamsFromConfig, FullExperimentRunnerOptimalPerturb,
    RunExperiment -> std::optional<ExperimentResults>) compiles warning-free and links against the
    library; without a GPU, RunExperiment returns no result and says why (no CPU fallback)."""
    src = tmp_path / "caller.cpp"
    src.write_text(CALLER)
    exe = tmp_path / "caller"
    lib_dir = os.path.dirname(_abi.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                    "-o", str(exe), "-L", lib_dir, "-ltwisty_b200", f"-Wl,-rpath,{lib_dir}"], check=True)
    cfg = tmp_path / "cfg.json"
    cfg.write_text(json.dumps(reference_config(pathsToGenerate=1000)))
    r = subprocess.run([str(exe), str(cfg)], capture_output=True, text=True, env={**os.environ, "CUDA_VISIBLE_DEVICES": ""})
    assert "segments 66 paths 1000 skip 1000 scatter 10 eps 0.01 bins 1024 end 8 0 0 arclength 10" in r.stdout, r.stdout
    if r.returncode == 3:
        assert "no CUDA device" in r.stdout
    else:   # a GPU is visible after all
        assert r.returncode == 0 and "paths 1000" in r.stdout


def test_reference_arm_loads_nothing_of_this_library():
    """bench.py's reference arm runs the reference's own loop (compiled from its sources into
    oracle/_ref) and must not load this library: a small run in a fresh process."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        pytest.skip("the reference build (make -C oracle ref) is absent")
    code = ("import sys; sys.path.insert(0, %r); import bench; "
            "v, ms, rec = bench.cpu_reference_run(20000, 2); "
            "assert rec['paths'] == 20000 and v > 0; "
            "assert 'twisty_b200' not in sys.modules, sorted(m for m in sys.modules if 'twisty' in m); print('ok')") % ROOT
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
