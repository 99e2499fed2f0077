"""The drop-in CLI (twisty_b200/twisty_full_experiment, the reference's
Experiments/FullExperiment.cpp driver rebuilt over include/twisty_b200_runner.hpp) on a
reference configuration: it writes Results.dat under <experimentDir>/<name>/<timestamp>/ with
the reference's lines, and its experiment weight is the one the Python runner mirror gives for
the same config. Needs a B200."""
import glob
import math
import json
import os
import subprocess

import pytest

from conftest import ROOT, golden_json

import twisty_b200 as T

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "twisty_b200", "twisty_full_experiment")


def test_full_experiment_cli_results_match_the_api(tmp_path):
    cfg = golden_json("chain_66.json")["config"]
    ep = cfg["experiment"]["experimentParams"]
    ep["pathsToGenerate"] = 200_000
    ep["experimentDir"] = str(tmp_path)
    ep["name"] = "cli"
    path = tmp_path / "cfg.json"
    path.write_text(json.dumps(cfg))
    r = subprocess.run([CLI, str(path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    found = glob.glob(str(tmp_path / "cli" / "*" / "Results.dat"))
    assert len(found) == 1, found
    text = open(found[0]).read()
    lines = {ln.split(":")[0].strip(): ln.split(":", 1)[1].strip() for ln in text.splitlines() if ":" in ln}
    for key in ("Scatter value", "Total experiment weight", "Avg path weight", "Total experiment time (ms)", "Perturb time (ms)"):
        assert any(k.startswith(key) for k in lines), (key, text)
    log10_cli = float(lines["Total experiment weight log10"])
    assert os.path.exists(os.path.join(os.path.dirname(found[0]), "cli.json"))   # the config copied beside
    params, bc = T.ParseExperimentParamsFromConfig(cfg)
    res = T.FullExperimentRunnerOptimalPerturbOptimized_GPU(params).RunExperiment(bc)
    assert res.totalPathsGenerated == 200_000
    assert abs(log10_cli - res.experimentWeightLog10) < 1e-12 * abs(res.experimentWeightLog10)
    # the convergence record (ExperimentRunner::UpdateConvergenceWeight's file): running means
    # per 1e6 paths, the last one over every path
    conv = glob.glob(str(tmp_path / "cli" / "*" / "main" / "ConvergenceWeights" / "ConvergenceWeights.txt"))
    assert len(conv) == 1, conv
    last = open(conv[0]).read().strip().splitlines()[-1].split(",")
    paths, mean = int(last[0]), float(last[1])
    assert paths == 200_000
    assert abs(math.log10(mean * paths) - log10_cli) < 1e-5


def test_full_experiment_cli_writes_the_histogram_on_request(tmp_path):
    cfg = golden_json("chain_66.json")["config"]
    ep = cfg["experiment"]["experimentParams"]
    ep["pathsToGenerate"] = 100_000
    ep["experimentDir"] = str(tmp_path)
    ep["name"] = "hist"
    path = tmp_path / "cfg.json"
    path.write_text(json.dumps(cfg))
    r = subprocess.run([CLI, str(path), "--histogram"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    found = glob.glob(str(tmp_path / "hist" / "*" / "main" / "histogram.txt"))
    assert len(found) == 1, found
    lines = open(found[0]).read().splitlines()
    assert lines[0] == "Histogram" and len(lines) == 501
    counts = [int(ln.split()[2]) for ln in lines[1:]]
    # N = 66 paths weigh ~1e-75, below the five-segment range: all in the first bucket
    assert sum(counts) == 100_000 and counts[0] == 100_000
    lo, hi = float(lines[1].split()[0]), float(lines[-1].split()[1])
    assert lo == pytest.approx(4.69653e-16) and hi == pytest.approx(1.17517e-13)
