"""Build recipe for the CUDA library twisty_b200/libtwisty_b200.so (sm_100a).

    python -m twisty_b200.build [--force] [--verbose-ptxas]

Every translation unit under twisty_b200/csrc is compiled by nvcc for
``-gencode arch=compute_100a,code=sm_100a`` into twisty_b200/_build/, then linked into
one shared library with the CUDA runtime linked statically. Objects are rebuilt when
their source or any header under csrc/ or include/ is newer. No GPU is needed to build.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtwisty_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3,-ffp-contract=off", "-I",
          os.path.join(ROOT, "include")]
# Translation units whose FP32 arithmetic must keep the reference's exact rounding. Their
# device code spells every operation with round-to-nearest intrinsics already; the flag
# also keeps any remaining plain expression from being contracted.
NO_FMAD = {"chain_plain.cu", "norm.cu"}


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = os.path.join(cuda, "bin", "nvcc")
    return p if os.path.exists(p) else (shutil.which("nvcc") or "nvcc")


def _host_compiler() -> list[str]:
    # The system g++ (the image's CXX may point at a relocated toolchain).
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return ["-ccbin", c]
    return []


def _sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, force: bool, ptxas_verbose: bool) -> tuple[str, str]:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _headers_mtime()):
        return obj, ""
    cmd = [_nvcc(), *_host_compiler(), *ARCH, *COMMON, "-c", src, "-o", obj]
    if os.path.basename(src) in NO_FMAD:
        cmd.insert(-4, "--fmad=false")
    if ptxas_verbose and src.endswith(".cu"):
        cmd.insert(-4, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, ptxas_verbose), srcs))
    objs = [o for o, _ in results]
    logs = "".join(l for _, l in results)
    if ptxas_verbose and logs:
        print(logs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [_nvcc(), *_host_compiler(), *ARCH, "--shared", "-cudart", "static", "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    # drop-in CLI for the reference's Experiments/FullExperiment.cpp, linked to the library
    cli_src = os.path.join(HERE, "cli", "full_experiment.cpp")
    cli = os.path.join(HERE, "twisty_full_experiment")
    hdr = os.path.join(ROOT, "include", "twisty_b200_runner.hpp")
    if force or not os.path.exists(cli) or os.path.getmtime(cli) < max(os.path.getmtime(cli_src), os.path.getmtime(hdr),
                                                                       os.path.getmtime(LIB)):
        gxx = (_host_compiler() or ["", "g++"])[1]
        r = subprocess.run([gxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), cli_src, "-o", cli,
                            "-L", HERE, "-ltwisty_b200", "-Wl,-rpath,$ORIGIN"], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"CLI build failed:\n{r.stderr}")
    if not quiet:
        print(LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    try:
        build(force=a.force, ptxas_verbose=a.verbose_ptxas, quiet=False)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
