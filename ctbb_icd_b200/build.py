"""Build libctbb_icd_b200.so (and the ctbb_icd command-line program) in-tree.

    python -m ctbb_icd_b200.build [--force]

CUDA sources are compiled for sm_100a only (-gencode arch=compute_100a,
code=sm_100a). Files whose results must match the reference bit for bit
(matrix builder, sequential ICD, slice rotation) are compiled with
-fmad=false so no multiply-add is contracted. Host sources use the system
g++ with OpenMP and -ffp-contract=off for the same reason. Objects go to
ctbb_icd_b200/_build/ (git-ignored); the .so lands next to this file so it
travels with the source tree.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libctbb_icd_b200.so")
CLI = os.path.join(HERE, "ctbb_icd")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOSTCXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
EXACT_CU = {"ssm.cu", "icd_seq.cu", "rotate.cu"}
CU_SOURCES = ["ctx.cu", "ssm.cu", "rotate.cu", "recon.cu", "icd_seq.cu", "icd_grouped.cu", "cnn.cu", "cnn_tc.cu",
              "tune.cu"]
CPP_SOURCES = ["host_setup.cpp"]
HEADERS = ["common.h", "gpu_internal.h", "phantom.h"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    inc = os.path.join(os.path.dirname(HERE), "include", "ctbb_icd_b200.h")
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [inc]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs + [__file__]):
            flags = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-fopenmp", "-ccbin", HOSTCXX, "-c", s, "-o", o]
            if src in EXACT_CU:
                flags.insert(1, "-fmad=false")
            _run(flags, verbose)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs + [__file__]):
            _run([HOSTCXX, "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off",
                  "-I", "/usr/local/cuda/include", "-c", s, "-o", o], verbose)
    if force or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-ccbin", HOSTCXX, "-cudart", "static", "-o", LIB, *objs,
              "-Xcompiler", "-fopenmp", "-lgomp"], verbose)
    main_src = os.path.join(CSRC, "main.cpp")
    if os.path.exists(main_src) and (force or _newer(CLI, [main_src, LIB] + hdrs)):
        _run([HOSTCXX, "-O2", "-std=c++17", "-I", os.path.join(os.path.dirname(HERE), "include"),
              main_src, "-o", CLI, "-L", HERE, "-lctbb_icd_b200", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


def build_oracle(verbose: bool = False) -> None:
    """Build the CPU checker: oracle/_ref/liboracle_port.so, plus the
    reference program itself when its sources are present."""
    root = os.path.dirname(HERE)
    oracle = os.path.join(root, "oracle")
    targets = ["port"]
    ref = reference_src()
    if ref:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", oracle, *targets, f"REF={ref or ''}"], check=True,
                   stdout=None if verbose else subprocess.DEVNULL)


def reference_src():
    """The CTBB_ICD source tree (its src/ directory) the oracle builds the
    reference program from: $CTBB_REFERENCE_SRC, else a checkout named
    `reference` beside the repository's directory (reference/src) when one
    is present; None when neither exists (then only the CPU restatement
    is built)."""
    env = os.environ.get("CTBB_REFERENCE_SRC")
    if env:
        return env if os.path.isdir(env) else None
    guess = os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference", "src")
    return guess if os.path.isfile(os.path.join(guess, "icd_iteration.cpp")) else None


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--no-oracle", action="store_true")
    a = ap.parse_args(argv)
    if not shutil.which(NVCC) and not os.path.exists(NVCC):
        sys.exit(f"nvcc not found at {NVCC}")
    print(build(force=a.force, verbose=a.verbose))
    if not a.no_oracle:
        build_oracle(verbose=a.verbose)


if __name__ == "__main__":
    main()
