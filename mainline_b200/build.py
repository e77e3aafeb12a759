"""Build the engine's C-ABI shared library (libqwg.so) in-tree for sm_100a.

    python -m mainline_b200.build            # or __graft_entry__.build()

The library has no Python or torch dependency: plain nvcc + g++ objects,
static CUDA runtime, exported symbols are the qwg_* functions of include/qwg.h.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libqwg.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                  "-I" + os.path.join(ROOT, "include")]

SOURCES_CU = ["qwg_engine.cu"]
SOURCES_CXX = ["qwg_deck.cpp", "qwg_server.cpp", "qwg_log.cpp", "qwg_configs.cpp"]
# walker-kernel families: qwg_walkers.cu once per (working precision, orbital capacity)
FAMILIES = [(real, mm) for real in ("double", "float") for mm in (8, 16, 32, 0, -1)]  # -1: complex orbitals


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, extra_nvflags=None, phases: bool = False) -> str:
    """Build libqwg.so; phases=True builds the profiling library
    libqwg_phases.so (walker-kernel phase counters, -DQWG_PHASES) in its own
    object folder."""
    if phases:
        global BUILD, LIB
        saved = BUILD, LIB
        BUILD, LIB = os.path.join(HERE, "_build_phases"), os.path.join(HERE, "libqwg_phases.so")
        try:
            return build(verbose, list(extra_nvflags or []) + ["-DQWG_PHASES"], False)
        finally:
            BUILD, LIB = saved
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    headers.append(os.path.join(ROOT, "include", "qwg.h"))
    objs, jobs = [], []
    for src in SOURCES_CXX:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _stale(o, [s] + headers):
            _run(["g++", "-c", *CXXFLAGS, "-I" + os.path.join(ROOT, "include"), s, "-o", o])
        objs.append(o)
    units = [(os.path.join(CSRC, src), os.path.join(BUILD, src + ".o"), []) for src in SOURCES_CU]
    wsrc = os.path.join(CSRC, "qwg_walkers.cu")
    for real, mm in FAMILIES:
        units.append((wsrc, os.path.join(BUILD, f"qwg_walkers_{real}_{'cpx' if mm < 0 else mm}.o"),
                      [f"-DQWG_REAL={real}", f"-DQWG_MM={mm}"]))
    for s, o, defs in units:
        if _stale(o, [s] + headers):
            cmd = [NVCC, "-c", *NVFLAGS, *defs, *(extra_nvflags or []), s, "-o", o]
            cmd += ["-Xptxas", "-v"] if verbose else []
            jobs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        objs.append(o)
    failed = None
    for cmd, p in jobs:  # families compile in parallel
        out, err = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out + err)
            failed = cmd
        elif verbose:
            sys.stderr.write(err)
    if failed:
        raise RuntimeError("build step failed: " + " ".join(failed))
    if _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, phases="--phases" in sys.argv))
