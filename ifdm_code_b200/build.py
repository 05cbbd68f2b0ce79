"""Build recipe for libifdm_b200.so, the BECMPI drop-in executable and the readsnap tool (sm_100a).

    python -m ifdm_code_b200.build [--force] [--verbose]

Objects go to ifdm_code_b200/_build/, the library to ifdm_code_b200/, the
executables to ifdm_code_b200/bin/.  nvcc cross-compiles for sm_100a, so this
runs on machines without a GPU.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
import time

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libifdm_b200.so")
BIN = os.path.join(PKG, "bin", "BECMPI")
READSNAP = os.path.join(PKG, "bin", "readsnap")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                     "-ccbin", "g++", "-I" + CSRC, "-I" + INC]
# the IC deposit reproduces the reference's rounding step by step: no FMA contraction
PER_FILE = {"ic_pipeline.cu": ["--fmad=false"]}
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-Wall", "-I" + CSRC, "-I" + INC]

CU_SOURCES = ["step_engine.cu", "batch_engine.cu", "batch_fp64.cu", "batch_fp32.cu", "batch_mixed.cu",
              "ic_pipeline.cu", "static_poisson.cu", "diagnostics.cu"]
CPP_SOURCES = ["ifdm_api.cpp", "io.cpp", "snapshot_stream.cpp", "ic_stream.cpp"]


def _cuda_home() -> str:
    for cand in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if cand and os.path.exists(os.path.join(cand, "bin", "nvcc")):
            return cand
    nvcc = shutil.which("nvcc")
    if nvcc:
        return os.path.dirname(os.path.dirname(nvcc))
    raise RuntimeError("nvcc not found")


def _newest_header() -> float:
    t = 0.0
    for d in (CSRC, INC):
        for f in os.listdir(d):
            if f.endswith((".h", ".hpp", ".cuh")):
                t = max(t, os.path.getmtime(os.path.join(d, f)))
    return t


def _stale(out: str, src: str, hdr_time: float) -> bool:
    if not os.path.exists(out):
        return True
    ot = os.path.getmtime(out)
    return ot < os.path.getmtime(src) or ot < hdr_time


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every CUDA/C++ source for sm_100a; returns the library path."""
    cuda = _cuda_home()
    nvcc = os.path.join(cuda, "bin", "nvcc")
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    hdr = _newest_header()
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        out = os.path.join(OBJ, s + ".o")
        objs.append(out)
        if force or _stale(out, src, hdr):
            jobs.append([nvcc] + NVCC_FLAGS + PER_FILE.get(s, []) + ["-c", src, "-o", out])
    for s in CPP_SOURCES:
        src = os.path.join(CSRC, s)
        out = os.path.join(OBJ, s + ".o")
        objs.append(out)
        if force or _stale(out, src, hdr):
            jobs.append(["g++"] + CXX_FLAGS + ["-I" + os.path.join(cuda, "include"), "-c", src, "-o", out])
    # an object is stamped with the time its compile started, so a source or
    # header edited while it compiled stays newer than it and is rebuilt next time
    t_start = time.time()

    def compile_one(cmd):
        _run(cmd, verbose)
        os.utime(cmd[cmd.index("-o") + 1], (t_start, t_start))

    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(compile_one, jobs))
    if force or jobs or not os.path.exists(LIB):
        _run([nvcc] + ARCH + ["-shared", "-ccbin", "g++", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl"],
             verbose)
    main_src = os.path.join(CSRC, "becmpi_main.cpp")
    if force or _stale(BIN, main_src, hdr) or os.path.getmtime(BIN) < os.path.getmtime(LIB):
        _run(["g++", "-O2", "-std=c++17", "-I" + INC, main_src, "-o", BIN, "-L" + PKG, "-lifdm_b200",
              "-Wl,-rpath,$ORIGIN/.."], verbose)
    build_readsnap(force, verbose)
    return LIB


def build_readsnap(force: bool = False, verbose: bool = False) -> str:
    """The host-only slice tool (no CUDA); returns its path."""
    src = os.path.join(CSRC, "readsnap_main.cpp")
    os.makedirs(os.path.dirname(READSNAP), exist_ok=True)
    if force or _stale(READSNAP, src, os.path.getmtime(src)):
        _run(["g++", "-O2", "-std=c++17", src, "-o", READSNAP], verbose)
    return READSNAP


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
