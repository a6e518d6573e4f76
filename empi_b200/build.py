"""Builds the sm_100a engine in-tree: empi_b200/libempi_b200.so and the
empi-gpu CLI (empi_b200/empi-gpu).

    python -m empi_b200.build [--force]

nvcc cross-compiles for sm_100a without a GPU.  The CUDA runtime is linked
statically so the library loads without extra library paths.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libempi_b200.so")
CHECK_LIB = os.path.join(HERE, "libempi_b200_check.so")
CLI = os.path.join(HERE, "empi-gpu")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
                     "--expt-relaxed-constexpr", "-diag-suppress", "177"]
SOURCES = ["engine.cu", "refresh_single.cu", "refresh_mmp1.cu", "refresh_mmp3.cu", "persist_single.cu",
           "persist_mmp1.cu", "persist_mmp3.cu", "proposal.cu", "geometry.cpp", "hostio.cpp", "tune.cpp"]
# Device code of the engine: single-precision math with approximate division,
# square root and exp2 and flush-to-zero (the FP32 energy maps; FP64 code is
# unaffected).  The FP32 maps only rank candidates: every bin within 1e-4 of
# the maximum is re-scored in FP64, and the parity tests bound the map error.
ENGINE_FLAGS = ["--use_fast_math"]
HEADERS = ["fft.cuh", "common.cuh", "kernels.cuh", "refresh.cuh", "persist.cuh", "refresh_kernels.hpp", "plan.hpp", "geometry.hpp",
           "engine.hpp", "tune.hpp", "proposal.hpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def _stale(target, deps) -> bool:
    return not os.path.exists(target) or os.path.getmtime(target) < _newest(deps)


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    """Builds the library (and the CLI).  checked=True builds the diagnostic
    variant libempi_b200_check.so instead: every data-dependent index is
    bounds-checked on the device (-DEMPI_CHECK); select it with
    EMPI_B200_LIB."""
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [
        os.path.join(ROOT, "include", "empi_b200.h"), __file__]
    lib = CHECK_LIB if checked else LIB
    bdir = BUILD + ("_check" if checked else "")
    extra = ["-DEMPI_CHECK"] if checked else []
    os.makedirs(bdir, exist_ok=True)
    cc = nvcc()
    ccbin = ["-ccbin", host_cxx()]
    if force or _stale(lib, deps):
        from concurrent.futures import ThreadPoolExecutor

        objs, cmds = [], []
        for src in SOURCES:
            obj = os.path.join(bdir, src + ".o")
            cmd = [cc] + ccbin + NVCC_FLAGS + ENGINE_FLAGS + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
            if src.endswith(".cpp"):
                cmd = [cc] + ccbin + ["-x", "cu"] + NVCC_FLAGS + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
            if verbose:
                print(" ".join(cmd))
            cmds.append(cmd)
            objs.append(obj)
        # the translation units compile in parallel (the refresh kernels of each
        # variant mode are the slow ones)
        with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
            for r in pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds):
                if r.returncode != 0:
                    raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
        tmp = lib + ".tmp"
        cmd = [cc] + ccbin + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs
        subprocess.run(cmd, check=True)
        os.replace(tmp, lib)
    if checked:
        return lib
    cli_src = os.path.join(CSRC, "empi_cli.cpp")
    if force or _stale(CLI, [cli_src, LIB]):
        cmd = [host_cxx(), "-O2", "-std=c++17", "-o", CLI, cli_src, "-L" + HERE, "-lempi_b200",
               "-Wl,-rpath,$ORIGIN"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, checked="--checked" in sys.argv))
