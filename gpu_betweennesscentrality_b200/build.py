"""Build recipe of libqbc_b200.so and the drop-in CLIs (MHLQBC, QBC, RQ), in-tree.

    python -m gpu_betweennesscentrality_b200.build [--force]

Device code is compiled for sm_100a only (B200).  Objects go to ``_build/``; the shared
library lands next to this file and the CLIs in ``bin/`` with an rpath to the library.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libqbc_b200.so")
BIN = os.path.join(PKG, "bin")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
CLIS = {"MHLQBC": "QBC_CLI_MHL", "QBC": "QBC_CLI_QBC", "RQ": "QBC_CLI_RQ"}


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    # the system g++ (with libstdc++ shared); an $CXX wrapper may link libstdc++ statically
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("g++ not found")


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    nvcc, cxx = _nvcc(), _cxx()
    headers = [os.path.join(CSRC, h) for h in ("host.h", "device.h", "device_state.h")] + [os.path.join(INCLUDE, "qbc_b200.h")]
    objs = []
    for src, kind in (("host.cpp", "cxx"), ("index_file.cpp", "cxx"), ("capi.cpp", "cxx"), ("device.cu", "cu"), ("sssp.cu", "cu"), ("sweep.cu", "cu")):
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if not force and not _stale(o, [s] + headers + [__file__]):
            continue
        if kind == "cxx":
            cmd = [cxx, "-O3", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function", "-pthread", "-fopenmp",
                   "-I", INCLUDE, "-c", s, "-o", o]
        else:
            cmd = [nvcc, "-O3", "-std=c++17", *GENCODE, "-lineinfo", "-ccbin", cxx, "-Xcompiler", "-fPIC",
                   "-I", INCLUDE, "-c", s, "-o", o]
        _run(cmd, verbose)
    if force or _stale(LIB, objs):
        _run([nvcc, "-shared", *GENCODE, "-ccbin", cxx, "-o", LIB, *objs, "-lpthread", "-lgomp"], verbose)
    cli_src = os.path.join(CSRC, "cli.cpp")
    for name, macro in CLIS.items():
        out = os.path.join(BIN, name)
        if force or _stale(out, [cli_src, LIB, os.path.join(INCLUDE, "qbc_graph.hpp")] + headers):
            _run([cxx, "-O2", "-std=c++17", f"-D{macro}", "-I", INCLUDE, cli_src, "-o", out,
                  "-L", PKG, "-lqbc_b200", "-Wl,-rpath,$ORIGIN/.."], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
