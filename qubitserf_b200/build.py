"""Build libqsfb200.so in-tree: host C++ with g++, kernels with nvcc for sm_100a only.

    python -m qubitserf_b200.build          # incremental
    python -m qubitserf_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libqsfb200.so"
CLI_SRC = PKG / "cli" / "distfind_cli.cpp"
CLI = PKG / "qsfb-distfind"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-pthread",
            f"-I{CUDA_HOME / 'include'}", f"-I{ROOT / 'include'}"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                  "--expt-relaxed-constexpr", f"-I{ROOT / 'include'}"]


def _sources():
    return sorted(CSRC.glob("*.cpp")), sorted(CSRC.glob("*.cu"))


def _headers_mtime():
    hs = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(cmd):
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("compile failed:\n  " + " ".join(cmd) + "\n" + p.stdout + p.stderr)
    return p.stderr


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    cpps, cus = _sources()
    hdr = _headers_mtime()
    jobs, objs = [], []
    for src in cpps + cus:
        obj = OBJ / (src.name + ".o")
        objs.append(obj)
        if not force and obj.exists() and obj.stat().st_mtime > max(src.stat().st_mtime, hdr):
            continue
        if src.suffix == ".cu":
            cmd = [NVCC, *NVFLAGS, "-Xptxas", "-v", "-c", str(src), "-o", str(obj)]
        else:
            cmd = [os.environ.get("CXX", "g++"), *CXXFLAGS, "-c", str(src), "-o", str(obj)]
        jobs.append(cmd)
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
            for err in ex.map(_compile, jobs):
                if verbose and err:
                    print(err, file=sys.stderr)
    if force or jobs or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lpthread"]
        _compile(cmd)
        shutil.move(str(tmp), str(LIB))
    build_cli(force)
    return LIB


def build_cli(force: bool = False) -> Path:
    """The qsfb-distfind command line: a thin executable over the library's C ABI (found
    next to it through an $ORIGIN run path)."""
    if not force and CLI.exists() and CLI.stat().st_mtime > max(CLI_SRC.stat().st_mtime,
                                                                LIB.stat().st_mtime):
        return CLI
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-Wall", "-Wextra",
           f"-I{ROOT / 'include'}", str(CLI_SRC), "-o", str(CLI), f"-L{PKG}", "-lqsfb200",
           "-Wl,-rpath,$ORIGIN"]
    _compile(cmd)
    return CLI


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
