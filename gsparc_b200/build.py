"""Build the engine: libgsparc_b200.so (C ABI) and the `gsparc` CLI, for sm_100a.

Objects go to gsparc_b200/_build/, the library to gsparc_b200/lib/ and the CLI
to gsparc_b200/bin/ (all in-tree, none committed).  Rebuilds only what changed.

    python -m gsparc_b200.build [--force] [--jobs N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
BINDIR = os.path.join(PKG, "bin")
LIB = os.path.join(LIBDIR, "libgsparc_b200.so")
CLI = os.path.join(BINDIR, "gsparc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
              "-I" + os.path.join(ROOT, "include"), "-I" + CSRC] + ARCH
LIB_SOURCES = ["util.cpp", "prep.cu", "accumulate.cu", "rowwin.cu", "engine.cu", "capi.cpp", "tns_io.cpp",
               "noalloc.cu", "batch.cu", "stream.cu", "serve.cpp", "wide.cu", "chain.cu", "tune.cpp", "verify.cu",
               "partition.cpp", "radix.cu"]
CLI_SOURCES = ["cli.cpp"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _deps() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _compile(src: str, force: bool, extra: list[str]) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if force or _stale(obj, [src] + _deps()):
        cmd = [nvcc(), "-c", src, "-o", obj] + NVCC_FLAGS + extra
        if src.endswith(".cpp"):
            cmd = [nvcc(), "-x", "cu", "-c", src, "-o", obj] + NVCC_FLAGS + extra
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int = 0, verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BINDIR, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    srcs = [os.path.join(CSRC, s) for s in LIB_SOURCES]
    jobs = jobs or min(8, os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, extra), srcs))
        cli_objs = list(ex.map(lambda s: _compile(s, force, extra), [os.path.join(CSRC, s) for s in CLI_SOURCES]))
    if force or _stale(LIB, objs):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-Xcompiler", "-fPIC", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if force or _stale(CLI, cli_objs + [LIB]):
        cmd = [nvcc(), "-o", CLI] + cli_objs + ARCH + ["-L" + LIBDIR, "-lgsparc_b200", "-lpthread",
                                                      "-Xlinker", "-rpath,$ORIGIN/../lib"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("--ptxas", action="store_true", help="print ptxas register/smem usage")
    a = ap.parse_args(argv)
    print(build(a.force, a.jobs, a.ptxas))
    return 0


if __name__ == "__main__":
    sys.exit(main())
