"""Build the in-tree CUDA library ``liblangevin_b200.so`` for sm_100a.

The library is compiled with nvcc directly (no JIT cache): the built ``.so`` sits
next to this file, so it travels with the source tree to the GPU machine.
"""
from __future__ import annotations

import concurrent.futures as _cf
import os
import shutil
import subprocess
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
CSRC = PKG_DIR / "csrc"
INCLUDE = PKG_DIR.parent / "include"
LIB_NAME = "liblangevin_b200.so"
LIB_PATH = PKG_DIR / LIB_NAME
BUILD_DIR = PKG_DIR / "_build"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    # single-precision only: FTZ and the fast divide/sqrt; FP64 is unaffected
    "-ftz=true", "-prec-div=false", "-prec-sqrt=false",
    "--expt-relaxed-constexpr",
]
SOURCES = ["lim_kernels.cu", "lim_capi.cu", "lim_noalloc.cu", "lim_batch.cu", "lim_batch_capi.cu", "lim_sample.cu", "lim_reduce.cu", "lim_tables.cu",
           "lim_adjoint.cu", "lim_adjoint_capi.cu", "lim_static.cu"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build liblangevin_b200.so")


def _host_compiler() -> list[str]:
    # nvcc needs a host g++ whose runtime matches the system one
    gxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else shutil.which("g++")
    return ["-ccbin", gxx] if gxx else []


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every CUDA source for sm_100a and link the shared library."""
    nvcc = nvcc_path()
    BUILD_DIR.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))
    objs = []
    jobs = []
    for src in SOURCES:
        s = CSRC / src
        o = BUILD_DIR / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc, *_host_compiler(), *ARCH_FLAGS, *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(s), "-o", str(o)]
            jobs.append(cmd)
    with _cf.ThreadPoolExecutor(max_workers=max(1, len(jobs))) as ex:
        results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), jobs))
    for cmd, r in zip(jobs, results):
        if verbose or r.returncode != 0:
            print(" ".join(cmd))
            print(r.stdout, r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed ({r.returncode}) on {cmd[-3]}")
    if force or jobs or _stale(LIB_PATH, objs):
        cmd = [nvcc, *_host_compiler(), *ARCH_FLAGS, "-shared", "-o", str(LIB_PATH), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            print(" ".join(cmd))
            print(r.stdout, r.stderr)
            raise RuntimeError("nvcc link failed")
    return LIB_PATH


def ptxas_report() -> str:
    """Register / spill / shared-memory usage of every kernel (-Xptxas -v)."""
    nvcc = nvcc_path()
    out = []
    for src in SOURCES:
        cmd = [nvcc, *_host_compiler(), *ARCH_FLAGS, *NVCC_FLAGS, "-Xptxas", "-v", "-I", str(INCLUDE),
               "-c", str(CSRC / src), "-o", os.devnull]
        r = subprocess.run(cmd, capture_output=True, text=True)
        out.append(r.stderr)
    return "\n".join(out)


if __name__ == "__main__":
    print(build(force=True, verbose=False))
