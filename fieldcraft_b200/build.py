"""Builds the native library in the source tree: ``fieldcraft_b200/libfieldcraft_b200.so``.

Host C++ (the symbolic analysis and the structured-hex8 input builder) is compiled with g++;
the CUDA kernels and the C ABI with nvcc for sm_100a only. The result is one shared library
with the C ABI of ``include/fieldcraft_chol.h`` and ``include/fieldcraft_fem.h``. It loads on a
machine without a GPU (nothing touches CUDA until a handle is created).
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libfieldcraft_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-pthread", f"-I{ROOT / 'include'}"]
NVCCFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", f"-I{ROOT / 'include'}",
                    f"-I{CSRC}", "-Xptxas", "-warn-spills"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build fieldcraft_b200")


def _sources():
    host = sorted((CSRC / "host").glob("*.cpp"))
    cuda = sorted((CSRC / "cuda").glob("*.cu")) + sorted(CSRC.glob("*.cu"))
    headers = sorted(CSRC.rglob("*.cuh")) + sorted(CSRC.rglob("*.hpp")) + sorted((ROOT / "include").glob("*.h"))
    return host, cuda, headers


def _stale(obj: Path, src: Path, headers) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in headers)


def build(verbose: bool = False, force: bool = False) -> Path:
    host, cuda, headers = _sources()
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    cxx = os.environ.get("CXX", "g++")
    jobs = []
    objs = []
    for src in host:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src, headers):
            jobs.append([cxx, *CXXFLAGS, "-c", str(src), "-o", str(obj)])
    for src in cuda:
        obj = BUILD / (src.stem + ".cu.o")
        objs.append(obj)
        if force or _stale(obj, src, headers):
            jobs.append([nvcc, *NVCCFLAGS, "-c", str(src), "-o", str(obj)])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, flush=True)

    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        list(ex.map(run, jobs))
    if jobs or force or not LIB.exists():
        run([nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lpthread"])
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
