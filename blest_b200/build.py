"""Build libblest_b200.so in-tree: host C++ (g++/OpenMP) + sm_100a CUDA
(nvcc -gencode arch=compute_100a,code=sm_100a), linked into one shared
library next to this file. Usage: python blest_b200/build.py [--force | --ptxas]
(by path: importing the package needs the library this builds)."""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libblest_b200.so"
CLI = PKG / "blest"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXX = shutil.which("g++") or "g++"
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CXXFLAGS = ["-std=c++20", "-O3", "-fPIC", "-fopenmp", "-Wall", "-Wextra", f"-I{INCLUDE}", f"-I{CSRC / 'host'}"]
NVCCFLAGS = ["-std=c++20", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-fopenmp", f"-I{INCLUDE}",
             f"-I{CSRC / 'host'}", f"-I{CSRC / 'device'}", "--expt-relaxed-constexpr"]


def _headers() -> list[Path]:
    return [*INCLUDE.glob("*.h"), *CSRC.rglob("*.hpp"), *CSRC.rglob("*.cuh")]


def _stale(obj: Path, src: Path, newest_header: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or newest_header > t


def _compile(src: Path, obj: Path) -> tuple[Path, str]:
    if src.suffix == ".cu":
        cmd = [NVCC, *NVCCFLAGS, "-c", str(src), "-o", str(obj)]
    else:
        cmd = [CXX, *CXXFLAGS, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    lib_srcs = sorted([*(CSRC / "host").glob("*.cpp"), *(CSRC / "device").glob("*.cu")])
    newest = max((h.stat().st_mtime for h in _headers()), default=0.0)
    jobs = []
    objs = []
    for src in lib_srcs:
        obj = BUILD / (src.parent.name + "_" + src.name + ".o")
        objs.append(obj)
        if force or _stale(obj, src, newest):
            jobs.append((src, obj))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
            for obj, log in ex.map(lambda j: _compile(*j), jobs):
                if verbose and log.strip():
                    print(log, file=sys.stderr)
    if jobs or not LIB.exists():
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lgomp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    cli_src = CSRC / "cli" / "main.cpp"
    if cli_src.exists() and (force or not CLI.exists() or cli_src.stat().st_mtime > CLI.stat().st_mtime
                             or LIB.stat().st_mtime > CLI.stat().st_mtime):
        cmd = [CXX, "-std=c++20", "-O2", f"-I{INCLUDE}", str(cli_src), "-o", str(CLI), f"-L{PKG}",
               "-lblest_b200", f"-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"CLI build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


def ptxas_report() -> str:
    """Registers / spills / shared memory of every kernel (-Xptxas -v)."""
    out = []
    for src in sorted((CSRC / "device").glob("*.cu")):
        cmd = [NVCC, *NVCCFLAGS, "-Xptxas", "-v", "-c", str(src), "-o", "/dev/null"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        out.append(f"== {src.name}\n{r.stderr}")
    return "\n".join(out)


if __name__ == "__main__":
    if "--ptxas" in sys.argv:
        print(ptxas_report())
    else:
        print(build(force="--force" in sys.argv, verbose=True))
