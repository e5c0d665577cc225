"""Builds libdsmc_b200.so in-tree (master_b200/libdsmc_b200.so) and the
dsmc_b200_main executable.

Kernels are compiled for sm_100a only (B200).  Host C++ is compiled without
floating-point contraction so the geometry generator rounds exactly as the
reference's build does.  Incremental: an object is rebuilt when its source or
any header in csrc/ or include/ is newer.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libdsmc_b200.so"
MAIN = PKG / "dsmc_b200_main"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
               f"-I{INCLUDE}", f"-I{CSRC}"]

# source -> extra flags
CUDA_SOURCES = {
    "kernels_split.cu": [],
    # the reference's fp64 arithmetic: no fused multiply-add
    "kernels_fp64.cu": ["-fmad=false"],
    "api.cu": [],
    "cell_layout.cu": [],
    # must round exactly as the CPU geometry path
    "geometry_gpu.cu": ["-fmad=false"],
    # the warm-start surrogate's tcgen05 convolutions and training kernels
    "surrogate.cu": [],
}
CXX_SOURCES = ["host_setup.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers_mtime() -> float:
    files = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return max((f.stat().st_mtime for f in files), default=0.0)


def _stale(target: Path, *deps: float) -> bool:
    return not target.exists() or target.stat().st_mtime < max(deps)


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ... {cmd[-1]}")


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    hdr = _headers_mtime()
    objs = []
    for src, extra in CUDA_SOURCES.items():
        s = CSRC / src
        o = BUILD / (src + ".o")
        if _stale(o, s.stat().st_mtime, hdr):
            if verbose:
                print("nvcc", src)
            _run([nvcc, *ARCH, *NVCC_COMMON, *extra, "-c", str(s), "-o", str(o)])
        objs.append(o)
    for src in CXX_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        if _stale(o, s.stat().st_mtime, hdr):
            if verbose:
                print("g++", src)
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", f"-I{INCLUDE}", f"-I{CSRC}",
                  f"-I{Path(nvcc).resolve().parent.parent / 'include'}",
                  "-c", str(s), "-o", str(o)])
        objs.append(o)
    newest = max(o.stat().st_mtime for o in objs)
    if _stale(LIB, newest):
        _run([nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs)])
    main_src = CSRC / "main.cpp"
    if main_src.exists() and _stale(MAIN, main_src.stat().st_mtime, LIB.stat().st_mtime, hdr):
        _run(["g++", "-O2", "-std=c++17", f"-I{INCLUDE}", str(main_src), "-o", str(MAIN), f"-L{PKG}",
              "-ldsmc_b200", f"-Wl,-rpath,{PKG}", "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
