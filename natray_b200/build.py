"""Builds the in-tree native library natray_b200/libnatray.so for sm_100a.

Every CUDA source is compiled by nvcc for `-gencode arch=compute_100a,code=sm_100a` only; host
C++ sources by g++. Floating-point contraction is off in both (`-fmad=false`,
`-ffp-contract=off`) so that the fixed-point transfer sums are bit-identical to a CPU
evaluation of the same expressions. Host code also takes `-fno-math-errno`: math functions
leave errno alone, so the compiler may treat them as pure (their values do not change). Usage:
`python -m natray_b200.build`.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libnatray.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-math-errno", "-fvisibility=hidden", "-Wall", "-Wno-unused-function"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off",
                  "-Xptxas", "-warn-spills", "--expt-relaxed-constexpr"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    inc = ["-I", str(ROOT / "include"), "-I", str(CSRC)]
    headers = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "natray.h"]
    objs = []
    for src in sorted(CSRC.glob("*.cpp")):
        o = OBJ / (src.stem + ".o")
        if force or _stale(o, [src] + headers):
            _run(["g++", *CXXFLAGS, *inc, "-c", str(src), "-o", str(o)])
        objs.append(o)
    for src in sorted(CSRC.glob("*.cu")):
        o = OBJ / (src.stem + ".cu.o")
        if force or _stale(o, [src] + headers):
            _run([NVCC, *NVFLAGS, *inc, "-c", str(src), "-o", str(o)])
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static", "-lrt", "-lpthread", "-ldl"])
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
