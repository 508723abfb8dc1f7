"""Builds the oracle (test infrastructure, see oracle.cpp) into oracle/libntr_oracle.so.

g++ -O3 with OpenMP and without floating-point contraction, so every expression is evaluated
with the association written in the source. Usage: `python oracle/build.py`.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
LIB = HERE / "libntr_oracle.so"
SRC = HERE / "oracle.cpp"


def build(force: bool = False) -> Path:
    deps = [SRC, ROOT / "include" / "natray.h"]
    if not force and LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in deps):
        return LIB
    cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
           "-march=x86-64-v3", "-fvisibility=hidden", "-I", str(ROOT / "include"), str(SRC), "-o", str(LIB)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
