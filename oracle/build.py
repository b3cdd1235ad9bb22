"""TEST INFRASTRUCTURE: build recipe of the oracle (CPU restatement of the
slosh substep).  Compiles ``oracle/slosh_oracle.cpp`` with g++ into
``oracle/build/liboracle.so`` (OpenMP, no FMA contraction so that float
operations round as written)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
SRC = os.path.join(HERE, "slosh_oracle.cpp")
HDR = os.path.join(HERE, "..", "include", "slosh_b200.h")

FLAGS = ["-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared"]


def build_oracle(force: bool = False) -> str:
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if os.path.getmtime(SRC) <= t and os.path.getmtime(HDR) <= t:
            return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = LIB + ".tmp"
    res = subprocess.run(["g++", *FLAGS, SRC, "-o", tmp], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("g++ failed:\n" + res.stdout + res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build_oracle(force=True))
