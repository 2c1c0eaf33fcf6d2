"""Build recipe for the CPU oracle (test infrastructure).

Compiles ``oracle/vmc_oracle.c`` into ``oracle/_build/libpmo_oracle.so`` with
gcc and OpenMP.  Used by ``__graft_entry__.build()``, the tests and the CPU
baseline leg of ``bench.py``; the product path never loads the result.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libpmo_oracle.so")
SOURCES = ["vmc_oracle.c", "vmc_oracle_body.h", "philox_ref.h", "../include/pmo_b200.h"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(os.path.join(HERE, s)) > t for s in SOURCES)


def build(force: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [
        "gcc", "-O2", "-std=gnu11", "-fPIC", "-shared", "-fopenmp",
        "-fno-fast-math", "-ffp-contract=off",
        "-Wall", "-Wno-unused-function", "-Wno-maybe-uninitialized",
        os.path.join(HERE, "vmc_oracle.c"), "-o", LIB + ".tmp", "-lm",
    ]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
