"""Builds the oracle's C restatement into oracle/_build/liblucem_oracle.so.

Test infrastructure: the parity tests, the smoke check and the benchmark's
CPU-baseline leg load this library to check results.  Plain gcc, OpenMP, no
-ffast-math (the restatement must keep the reference's f32 rounding).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liblucem_oracle.so")
SOURCES = [os.path.join(HERE, "lucem_oracle.c")]
DEPS = SOURCES + [os.path.join(HERE, "lucem_oracle.h"), os.path.join(HERE, "lucem_oracle_body.inc")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in DEPS)


def build(force: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-o", LIB, *SOURCES, "-lm"]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
