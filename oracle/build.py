"""Build recipe for the C restatement (test infrastructure only).

    python oracle/build.py        -> oracle/libpk_oracle.so

gcc + OpenMP; no reference sources are compiled (the reference is Rust and
cannot be built in this image).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRCS = [os.path.join(HERE, "pk_oracle.c"), os.path.join(HERE, "pk_oracle_whir.c")]
LIB = os.path.join(HERE, "libpk_oracle.so")


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(
        [os.path.getmtime(s) for s in SRCS] + [os.path.getmtime(os.path.join(HERE, "pk_oracle.h"))]
    ):
        return LIB
    cmd = ["gcc", "-O3", "-fopenmp", "-Wall", "-Wextra", "-shared", "-fPIC", "-o", LIB] + SRCS
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
