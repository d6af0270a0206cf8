"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``cw_oracle.c`` into ``oracle/libcworacle.so`` with gcc.  The
reference itself is Rust and cannot be compiled in this environment (no cargo
or rustc, crates not vendored), so there is no ``oracle/_ref`` build: the
oracle is a restatement of the reference's functions.

``-ffp-contract=off`` keeps every multiply and add separately rounded, as
Rust does, and ``-march=x86-64-v3`` (AVX2) keeps the library loadable on any
recent x86-64 host.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cw_oracle.c")
LIB = os.path.join(HERE, "libcworacle.so")


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
           "-fPIC", "-shared", "-std=c11", "-Wall", "-Wno-unknown-pragmas", SRC, "-o", LIB + ".tmp", "-lm"]
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
