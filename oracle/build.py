"""Build the CPU oracle (test infrastructure) into oracle/liboracle.so.

The oracle is a C restatement of numax.linalg's algorithms; it is the
checker for the CUDA library, never part of it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("nmx_oracle.c", "nmx_oracle_impl.h")]
    if not force and os.path.exists(LIB) and all(
        os.path.getmtime(LIB) >= os.path.getmtime(s) for s in srcs
    ):
        return LIB
    # -ffp-contract=off keeps every multiply and add separately rounded, as
    # the restated loops are written; -O2 without -ffast-math keeps IEEE order.
    cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp",
           "-ffp-contract=off", srcs[0], "-o", LIB, "-lm"]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
