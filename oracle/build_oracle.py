"""Build recipe for the CPU oracle (test infrastructure only).

Compiles the C restatement in this folder into ``oracle/liboracle.so`` with gcc. The flags keep IEEE
semantics the reference's .NET JIT has: no FMA contraction, no fast-math.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = ["o_common.c", "o_forging3d.c", "o_forging2d.c"]
LIB = os.path.join(HERE, "liboracle.so")


def build_oracle(force: bool = False) -> str:
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    deps = srcs + [os.path.join(HERE, "ifea_oracle.h"), os.path.join(HERE, "o_internal.h")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    cmd = ["gcc", "-O2", "-std=gnu11", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
           "-Wall", "-Wno-unused-function", "-o", LIB] + srcs + ["-lm"]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
