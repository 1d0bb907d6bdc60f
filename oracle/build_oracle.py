"""Build recipe for the CPU oracle (test infrastructure only).

Compiles the C restatement in this folder into ``oracle/liboracle.so`` with gcc. The restatement of the
reference's arithmetic keeps the IEEE semantics of the .NET JIT: no FMA contraction, no fast-math. The sparse
factorisation (o_spd.c), whose rounding the reference does not fix, is compiled with contraction allowed and
dispatches its dense inner kernel by CPU features at load time.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = ["o_common.c", "o_forging3d.c", "o_forging2d.c", "o_spd.c"]
LIB = os.path.join(HERE, "liboracle.so")
COMMON = ["-std=gnu11", "-fPIC", "-fno-fast-math", "-fopenmp", "-Wall", "-Wno-unused-function"]
FLAGS = {"o_spd.c": ["-O3", "-ffp-contract=fast"]}
DEFAULT = ["-O2", "-ffp-contract=off"]


def build_oracle(force: bool = False) -> str:
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    deps = srcs + [os.path.join(HERE, "ifea_oracle.h"), os.path.join(HERE, "o_internal.h"), __file__]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for s in SOURCES:
        obj = os.path.join(objdir, s + ".o")
        subprocess.check_call(["gcc"] + FLAGS.get(s, DEFAULT) + COMMON + ["-c", os.path.join(HERE, s), "-o", obj])
        objs.append(obj)
    subprocess.check_call(["gcc", "-shared", "-fopenmp", "-o", LIB] + objs + ["-lm"])
    return LIB


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
