"""Build recipe for the CPU oracle (test infrastructure): oracle/front_oracle.c -> oracle/liboracle.so.

Strict IEEE: -ffp-contract=off and no fast-math, so every fused multiply-add in the oracle is an explicit fma()."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "front_oracle.c")
OUT = os.path.join(HERE, "liboracle.so")


def build(force=False):
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    cmd = ["gcc", "-O2", "-march=x86-64-v2", "-mfma", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-shared",
           "-fPIC", "-o", OUT + ".tmp", SRC, "-lm"]
    subprocess.check_call(cmd)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
