"""Build recipe for the CPU oracle (test infrastructure): oracle/{front,ba,sgm,ext}_oracle.c -> oracle/liboracle.so.

Strict IEEE: -ffp-contract=off and no fast-math, so every fused multiply-add in the oracle is an explicit fma()."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRCS = [os.path.join(HERE, f) for f in ("front_oracle.c", "ba_oracle.c", "sgm_oracle.c", "ext_oracle.c")]
OUT = os.path.join(HERE, "liboracle.so")


def build(force=False):
    if not force and os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(s) for s in SRCS):
        return OUT
    cmd = ["gcc", "-O2", "-march=x86-64-v2", "-mfma", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-shared",
           "-fPIC", "-o", OUT + ".tmp"] + SRCS + ["-lm"]
    subprocess.check_call(cmd)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
