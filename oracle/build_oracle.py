"""Compile the oracle's C restatement (oracle/upbp_oracle.c) into oracle/liboracle.so (test infrastructure)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")      # FP32 restatement
LIB64 = os.path.join(HERE, "liboracle64.so")  # FP64 oracle (same candidates, FP64 contributions)


def build() -> str:
    for lib, real in ((LIB, "float"), (LIB64, "double")):
        cmd = ["gcc", "-std=c99", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared", "-Wall",
               "-Wno-unused-function", "-DORACLE_REAL=" + real, os.path.join(HERE, "upbp_oracle.c"), "-o", lib, "-lm"]
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build())
    sys.exit(0)
