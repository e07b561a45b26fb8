"""Build recipe for the CPU oracle (test infrastructure).

Compiles oracle/oracle_capi.cpp into oracle/_build/liboracle.so with g++/OpenMP.
Run directly (``python oracle/build_oracle.py``) or through ``__graft_entry__.build``.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
# The same oracle with fused multiply-adds wherever the compiler forms them (as the
# GPU's compiler does): its FP64 results differ from the plain oracle's by rounding
# only, which measures the FP64 noise floor of an output (deep-zoom normals).
LIB_FMA = os.path.join(OUT_DIR, "liboracle_fma.so")


def build(force: bool = False, fma: bool = False) -> str:
    src = os.path.join(HERE, "oracle_capi.cpp")
    deps = [src, os.path.join(HERE, "oracle.hpp"), os.path.join(HERE, "..", "include", "nd_march.h")]
    lib = LIB_FMA if fma else LIB
    if not force and os.path.exists(lib) and all(os.path.getmtime(lib) >= os.path.getmtime(d) for d in deps):
        return lib
    os.makedirs(OUT_DIR, exist_ok=True)
    # -ffp-contract=off keeps the oracle's float mode free of FMA contraction
    cmd = ["g++", "-std=c++17", "-O3", "-march=x86-64-v3", "-ffp-contract=fast" if fma else "-ffp-contract=off",
           "-fopenmp", "-fPIC", "-shared", src, "-o", lib + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(lib + ".tmp", lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
    print(build(force="--force" in sys.argv, fma=True))
