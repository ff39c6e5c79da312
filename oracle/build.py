"""Build recipe for the CPU oracle (test infrastructure).

Produces, under oracle/_build/:
  libsv_oracle.so      serial build (the parity checker)
  libsv_oracle_omp.so  OpenMP build of the same passes (the timed CPU baseline)

Both are compiled with -O2 -ffp-contract=off: an x86-64 build without -mfma contracts no
multiply-add, which is what the reference's own CPU build does, and the FP64 parity
comparison relies on every operation being a separately rounded IEEE operation.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build")
SRC = os.path.join(HERE, "sv_oracle_capi.cpp")
DEPS = [SRC, os.path.join(HERE, "sv_oracle.hpp"),
        os.path.join(HERE, "..", "mfcm_b200", "csrc", "sv_pow43.h"),
        os.path.join(HERE, "..", "include", "sv.h")]

FLAGS = ["-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared"]


def _stale(target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in DEPS)


def build(force=False, verbose=False):
    os.makedirs(OUT, exist_ok=True)
    outs = {
        "serial": (os.path.join(OUT, "libsv_oracle.so"), []),
        "omp": (os.path.join(OUT, "libsv_oracle_omp.so"), ["-fopenmp"]),
    }
    for name, (target, extra) in outs.items():
        if force or _stale(target):
            cmd = ["g++"] + FLAGS + extra + [SRC, "-o", target]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    return {k: v[0] for k, v in outs.items()}


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
