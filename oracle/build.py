"""Build recipe for the CPU oracle (test infrastructure).

Produces, under oracle/_build/:
  libsv_oracle.so      serial build (the parity checker)
  libsv_oracle_omp.so  OpenMP build of the same passes (the timed CPU baseline)
  sv_oracle_san        with --sanitize: the oracle under ASan + UBSan, driven over its whole
                       C-ABI by sanitize_main.cpp (tests/test_oracle_sanitize.py runs it)

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


SAN_SRC = os.path.join(HERE, "sanitize_main.cpp")
SAN_FLAGS = ["-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", "-ffp-contract=off",
             "-fsanitize=address,undefined", "-fno-sanitize-recover=all"]


def build_sanitized(force=False, verbose=False):
    """oracle/_build/sv_oracle_san: the oracle and a driver over its whole C-ABI
    (sanitize_main.cpp) under AddressSanitizer and UndefinedBehaviorSanitizer."""
    os.makedirs(OUT, exist_ok=True)
    target = os.path.join(OUT, "sv_oracle_san")
    if force or _stale(target) or os.path.getmtime(SAN_SRC) > os.path.getmtime(target):
        cmd = ["g++"] + SAN_FLAGS + [SRC, SAN_SRC, "-o", target]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return target


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
    if "--sanitize" in sys.argv:
        print(build_sanitized(force="--force" in sys.argv, verbose=True))
