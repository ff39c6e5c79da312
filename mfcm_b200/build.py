"""Build the CUDA library mfcm_b200/lib/libsv_b200.so for sm_100a (in-tree, so the built
.so travels with the source tree).

sv_f64.cu is compiled with -fmad=false: the FP64 path must round every multiply and add
separately, like the reference's CPU arithmetic. sv_f32.cu keeps contraction on.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
OBJ_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIB_DIR, "libsv_b200.so")
INCLUDE = os.path.join(HERE, "..", "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE] + ARCH
UNITS = {
    "sv_f64.cu": ["-fmad=false"],
    "sv_f32.cu": [],
    "sv_capi.cu": [],
    "sv_noalloc.cu": [],
}


def _nvcc():
    for c in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if os.path.exists(c) or c == "nvcc":
            return c


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "sv.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    deps = _deps()
    objs = []
    nvcc = _nvcc()
    for unit, flags in UNITS.items():
        obj = os.path.join(OBJ_DIR, unit + ".o")
        objs.append(obj)
        if force or _stale(obj, deps):
            cmd = [nvcc] + COMMON + list(flags) + list(extra) + ["-c", os.path.join(CSRC, unit), "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.check_call(cmd)
    if force or _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    extra = [a for a in sys.argv[1:] if a.startswith("-X") or a.startswith("--")]
    extra = [a for a in extra if a != "--force"]
    print(build(force="--force" in sys.argv, verbose=True, extra=extra))
