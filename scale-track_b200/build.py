"""Builds libscaletrack.so in place for sm_100a with nvcc (no JIT, no torch extension).

    python scale-track_b200/build.py [--force]

Every .cu in csrc/ is compiled with --fmad=false (the reference's arithmetic has no fused
multiply-adds, and the CPU oracle must see the same roundings) and linked with the static
CUDA runtime into scale-track_b200/libscaletrack.so, which travels with the repository
snapshot to the GPU machine.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libscaletrack.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fvisibility=hidden", "-Xptxas", "-warn-spills",
    "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in deps())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    env = dict(os.environ)
    # the system compiler pairs with the CUDA toolkit's supported host compiler list
    ccbin = []
    if os.path.exists("/usr/bin/g++"):
        ccbin = ["-ccbin", "/usr/bin/g++"]
    objs = []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        cmd = [cc] + ccbin + NVCC_FLAGS + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd, env=env)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [cc] + ccbin + ARCH + ["-shared", "-o", tmp] + objs + ["-Xlinker", "--no-undefined"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd, env=env)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
