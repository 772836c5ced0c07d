"""Build libp3mx.so (sm_100a) in-tree with nvcc.

    python -m espresso_b200.build          # or: python espresso_b200/build.py
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libp3mx.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cuh"))] + [os.path.join(HERE, "..", "include", "p3mx.h")]


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force=False, verbose=False):
    if not force and not needs_build():
        return OUT
    cmd = [nvcc_path(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--use_fast_math=false",
           "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
           "-ccbin", shutil.which("g++") or "g++",
           "-o", OUT + ".tmp", os.path.join(CSRC, "p3mx_all.cu")]
    cmd = [c for c in cmd if c != "--use_fast_math=false"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
