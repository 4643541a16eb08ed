"""Builds libtwofold_b200.so in-tree for sm_100a.

Float semantics match the reference's build (-ffp-contract=off, IEEE division and square root): device code
compiles with --fmad=false and precise division and square root; host code with -ffp-contract=off.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libtwofold_b200.so")

SOURCES = [os.path.join(CSRC, "tf_engine.cu")]
HEADERS = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
    os.path.join(ROOT, "include", "twofold_b200.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden,-O2",
    "-Xptxas", "-v",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(p) > t for p in SOURCES + HEADERS + [__file__])


def build(force=False, verbose=False, out=None, defines=()):
    """Builds the library; `defines` adds -D flags (TF_DEVICE_CHECKS builds the index-checking variant)."""
    target = out or OUT
    if not force and out is None and not stale():
        return OUT
    cmd = [nvcc()] + NVCC_FLAGS + [f"-D{d}" for d in defines] + ["-shared", "-o", target] + SOURCES
    res = subprocess.run(cmd, capture_output=True, text=True)
    log = res.stdout + res.stderr
    with open(os.path.join(HERE, "build.log"), "w") as f:
        f.write(" ".join(cmd) + "\n" + log)
    if res.returncode != 0:
        sys.stderr.write(log)
        raise RuntimeError("nvcc failed building libtwofold_b200.so")
    if verbose:
        sys.stderr.write(log)
    return target


if __name__ == "__main__":
    if "--checked" in sys.argv:
        print(build(force=True, out=sys.argv[sys.argv.index("--checked") + 1], defines=("TF_DEVICE_CHECKS",)))
    else:
        print(build(force="--force" in sys.argv, verbose=True))
