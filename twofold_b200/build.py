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

SOURCES = [os.path.join(CSRC, f) for f in ("tf_engine.cu", "tf_noalloc.cu", "tf_adjoint.cu")]
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


CHECKED_OUT = os.path.join(HERE, "libtwofold_b200_checked.so")


def _command(target, defines):
    return [nvcc()] + NVCC_FLAGS + [f"-D{d}" for d in defines] + ["-shared", "-o", target] + SOURCES


def build(force=False, verbose=False, out=None, defines=(), checked=True):
    """Builds libtwofold_b200.so and, alongside it, libtwofold_b200_checked.so: the same library with every
    device index check on (TF_DEVICE_CHECKS), which records the first out-of-range index instead of using it.
    `out`/`defines` build a single variant instead."""
    if out is not None:
        jobs = [(out, tuple(defines))]
    else:
        if not force and not stale() and (not checked or os.path.exists(CHECKED_OUT)):
            return OUT
        jobs = [(OUT, ())] + ([(CHECKED_OUT, ("TF_DEVICE_CHECKS",))] if checked else [])
    procs = [(t, subprocess.Popen(_command(t, d), stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
             for t, d in jobs]
    for target, proc in procs:
        log = proc.communicate()[0]
        if target == OUT:
            with open(os.path.join(HERE, "build.log"), "w") as f:
                f.write(" ".join(_command(target, ())) + "\n" + log)
        if proc.returncode != 0:
            sys.stderr.write(log)
            raise RuntimeError(f"nvcc failed building {os.path.basename(target)}")
        if verbose:
            sys.stderr.write(log)
    return jobs[0][0]


if __name__ == "__main__":
    if "--checked" in sys.argv:
        print(build(force=True, out=sys.argv[sys.argv.index("--checked") + 1], defines=("TF_DEVICE_CHECKS",)))
    else:
        print(build(force="--force" in sys.argv, verbose=True))
