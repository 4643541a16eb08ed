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

# The engine (host code, no kernels) and the kernel groups it launches (tf_launch.h), which compile in parallel.
SOURCES = [os.path.join(CSRC, f) for f in ("tf_engine.cu", "tf_k_broad.cu", "tf_k_collide.cu", "tf_k_refresh.cu",
                                           "tf_k_solve.cu", "tf_k_finish.cu", "tf_k_flat.cu", "tf_noalloc.cu",
                                           "tf_adjoint.cu")]
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


# The differentiable model (tf_adjoint.cu) is not held to the reference's bits, so it may contract
# multiply-adds; every other source is compiled without contraction.
CONTRACTED = {"tf_adjoint.cu"}
BUILD_DIR = os.path.join(HERE, "_build")


# The flat solve's CTAs read what other CTAs of the same launch wrote before a grid barrier: its global loads
# must come from L2, not from an SM's L1, which is not kept coherent with other SMs' stores.
L2_LOADS = {"tf_k_flat.cu"}


def _flags(source):
    flags = list(NVCC_FLAGS)
    if os.path.basename(source) in CONTRACTED:
        flags[flags.index("--fmad=false")] = "--fmad=true"
    if os.path.basename(source) in L2_LOADS:
        flags += ["-Xptxas", "-dlcm=cg"]
    return flags


def _object(source, variant):
    return os.path.join(BUILD_DIR, variant, os.path.basename(source)[:-3] + ".o")


def _compile_command(source, variant, defines):
    return [nvcc()] + _flags(source) + [f"-D{d}" for d in defines] + ["-c", "-o", _object(source, variant), source]


def _link_command(target, variant):
    return [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", target] + \
        [_object(src, variant) for src in SOURCES]


def _command(target, defines):
    """The compile commands (one per source) and the link command of one library variant."""
    variant = os.path.basename(target)[:-3]
    return [_compile_command(src, variant, defines) for src in SOURCES], _link_command(target, variant)


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
    # Every stale object of every variant compiles in parallel (an object is stale when its source, a header or
    # this file is newer, or a forced build); each variant links once its objects are done.
    newest_shared = max(os.path.getmtime(p) for p in HEADERS + [__file__])
    procs = []
    for target, defines in jobs:
        compiles, link = _command(target, defines)
        os.makedirs(os.path.dirname(_object(SOURCES[0], os.path.basename(target)[:-3])), exist_ok=True)
        for cmd in compiles:
            obj, src = cmd[cmd.index("-o") + 1], cmd[-1]
            if not force and os.path.exists(obj) and \
                    os.path.getmtime(obj) > max(newest_shared, os.path.getmtime(src)):
                continue
            procs.append((target, cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    logs = {}
    for target, _ in jobs:
        logs[target] = []
    for target, cmd, proc in procs:
        out = proc.communicate()[0]
        logs[target].append(" ".join(cmd) + "\n" + out)
        if proc.returncode != 0:
            sys.stderr.write(out)
            raise RuntimeError(f"nvcc failed compiling {cmd[-1]} for {os.path.basename(target)}")
    for target, defines in jobs:
        link = _command(target, defines)[1]
        res = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        logs[target].append(" ".join(link) + "\n" + res.stdout)
        if res.returncode != 0:
            sys.stderr.write(res.stdout)
            raise RuntimeError(f"nvcc failed linking {os.path.basename(target)}")
        if target == OUT:
            with open(os.path.join(HERE, "build.log"), "w") as f:
                f.write("\n".join(logs[target]))
        if verbose:
            sys.stderr.write("\n".join(logs[target]))
    return jobs[0][0]


if __name__ == "__main__":
    if "--checked" in sys.argv:
        print(build(force=True, out=sys.argv[sys.argv.index("--checked") + 1], defines=("TF_DEVICE_CHECKS",)))
    else:
        print(build(force="--force" in sys.argv, verbose=True))
