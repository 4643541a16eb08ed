"""Generates tests/golden/dropin_pyramid.txt: the output of tests/dropin/pyramid_step.cpp built against the
reference's own public header and sources (include/twofold/twofold.h, src/*.cpp) and run with its default
arguments. The drop-in test builds the same program against include/twofold_b200/world.hpp and compares.

    python tests/golden/make_dropin_golden.py [reference checkout]
"""
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PROGRAM = os.path.join(ROOT, "tests", "dropin", "pyramid_step.cpp")
OUT = os.path.join(HERE, "dropin_pyramid.txt")
ARGS = ["6", "60"]


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    sources = sorted(os.path.join(ref, "src", f) for f in os.listdir(os.path.join(ref, "src")) if f.endswith(".cpp"))
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "pyramid_ref")
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", f"-I{os.path.join(ref, 'include')}",
                        "-DTWOFOLD_HEADER=<twofold/twofold.h>", PROGRAM, *sources, "-o", exe], check=True)
        out = subprocess.run([exe, *ARGS], check=True, capture_output=True, text=True).stdout
    with open(OUT, "w") as f:
        f.write(f"# {os.path.basename(PROGRAM)} {' '.join(ARGS)} against the reference\n")
        f.write(out)
    print(OUT)


if __name__ == "__main__":
    main()
