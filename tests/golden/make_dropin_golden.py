"""Generates tests/golden/dropin_pyramid.txt, dropin_joints.txt and dropin_setters.txt: the output of
tests/dropin/pyramid_step.cpp, joints_step.cpp and setters_step.cpp built against the reference's own public header and sources (include/twofold/twofold.h,
src/*.cpp) and run with the arguments below. The drop-in test builds the same programs against
include/twofold_b200/world.hpp and compares.

    python tests/golden/make_dropin_golden.py [reference checkout]
"""
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# (program, arguments, golden file)
PROGRAMS = [
    ("pyramid_step.cpp", ["6", "60"], "dropin_pyramid.txt"),
    ("joints_step.cpp", ["60"], "dropin_joints.txt"),
    ("setters_step.cpp", ["160"], "dropin_setters.txt"),
]


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TWOFOLD_REF", "/root/reference")
    sources = sorted(os.path.join(ref, "src", f) for f in os.listdir(os.path.join(ref, "src")) if f.endswith(".cpp"))
    for program, args, golden in PROGRAMS:
        src = os.path.join(ROOT, "tests", "dropin", program)
        out_path = os.path.join(HERE, golden)
        with tempfile.TemporaryDirectory() as tmp:
            exe = os.path.join(tmp, "program_ref")
            subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", f"-I{os.path.join(ref, 'include')}",
                            "-DTWOFOLD_HEADER=<twofold/twofold.h>", src, *sources, "-o", exe], check=True)
            out = subprocess.run([exe, *args], check=True, capture_output=True, text=True).stdout
        with open(out_path, "w") as f:
            f.write(f"# {program} {' '.join(args)} against the reference\n")
            f.write(out)
        print(out_path)


if __name__ == "__main__":
    main()
