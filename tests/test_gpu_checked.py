"""Runs a large batch on the index-checking build of the library (every device index range-checked, the
first failure recorded instead of used) and requires that no check fires and that the results match the
normal build bit for bit. This stands in for a device memory checker, which this GPU pool does not offer."""
import os
import subprocess
import sys

import numpy as np
import pytest

from twofold_b200 import build

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, {root!r})
from twofold_b200 import scenes
from twofold_b200.world import Batch
sc = {scene}
b = Batch.from_scene(sc)
b.step_checked(sc.dt, {steps})
b.step_checked(sc.dt, 8, graph=True)
s = b.states()
np.savez({out!r}, **s)
"""

UNEVEN = "scenes.config4(n_worlds=1024)"
# Joints, contacts solved a level at a time (planar piles), the bucketed continuous pass of a large world.
MIXED = ("scenes.Scene('mixed', [scenes.jointed(0), scenes.jointed(2), "
         "scenes.planar(n=48, cols=8, spheres=4, sphere_height=(3.0, 8.0), seed=0), "
         "scenes.planar(n=2048, cols=32, spheres=16, sphere_height=(3.0, 8.0), seed=1)])")


def _run(lib, out, scene=UNEVEN, steps=40):
    env = dict(os.environ)
    if lib:
        env["TWOFOLD_B200_LIB"] = lib
    code = SCRIPT.format(root=ROOT, scene=scene, steps=steps, out=out)
    res = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    return np.load(out)


@pytest.mark.skipif(not os.path.exists(build.CHECKED_OUT), reason="checked build missing")
def test_checked_build_finds_no_bad_index_and_matches(tmp_path):
    checked = _run(build.CHECKED_OUT, str(tmp_path / "checked.npz"))
    normal = _run(None, str(tmp_path / "normal.npz"))
    for k in ("p", "q", "v", "w"):
        assert np.array_equal(checked[k].view(np.uint32), normal[k].view(np.uint32)), k


@pytest.mark.skipif(not os.path.exists(build.CHECKED_OUT), reason="checked build missing")
def test_checked_build_on_joints_levels_and_large_sweeps(tmp_path):
    """The same check over jointed worlds, planar piles (their contacts solved a level at a time) and a
    2048-body planar world whose continuous pass buckets its swept bounds, in one batch."""
    checked = _run(build.CHECKED_OUT, str(tmp_path / "checked.npz"), scene=MIXED, steps=60)
    normal = _run(None, str(tmp_path / "normal.npz"), scene=MIXED, steps=60)
    for k in ("p", "q", "v", "w"):
        assert np.array_equal(checked[k].view(np.uint32), normal[k].view(np.uint32)), k
