"""Host-side scene building (shape cleaning, polyhedra, mass properties, body setup) against the oracle,
bit for bit, on the benchmark scenes. Runs on the CPU."""
import numpy as np
import pytest

import reference as R
from twofold_b200 import scenes
from twofold_b200.world import Batch

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle library not built")


def _check_masses(scene):
    b = Batch.from_scene(scene)
    for wi, w in enumerate(scene.worlds):
        r = R.RefWorld(w, scene.settings)
        for i in range(len(w.bodies)):
            m1, c1, i1 = b.mass(wi, i)
            m2, c2, i2 = r.mass(i)
            assert np.float32(m1) == np.float32(m2), (wi, i)
            assert np.array_equal(c1.view(np.uint32), c2.view(np.uint32)), (wi, i)
            assert np.array_equal(i1.view(np.uint32), i2.view(np.uint32)), (wi, i)
        # Initial poses and velocities after the reference's normalisation and lock projection.
        s1, s2 = b.world_states(wi), r.states()
        for k in ("p", "q", "v", "w", "awake"):
            assert np.array_equal(s1[k], s2[k]), (wi, k)


def test_pyramid_masses_bit_identical():
    _check_masses(scenes.config1())


def test_uneven_world_masses_bit_identical():
    _check_masses(scenes.config4(n_worlds=12))


def test_impact_world_masses_bit_identical():
    _check_masses(scenes.config5(n_worlds=3))


def test_odd_box_sizes_are_cleaned_like_the_reference():
    """Zero, negative and non-finite half extents and radii (src/shape.cpp:68-97)."""
    w = scenes.single("boxes", n=6, seed=5)
    w.shapes["half_extents"][1] = (0.0, 0.5, 0.5)
    w.shapes["half_extents"][2] = (-0.3, 0.2, 0.4)
    w.shapes["half_extents"][3] = (np.inf, 0.2, 0.4)
    w.shapes["geometry"][4] = 0  # sphere
    w.shapes["radius"][4] = 0.0
    _check_masses(scenes.Scene("odd", [w]))


def test_prism_outlines_are_cleaned_like_the_reference():
    """Prisms with clockwise, repeated, collinear and flat outlines (src/shape.cpp:13-130)."""
    _check_masses(scenes.Scene("prisms", [scenes.prisms(n=40, seed=s) for s in range(3)]))


def test_hulls_are_built_like_the_reference():
    """computeHull (src/hull.cpp) restated: vertex and face order decide the masses' float sums, so equal bits
    mean equal hulls; flat, collinear, single-point and repeated clouds included."""
    _check_masses(scenes.Scene("hulls", [scenes.hulls(n=48, seed=s) for s in range(3)]))


def test_hull_vertex_limits_are_kept_like_the_reference():
    _check_masses(scenes.Scene("hulls", [scenes.hulls(n=30, seed=7, max_vertices=m) for m in (4, 6, 8, 64)]))
