"""Host-side scene building (shape cleaning, polyhedra, mass properties, body setup) against the oracle,
bit for bit, on the benchmark scenes. Runs on the CPU."""
import numpy as np
import pytest

import reference as R
from twofold_b200 import abi, scenes
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


def _ragged_mesh():
    """A small mesh with every case the builder cleans: repeated vertices (merged), a non-finite vertex, out of
    range and repeated indices, a sliver, an edge shared by three triangles, open edges and folded neighbours
    both ways."""
    rng = np.random.default_rng(11)
    v, idx = scenes.terrain_mesh(cells=6, cell=0.7, seed=3)
    v = np.concatenate([v, v[:5], [[np.nan, 0, 0], [0.0, 5.0, 0.0], [0.0, 5.0, 1e-7], [1.0, 5.0, 0.0]]]).astype(np.float32)
    n0 = len(v) - 4
    extra = [n0 - 5, n0 - 4, n0 - 3,          # a triangle on the duplicated vertices
             0, 1, n0,                          # a non-finite corner: dropped
             0, 1, 999,                         # out of range: dropped
             2, 2, 3,                           # a repeated corner: dropped
             n0 + 1, n0 + 2, n0 + 3,            # a sliver: dropped
             0, 1, 10, 0, 1, 11]                # the edge 0-1 shared three times
    idx = np.concatenate([idx, np.asarray(extra, np.uint32)])
    v[7, 1] += rng.uniform(0.3, 0.6)           # a sharp fold
    return v, idx


def _soup_mesh(seed):
    """Random triangles over a small grid of vertices (so vertices repeat, edges are shared by one, two or more
    triangles, and some triangles are slivers or repeat a corner), with signed zeros that must merge."""
    rng = np.random.default_rng(seed)
    v = rng.integers(-3, 4, size=(60, 3)).astype(np.float32) * np.float32(0.5)
    v[rng.random(60) < 0.2] *= np.float32(-1.0)
    v[::7, 0] = np.float32(-0.0)
    v[1::7, 0] = np.float32(0.0)
    v[5] = v[2] + np.float32(1e-7)
    idx = rng.integers(0, 60, size=3 * 400).astype(np.uint32)
    return v, idx


@pytest.mark.parametrize("kind", ["terrain", "ragged", "soup0", "soup1", "soup2", "big_terrain"])
def test_meshes_are_built_like_the_reference(kind):
    if kind == "terrain":
        v, idx = scenes.terrain_mesh(cells=32, cell=0.5, seed=1)
    elif kind == "big_terrain":
        v, idx = scenes.terrain_mesh(cells=256, cell=0.5, seed=0)
    elif kind == "ragged":
        v, idx = _ragged_mesh()
    else:
        v, idx = _soup_mesh(int(kind[-1]))
    b = Batch([scenes.single("box_on_ground")])
    mine = b.read_mesh(b.create_mesh(v, idx))
    ref = R.mesh_read(R.mesh_create(v, idx))
    for k in ("vertices", "indices", "normals", "edges", "node_bounds", "node_ranges"):
        assert mine[k].shape == ref[k].shape, k
        assert np.array_equal(mine[k].view(np.uint8), ref[k].view(np.uint8)), k
    assert len(mine["normals"]) > 0


def test_terrain_scene_builds_like_the_reference():
    """Mass, centre and inertia of every body of a small terrain scene (spheres, boxes, hulls over a static
    mesh), and the mesh shape's own bounds."""
    sc = scenes.Scene("terrain", [scenes.terrain(cells=16, cols=4, levels=3, pitch=1.6, top=8.0)])
    _check_masses(sc)


@pytest.mark.parametrize("seed", range(2))
def test_cylinders_are_built_like_the_reference(seed):
    """Cylinder cleaning (thin discs and rods thickened), masses and inertias, among boxes, spheres and hulls."""
    w = scenes.cylinders(24, seed)
    w.shapes["half_height"][3] = 1e-9                      # a flat disc: thickened to a slab
    w.shapes["radius"][6] = 0.0                            # a line: thickened
    _check_masses(scenes.Scene("cylinders", [w]))


@pytest.mark.parametrize("seed", range(3))
def test_joints_are_made_like_the_reference(seed):
    """tf_joint_create restates World::createJoint on the host (src/world.cpp:2221-2333): each joint's anchors,
    axis and value (hinge angle, slider translation, distance, twist) as jointInfo reports them before any step
    match the reference's, which measures angles with correctly rounded atan2 as the device does."""
    w = scenes.jointed(seed)
    b = Batch.from_scene(scenes.Scene("jointed", [w]))
    r = R.RefWorld(w, lib=R.ROUNDED_LIB)
    for k in range(len(w.joints)):
        mine, theirs = b.joint_info(0, abi.tf_id(k, 0)), r.joint_info(abi.tf_id(k, 0))
        assert (mine.type, mine.body_a, mine.body_b, mine.broken) == (theirs.type, theirs.body_a, theirs.body_b, theirs.broken)
        for f in ("anchor_a", "anchor_b", "axis"):
            assert list(getattr(mine, f)) == list(getattr(theirs, f)), f"joint {k} {f}"
        assert mine.value == theirs.value, f"joint {k} value {mine.value} vs {theirs.value}"


def test_joints_refuse_what_this_build_does_not_run():
    """Joining a body to itself or to a missing body is invalid, as in the reference; a bad kind is rejected."""
    w = scenes.jointed(0)
    b = Batch.from_scene(scenes.Scene("jointed", [w]))
    with pytest.raises(RuntimeError):
        b.joint_create(0, abi.joint_desc(abi.TF_JOINT_POINT, abi.tf_id(1, 0), abi.tf_id(1, 0)))
    with pytest.raises(RuntimeError):
        b.joint_create(0, abi.joint_desc(abi.TF_JOINT_POINT, abi.tf_id(10_000, 0)))
    with pytest.raises(RuntimeError):
        b.joint_create(0, abi.joint_desc(9, abi.tf_id(1, 0)))


def _clouds():
    """Point clouds that take every path of the hull builder: random balls and boxes, points on a sphere (many
    nearly coplanar faces to merge), grids (exactly coplanar faces and ties between equal distances), repeated
    points, flat, collinear and single-point clouds (thickened), far from the origin, and non-finite points."""
    rng = np.random.default_rng(5)
    out = []
    for n in (4, 5, 8, 16, 40, 120):
        out.append(rng.normal(size=(n, 3)))
        out.append(rng.uniform(-1.0, 1.0, size=(n, 3)) * [2.0, 0.3, 1.0])
        s = rng.normal(size=(n, 3))
        out.append(s / np.linalg.norm(s, axis=1, keepdims=True))
    g = np.stack(np.meshgrid(*[np.arange(3.0)] * 3, indexing="ij"), -1).reshape(-1, 3)
    out.append(g)
    out.append(np.concatenate([g, g[::-1], g[:5]]))
    out.append(g * [1.0, 1.0, 0.0])                        # flat
    out.append(np.outer(np.linspace(0, 1, 9), [1.0, 2.0, 3.0]))  # collinear
    out.append(np.zeros((6, 3)))                           # one point
    out.append(rng.normal(size=(30, 3)) + 1e4)             # far from the origin
    nf = rng.normal(size=(20, 3))
    nf[3, 1] = np.nan
    nf[7, 2] = np.inf
    out.append(nf)
    return [np.asarray(c, np.float32) for c in out]


@pytest.mark.parametrize("max_vertices", [4, 6, 16, 64])
def test_hull_builder_matches_the_reference(max_vertices):
    """tf_hull_compute against the reference's computeHull on the same cloud: the same vertices in the same
    order, bit for bit, and the same face loops."""
    for k, cloud in enumerate(_clouds()):
        mv, mf = abi.hull_compute(cloud, max_vertices)
        rv, rf = R.hull_compute(cloud, max_vertices)
        assert mv.shape == rv.shape and np.array_equal(mv.view(np.uint32), rv.view(np.uint32)), f"cloud {k}: vertices"
        assert mf == rf, f"cloud {k}: faces"
