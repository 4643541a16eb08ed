"""Parity of the B200 step against the oracle (the reference's own World::step) on identical input.

Bars, per the contact pipeline's contract: the broadphase pair list, manifold point counts and feature ids
match bit for bit; positions, rotations and velocities after one step agree within 1e-5 (normwise
relative); repeated GPU runs are bit-identical. Longer runs check the same tolerance, which only holds if
every step matches closely.
"""
import numpy as np
import pytest

import reference as R
from parity import contact_table, first_difference, rel_err, state_errors, states_bitwise_equal
from twofold_b200 import scenes
from twofold_b200.world import Batch

pytestmark = pytest.mark.gpu

TOL = 1e-5

needs_oracle = pytest.mark.skipif(not R.available(), reason="oracle library not built")


def _compare_world(batch, wi, ref, label):
    mine = batch.world_states(wi)
    theirs = ref.states()
    errs = state_errors(mine, theirs)
    assert max(errs.values()) <= TOL, f"{label}: state error {errs}"
    return errs


def _check_pairs_and_manifolds(batch, wi, ref, label):
    cm, cr = batch.candidates(wi), ref.candidates()
    assert np.array_equal(cm, cr), f"{label}: candidate pairs differ at {first_difference(list(cm), list(cr))}"
    em, pm = contact_table(batch.contacts(wi, mode=1))
    er, pr = contact_table(ref.contacts(mode=1))
    assert em == er, f"{label}: contact keys/counts/features differ at {first_difference(em, er)}"
    assert rel_err(pm, pr) <= TOL, f"{label}: contact points differ by {rel_err(pm, pr)}"


@needs_oracle
@pytest.mark.parametrize("kind", ["box_on_ground", "sphere_on_ground", "boxes"])
@pytest.mark.parametrize("steps", [1, 30])
def test_small_worlds_match_reference(kind, steps):
    w = scenes.single(kind)
    sc = scenes.Scene(kind, [w])
    b = Batch.from_scene(sc)
    r = R.RefWorld(w, sc.settings)
    for _ in range(steps):
        b.step_checked(sc.dt)
        r.step(sc.dt)
    _check_pairs_and_manifolds(b, 0, r, f"{kind} after {steps}")
    _compare_world(b, 0, r, f"{kind} after {steps}")


@needs_oracle
@pytest.mark.parametrize("seed", range(4))
def test_tumbling_boxes_match_reference(seed):
    w = scenes.single("boxes", n=12, seed=seed)
    sc = scenes.Scene("boxes", [w])
    b = Batch.from_scene(sc)
    r = R.RefWorld(w, sc.settings)
    for s in range(120):
        b.step_checked(sc.dt)
        r.step(sc.dt)
        if s % 10 == 9:
            _check_pairs_and_manifolds(b, 0, r, f"boxes seed {seed} step {s + 1}")
            _compare_world(b, 0, r, f"boxes seed {seed} step {s + 1}")


@needs_oracle
@pytest.mark.parametrize("seed", range(3))
def test_prism_worlds_match_reference(seed):
    """Prisms (general polyhedra: face and edge queries with the Gauss-map pruning, clipping) against boxes,
    prisms and a half-space, including outlines the cleaning rewrote."""
    w = scenes.prisms(n=24, seed=seed)
    sc = scenes.Scene("prisms", [w])
    b = Batch.from_scene(sc)
    r = R.RefWorld(w, sc.settings)
    for s in range(90):
        b.step_checked(sc.dt)
        r.step(sc.dt)
        if s in (0, 29, 59, 89):
            _check_pairs_and_manifolds(b, 0, r, f"prisms seed {seed} step {s + 1}")
            _compare_world(b, 0, r, f"prisms seed {seed} step {s + 1}")


@needs_oracle
@pytest.mark.parametrize("seed", range(3))
def test_hull_worlds_match_reference(seed):
    """Hulls (computeHull's polyhedra, up to 16 vertices) against hulls, boxes, spheres and a half-space. The
    degenerate clouds (thickened to slabs a few millimetres thin) are in the continuous-pass test."""
    w = scenes.hulls(n=24, seed=seed, degenerate=False)
    sc = scenes.Scene("hulls", [w])
    b = Batch.from_scene(sc)
    r = R.RefWorld(w, sc.settings)
    for s in range(90):
        b.step_checked(sc.dt)
        r.step(sc.dt)
        if s in (0, 29, 59, 89):
            _check_pairs_and_manifolds(b, 0, r, f"hulls seed {seed} step {s + 1}")
            _compare_world(b, 0, r, f"hulls seed {seed} step {s + 1}")


@needs_oracle
@pytest.mark.parametrize("floor,seed,restitution",
                         [("box", 1, 0.0), ("box", 3, 0.2), ("halfspace", 3, 0.0), ("halfspace", 7, 0.2)])
def test_planar_worlds_match_reference(floor, seed, restitution):
    """Boxes and prisms locked to one plane (polygon profiles, half-plane profiles of a half-space floor, the
    kept poses, the planar rows of the solver and restitution), free spheres falling among them (3D pairs
    with planar bodies), a static container, and sleep: 240 steps."""
    w = scenes.planar(n=48, cols=8, spheres=4, sphere_height=(3.0, 8.0), floor=floor, seed=seed,
                      restitution=restitution)
    sc = scenes.Scene("planar", [w])
    b = Batch.from_scene(sc)
    r = R.RefWorld(w, sc.settings)
    for s in range(240):
        b.step_checked(sc.dt)
        r.step(sc.dt)
        if s in (0, 1, 9, 59, 119, 239):
            _check_pairs_and_manifolds(b, 0, r, f"planar {floor} seed {seed} step {s + 1}")
            _compare_world(b, 0, r, f"planar {floor} seed {seed} step {s + 1}")


@needs_oracle
@pytest.mark.parametrize("seed", range(3))
def test_terrain_worlds_match_reference(seed):
    """Spheres, boxes and hulls dropped on a terrain mesh: triangles from the tree, the two-faced triangle
    collisions, edges and corners without their own normal, manifolds grouped by normal into several
    contacts per pair (keys with parts), their reuse, and the refresh of fast pairs with the triangles ruled
    out at the step's start. Pairs, contacts and states are compared along 150 steps, and every step's swept
    pairs and impacts."""
    w = scenes.terrain(cells=16, cell=0.5, cols=4, levels=2, pitch=1.7, top=5.0, seed=seed)
    sc = scenes.Scene("terrain", [w])
    b = Batch.from_scene(sc)
    r = R.RefWorld(w, sc.settings)
    parts = 0
    for s in range(150):
        b.step_checked(sc.dt)
        r.step(sc.dt)
        mine, theirs = b.profile(0), r.profile()
        assert (mine.swept_pairs, mine.impacts) == (theirs.swept_pairs, theirs.impacts), f"terrain {seed} step {s + 1}"
        if s in (0, 1, 10, 30, 60, 90, 120, 149):
            _check_pairs_and_manifolds(b, 0, r, f"terrain seed {seed} step {s + 1}")
            _compare_world(b, 0, r, f"terrain seed {seed} step {s + 1}")
            parts = max(parts, max((c.part for c in r.contacts(mode=1)), default=0))
    assert parts > 0  # some pair met the terrain with more than one group of triangles


@needs_oracle
@pytest.mark.parametrize("kind", ["planar", "terrain"])
def test_big_worlds_match_reference(kind):
    """Worlds of more than 1024 bodies find their body pairs with the sweep along x over the whole grid:
    2048 planar bodies in a container, and 1296 spheres, boxes and hulls on a terrain mesh."""
    if kind == "planar":
        w = scenes.planar(n=2048, cols=32, spheres=16, sphere_height=(3.0, 8.0), seed=1)
    else:
        w = scenes.terrain(cells=48, cell=0.5, cols=12, levels=9, pitch=1.7, top=16.0, seed=1)
    sc = scenes.Scene(kind, [w])
    assert len(w.bodies) > 1024
    b = Batch.from_scene(sc)
    r = R.RefWorld(w, sc.settings)
    for s in range(60):
        b.step_checked(sc.dt)
        r.step(sc.dt)
        if s in (0, 1, 20, 40, 59):
            _check_pairs_and_manifolds(b, 0, r, f"big {kind} step {s + 1}")
            _compare_world(b, 0, r, f"big {kind} step {s + 1}")


@needs_oracle
@pytest.mark.parametrize("kind,seed", [("cylinders", 0), ("cylinders", 1), ("cylinders", 2), ("cylinders", 3),
                                       ("discs", 0), ("discs", 3), ("terrain", 0), ("terrain", 2)])
def test_cylinder_worlds_match_reference(kind, seed):
    """Cylinders against cylinders, boxes, hulls, spheres and a half-space (separating directions, GJK
    directions between rims and edges, the climb in deep overlaps, caps, sides and turned lines); discs
    standing on a plane among planar prisms (circle profiles); cylinders on a terrain mesh. Compared with the
    reference built with correctly rounded libm, so that worlds whose bodies the continuous pass moves are
    held to every step, not just to the first impact."""
    if kind == "cylinders":
        w, steps = scenes.cylinders(24, seed), 120
    elif kind == "discs":
        w, steps = scenes.planar(n=48, cols=8, spheres=4, sphere_height=(3.0, 8.0), seed=seed, discs=True), 240
    else:
        w, steps = scenes.terrain(cells=16, cell=0.5, cols=4, levels=2, pitch=1.7, top=5.0, seed=seed,
                                  cylinders=True), 150
    sc = scenes.Scene(kind, [w])
    b = Batch.from_scene(sc)
    r = R.RefWorld(w, sc.settings, lib=R.ROUNDED_LIB)
    for s in range(steps):
        b.step_checked(sc.dt)
        r.step(sc.dt)
        mine, theirs = b.profile(0), r.profile()
        assert (mine.swept_pairs, mine.impacts) == (theirs.swept_pairs, theirs.impacts), f"{kind} {seed} step {s + 1}"
        if s in (0, 1, 10, 30, 60, 90, steps - 1) or theirs.impacts:
            _check_pairs_and_manifolds(b, 0, r, f"{kind} seed {seed} step {s + 1}")
            _compare_world(b, 0, r, f"{kind} seed {seed} step {s + 1}")


def _continuous_world(kind, seed):
    if kind == "hulls":
        return scenes.hulls(n=24, seed=seed, degenerate=True)
    if kind.startswith("terrain"):
        return scenes.terrain(cells=16, cell=0.5, cols=4, levels=2, pitch=1.7, top=5.0, seed=seed, flat_hulls=True,
                              spin=0.3 if kind == "terrain_spin" else 0.0)
    return scenes.planar(n=48, cols=8, spheres=4, sphere_height=(3.0, 8.0), floor=kind, seed=seed)


CONTINUOUS_CASES = [("hulls", 0, 90), ("hulls", 1, 90), ("hulls", 2, 90), ("box", 0, 120), ("box", 2, 120),
                    ("halfspace", 5, 150), ("terrain", 0, 130), ("terrain", 3, 110), ("terrain_spin", 2, 70),
                    ("terrain_spin", 3, 70)]


@needs_oracle
@pytest.mark.parametrize("kind,seed,steps", CONTINUOUS_CASES)
def test_continuous_pass_matches_reference(kind, seed, steps):
    """Worlds where the reference's continuous pass moves bodies back: hulls thickened to slabs a few
    millimetres thin (alone, or on a terrain mesh, static or turning, whose triangles they are swept
    against), and planar piles whose prisms are pushed further in a step than they were moving. Swept pairs
    and impacts match step by step, and states and contacts within 1e-5, up to three steps after the first
    impact: from there the host's float sinf, cosf and atan2f, which round some arguments the other way,
    make the two runs drift apart by ulps that the pile then amplifies (the next test pins the rest)."""
    w = _continuous_world(kind, seed)
    sc = scenes.Scene(kind, [w])
    b = Batch.from_scene(sc)
    r = R.RefWorld(w, sc.settings)
    first = None
    for s in range(steps):
        b.step_checked(sc.dt)
        r.step(sc.dt)
        mine, theirs = b.profile(0), r.profile()
        assert (mine.swept_pairs, mine.impacts) == (theirs.swept_pairs, theirs.impacts), f"{kind} {seed} step {s + 1}"
        if theirs.impacts and first is None:
            first = s
        if first is None and s in (0, steps // 2) or first is not None and s <= first + 3:
            _check_pairs_and_manifolds(b, 0, r, f"{kind} seed {seed} step {s + 1}")
            _compare_world(b, 0, r, f"{kind} seed {seed} step {s + 1}")
        if first is not None and s > first + 3:
            break
    assert first is not None


@pytest.mark.skipif(not R.available(R.ROUNDED_LIB), reason="oracle library not built")
@pytest.mark.parametrize("kind,seed,steps", CONTINUOUS_CASES)
def test_continuous_pass_is_bit_identical_with_rounded_libm(kind, seed, steps):
    """The same worlds against the reference built with correctly rounded sinf, cosf, atan2f and asinf (the
    values this library's continuous pass uses): every step's states bit for bit, swept pairs and impacts,
    and pairs and contacts along the whole run."""
    w = _continuous_world(kind, seed)
    sc = scenes.Scene(kind, [w])
    b = Batch.from_scene(sc)
    r = R.RefWorld(w, sc.settings, lib=R.ROUNDED_LIB)
    impacts = 0
    for s in range(steps):
        b.step_checked(sc.dt)
        r.step(sc.dt)
        mine, theirs = b.profile(0), r.profile()
        assert (mine.swept_pairs, mine.impacts) == (theirs.swept_pairs, theirs.impacts), f"{kind} {seed} step {s + 1}"
        impacts += theirs.impacts
        assert states_bitwise_equal(b.world_states(0), r.states()), f"{kind} seed {seed} step {s + 1}"
        if theirs.impacts or s % 30 == 29:
            _check_pairs_and_manifolds(b, 0, r, f"{kind} seed {seed} step {s + 1}")
    assert impacts > 0


@needs_oracle
def test_pyramid_one_step_matches_reference():
    sc = scenes.config1()
    b = Batch.from_scene(sc)
    r = R.RefWorld(sc.worlds[0], sc.settings)
    b.step_checked(sc.dt)
    r.step(sc.dt)
    assert len(b.candidates(0)) == 590
    _check_pairs_and_manifolds(b, 0, r, "pyramid step 1")
    _compare_world(b, 0, r, "pyramid step 1")


@needs_oracle
def test_pyramid_full_run_matches_reference():
    sc = scenes.config1()
    b = Batch.from_scene(sc)
    r = R.RefWorld(sc.worlds[0], sc.settings)
    for s in range(sc.steps):
        b.step_checked(sc.dt)
        r.step(sc.dt)
        if s % 50 == 49:
            _check_pairs_and_manifolds(b, 0, r, f"pyramid step {s + 1}")
            _compare_world(b, 0, r, f"pyramid step {s + 1}")


@needs_oracle
@pytest.mark.parametrize("steps", [1, 60])
def test_batched_uneven_worlds_match_reference(steps):
    sc = scenes.config4(n_worlds=24)
    b = Batch.from_scene(sc)
    refs = [R.RefWorld(w, sc.settings) for w in sc.worlds]
    for _ in range(steps):
        b.step_checked(sc.dt)
        for r in refs:
            r.step(sc.dt)
    for wi, r in enumerate(refs):
        _check_pairs_and_manifolds(b, wi, r, f"world {wi} after {steps}")
        _compare_world(b, wi, r, f"world {wi} after {steps}")


@needs_oracle
def test_impact_worlds_match_reference():
    sc = scenes.config5(n_worlds=8)
    b = Batch.from_scene(sc)
    refs = [R.RefWorld(w, sc.settings) for w in sc.worlds]
    for s in range(40):
        b.step_checked(sc.dt)
        for r in refs:
            r.step(sc.dt)
    for wi, r in enumerate(refs):
        _check_pairs_and_manifolds(b, wi, r, f"impact world {wi}")
        _compare_world(b, wi, r, f"impact world {wi}")


def test_repeated_runs_are_bit_identical():
    sc = scenes.config4(n_worlds=16)
    out = []
    for _ in range(2):
        b = Batch.from_scene(sc)
        b.step_checked(sc.dt, 20)
        out.append(b.states())
        b.close()
    assert states_bitwise_equal(out[0], out[1])


def test_graph_replay_matches_direct_launches():
    sc = scenes.config4(n_worlds=16)
    a = Batch.from_scene(sc)
    g = Batch.from_scene(sc)
    a.step_checked(sc.dt, 8)
    g.step_checked(sc.dt, 4, graph=True)
    g.step_checked(sc.dt, 4, graph=True)
    assert states_bitwise_equal(a.states(), g.states())
