"""The oracle pinned against the reference's own known answers.

The oracle is the reference compiled from its sources (oracle/Makefile). These tests check that build
reproduces what the reference's test suite asserts (tests/test_world.cpp) and the committed golden vectors,
so a mis-built oracle cannot silently anchor the GPU parity tests.
"""
import os

import numpy as np
import pytest

import behaviour
import reference as R
from twofold_b200 import scenes

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle library not built")

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_mass_of_box_matches_reference_known_answer():
    """tests/test_world.cpp:68-94: a 1 x 2 x 3 box of density 2 weighs 12 kg."""
    b, s = scenes._bodies(1), scenes._shapes(1)
    s["half_extents"][0] = (0.5, 1.0, 1.5)
    s["density"][0] = 2.0
    r = R.RefWorld(scenes.World(b, s, np.arange(1)))
    m, c, i = r.mass(0)
    assert abs(m - 12.0) <= 1e-4
    assert abs(i[0, 0] - 12.0 * (4.0 + 9.0) / 12.0) <= 1e-3
    assert abs(i[2, 2] - 12.0 * (1.0 + 4.0) / 12.0) <= 1e-3
    assert abs(i[0, 1]) <= 1e-4


@pytest.mark.parametrize("name", sorted(behaviour.SCENARIOS))
def test_reference_known_answers(name):
    w, steps, check = behaviour.SCENARIOS[name]()
    r = R.RefWorld(w)
    r.step(behaviour.DT, steps)
    check(r.states(), r.contacts(mode=1))


def test_bounce_with_full_restitution():
    w, steps, _ = behaviour.bounce_with_full_restitution()
    r = R.RefWorld(w)
    landed, peak = False, 0.0
    for _ in range(steps):
        r.step(behaviour.DT)
        y = r.states()["p"][1, 1]
        landed = landed or y < 0.6
        if landed:
            peak = max(peak, y)
    assert landed and peak > 2.6


def test_identical_runs_match_exactly():
    """tests/test_world.cpp:523-551."""
    w, steps, _ = behaviour.mixed_column()
    outs = []
    for _ in range(2):
        r = R.RefWorld(w)
        r.step(behaviour.DT, steps)
        outs.append(r.states())
    for k in ("p", "q"):
        assert np.array_equal(outs[0][k], outs[1][k])


def test_copied_world_steps_identically():
    """tests/test_world.cpp:609-625."""
    w, _, _ = behaviour.mixed_column()
    r = R.RefWorld(w)
    r.step(behaviour.DT, 30)
    c = r.copy()
    r.step(behaviour.DT, 60)
    c.step(behaviour.DT, 60)
    a, b = r.states(), c.states()
    for k in ("p", "q", "v", "w"):
        assert np.array_equal(a[k], b[k])


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "golden.npz")), reason="no golden vectors")
def test_oracle_reproduces_golden_vectors():
    import golden.make_golden as mg

    g = np.load(os.path.join(GOLDEN, "golden.npz"))
    for name, run in mg.CASES.items():
        got = run()
        for key, value in got.items():
            ref = g[f"{name}/{key}"]
            assert ref.dtype == value.dtype and np.array_equal(ref, value), f"{name}/{key} differs from golden"
