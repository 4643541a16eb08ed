"""Parity at the sizes the benchmark configurations are quoted on, against the oracle (the reference's own
World::step compiled here).

* Terrain: 32,768 spheres, boxes and hulls over a 256 x 256-cell terrain mesh (131,072 triangles).
* Planar pile: 16,384 bodies locked to one plane, 256 free spheres and the static container.
* Batched uneven worlds: all 4096 worlds, one step and 25 steps.
* Differentiable impact: 1024 walls hit by a sphere, 120 steps, compared every 20 steps.

The first step of each is compared with the reference as built (its platform float functions): candidate
pairs, contact keys, parts, point counts and feature ids exactly, contact points and states within 1e-5. Longer
runs are compared with the reference built with correctly rounded sinf, cosf, atan2f and asinf, the values the
device's continuous pass uses, so that worlds whose bodies the continuous pass moves are held to every step
(the platform's float functions round some arguments the other way by one ulp, which piles amplify).
"""
import numpy as np
import pytest

import reference as R
from parity import contact_table, first_difference, rel_err, state_errors
from twofold_b200 import scenes
from twofold_b200.world import Batch

pytestmark = pytest.mark.gpu

TOL = 1e-5

needs_oracle = pytest.mark.skipif(not (R.available() and R.available(R.ROUNDED_LIB)),
                                  reason="oracle library not built")


def _check(batch, wi, ref, label):
    cm, cr = batch.candidates(wi), ref.candidates()
    assert np.array_equal(cm, cr), f"{label}: candidate pairs differ at {first_difference(list(cm), list(cr))}"
    em, pm = contact_table(batch.contacts(wi, mode=1))
    er, pr = contact_table(ref.contacts(mode=1))
    assert em == er, f"{label}: contact keys/counts/features differ at {first_difference(em, er)}"
    assert rel_err(pm, pr) <= TOL, f"{label}: contact points differ by {rel_err(pm, pr)}"
    errs = state_errors(batch.world_states(wi), ref.states())
    assert max(errs.values()) <= TOL, f"{label}: state error {errs}"


def _single_world(sc, checks):
    """One world: step 1 against the reference as built, then every step against the rounded build (swept
    pairs and impacts), with full comparisons at the steps in `checks`."""
    b = Batch.from_scene(sc)
    r1 = R.RefWorld(sc.worlds[0], sc.settings)
    rr = R.RefWorld(sc.worlds[0], sc.settings, lib=R.ROUNDED_LIB)
    b.step_checked(sc.dt)
    r1.step(sc.dt)
    rr.step(sc.dt)
    _check(b, 0, r1, f"{sc.name} step 1")
    del r1
    for s in range(1, max(checks)):
        b.step_checked(sc.dt)
        rr.step(sc.dt)
        mine, theirs = b.profile(0), rr.profile()
        assert (mine.swept_pairs, mine.impacts) == (theirs.swept_pairs, theirs.impacts), f"{sc.name} step {s + 1}"
        if s + 1 in checks:
            _check(b, 0, rr, f"{sc.name} step {s + 1}")
    return b


@needs_oracle
def test_terrain_full_size_matches_reference():
    sc = scenes.config2()
    assert len(sc.worlds[0].bodies) == 32768 + 1
    _single_world(sc, checks=(1, 10, 21))


@needs_oracle
def test_planar_pile_full_size_matches_reference():
    sc = scenes.config3()
    _single_world(sc, checks=(1, 30, 60))


@needs_oracle
def test_all_4096_uneven_worlds_match_reference():
    sc = scenes.config4()
    assert len(sc.worlds) == 4096
    b = Batch.from_scene(sc)
    refs = [R.RefWorld(w, sc.settings) for w in sc.worlds]
    threads = R.hardware_threads()
    b.step_checked(sc.dt)
    R.step_parallel(refs, sc.dt, 1, threads)
    for wi, r in enumerate(refs):
        _check(b, wi, r, f"world {wi} step 1")
    b.step_checked(sc.dt, 24, graph=True)
    R.step_parallel(refs, sc.dt, 24, threads)
    worst = 0.0
    for wi, r in enumerate(refs):
        errs = state_errors(b.world_states(wi), r.states())
        worst = max(worst, max(errs.values()))
        assert np.array_equal(b.candidates(wi), r.candidates()), f"world {wi} step 25: candidate pairs differ"
    assert worst <= TOL, f"step 25: state error {worst}"


@needs_oracle
def test_all_1024_impact_worlds_match_reference_for_120_steps():
    sc = scenes.config5()
    assert len(sc.worlds) == 1024
    b = Batch.from_scene(sc)
    first = [R.RefWorld(w, sc.settings) for w in sc.worlds]
    refs = [R.RefWorld(w, sc.settings, lib=R.ROUNDED_LIB) for w in sc.worlds]
    threads = R.hardware_threads()
    b.step_checked(sc.dt)
    R.step_parallel(first, sc.dt, 1, threads)
    R.step_parallel(refs, sc.dt, 1, threads)
    for wi, r in enumerate(first):
        _check(b, wi, r, f"impact world {wi} step 1")
    del first
    done = 1
    for upto in (20, 40, 60, 80, 100, 120):
        b.step_checked(sc.dt, upto - done, graph=True)
        R.step_parallel(refs, sc.dt, upto - done, threads)
        done = upto
        for wi, r in enumerate(refs):
            _check(b, wi, r, f"impact world {wi} step {upto}")
