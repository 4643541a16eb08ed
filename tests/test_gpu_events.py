"""Contact and hit events (World::contactEvents, World::hitEvents; src/world.cpp:963-981 for pairs the
narrowphase drops, :1424-1468 for the end-of-step report) and the step profile's touching-contact count,
through the C ABI, against the oracle after every step.

Bars: the contact events (shapes, bodies, begin or end, order) and the hits' pairs are identical; hit
points, normals and speeds agree within 1e-5 normwise relative; touching counts are equal.
"""
import numpy as np
import pytest

import reference as R
from parity import rel_err
from twofold_b200 import scenes
from twofold_b200.world import Batch

pytestmark = pytest.mark.gpu

TOL = 1e-5

needs_oracle = pytest.mark.skipif(not R.available(), reason="oracle library not built")


def _compare_events(batch, wi, ref, label):
    em, er = batch.contact_events(wi), ref.contact_events()
    assert em == er, f"{label}: contact events differ:\n{em}\n{er}"
    hm, hr = batch.hit_events(wi), ref.hit_events()
    assert [h[:4] for h in hm] == [h[:4] for h in hr], f"{label}: hit pairs differ:\n{hm}\n{hr}"
    if hr:
        pm = np.array([np.concatenate([h[4], h[5], [h[6]]]) for h in hm])
        pr = np.array([np.concatenate([h[4], h[5], [h[6]]]) for h in hr])
        assert rel_err(pm, pr) <= TOL, f"{label}: hit points, normals or speeds differ by {rel_err(pm, pr)}"
    tm, tr = batch.profile(wi).touching_contacts, ref.profile().touching_contacts
    assert tm == tr, f"{label}: touching contacts {tm} vs {tr}"
    return sum(e[4] for e in er), sum(not e[4] for e in er), len(hr)


def _run(sc, steps, lib=R.REF_LIB):
    """Steps every world of the scene on both sides and compares the events after each step; returns the
    totals of begun, ended and hit events over all worlds and steps."""
    b = Batch.from_scene(sc)
    refs = [R.RefWorld(w, sc.settings, lib=lib) for w in sc.worlds]
    totals = np.zeros(3, np.int64)
    for s in range(steps):
        b.step_checked(sc.dt)
        for wi, r in enumerate(refs):
            r.step(sc.dt)
            totals += _compare_events(b, wi, r, f"{sc.name} world {wi} step {s + 1}")
    return totals


@needs_oracle
@pytest.mark.parametrize("seed", range(3))
def test_falling_boxes_report_the_reference_events(seed):
    """Boxes dropped in a column onto a floor: pairs begin as they land, hits above 1 m/s, ends as they
    tumble apart."""
    sc = scenes.Scene("boxes", [scenes.single("boxes", n=12, seed=seed)])
    began, ended, hits = _run(sc, 120)
    assert began > 0 and hits > 0


@needs_oracle
def test_impact_walls_report_the_reference_events():
    """A sphere at about 10 m/s through a wall of boxes, in a batch of worlds: hits, and pairs that end as the
    wall breaks."""
    sc = scenes.config5(n_worlds=4)
    began, ended, hits = _run(sc, 60)
    assert began > 0 and ended > 0 and hits > 0


@needs_oracle
def test_uneven_worlds_report_the_reference_events():
    """Batched uneven worlds with restitution: bounces end pairs and begin them again; sleeping pairs keep
    their last report."""
    sc = scenes.config4(n_worlds=12, max_bodies=96)
    began, ended, hits = _run(sc, 150)
    assert began > 0 and ended > 0 and hits > 0


@needs_oracle
def test_planar_and_terrain_worlds_report_the_reference_events():
    """A planar pile (polygon and half-plane pairs) and a terrain mesh (pairs made of several contacts, one
    per group of triangle normals), against the reference built with correctly rounded libm."""
    planar = scenes.Scene("planar", [scenes.planar(n=48, cols=8, spheres=4, sphere_height=(3.0, 8.0), seed=0)])
    began, ended, hits = _run(planar, 150, lib=R.ROUNDED_LIB)
    assert began > 0
    terrain = scenes.Scene("terrain", [scenes.terrain(cells=16, cell=0.5, cols=4, levels=2, pitch=1.7, top=5.0,
                                                      seed=0)])
    began, ended, hits = _run(terrain, 120, lib=R.ROUNDED_LIB)
    assert began > 0 and hits > 0


@needs_oracle
def test_jointed_worlds_report_the_reference_events():
    """Joined pairs never collide, so they make no events; jointed chains and doors touch the ground and the
    loose boxes dropped on them."""
    sc = scenes.Scene("jointed", [scenes.jointed(0), scenes.jointed(1)])
    began, ended, hits = _run(sc, 120, lib=R.ROUNDED_LIB)
    assert began > 0 and hits > 0
