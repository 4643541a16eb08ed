"""Joints in the step (src/joint.cpp, src/world.cpp:1545-1560, 1623-1691, 2221-2333) against the oracle, through
the C ABI: every joint kind with its limits, motor, spring, friction and break limits, joined to the world and
to bodies, a kinematic end, a locked end, joined pairs that do not collide, and islands that fall asleep
through their joints.

Bars: body states within 1e-5 normwise relative after every step that is checked; candidate pairs and
manifolds identical; each joint's value, force and torque within 1e-5 and its broken flag equal; the joints
that broke in each step identical. The oracle is the reference built with correctly rounded libm, since joints
measure angles with atan2 and asin (hinge angles, twist, swing cones).
"""
import numpy as np
import pytest

import reference as R
from parity import contact_table, first_difference, rel_err, state_errors
from twofold_b200 import abi, scenes
from twofold_b200.world import Batch

pytestmark = pytest.mark.gpu

TOL = 1e-5

needs_oracle = pytest.mark.skipif(not R.available(R.ROUNDED_LIB), reason="oracle library not built")


def _joint_rows(infos):
    return np.array([[i.value, *i.force, *i.torque, *i.anchor_a, *i.anchor_b, *i.axis] for i in infos], np.float64)


def _compare(b, wi, r, n_joints, label):
    errs = state_errors(b.world_states(wi), r.states())
    assert max(errs.values()) <= TOL, f"{label}: state error {errs}"
    mine = [b.joint_info(wi, abi.tf_id(k, 0)) for k in range(n_joints)]
    theirs = [r.joint_info(abi.tf_id(k, 0)) for k in range(n_joints)]
    assert [(i.type, i.body_a, i.body_b, i.broken) for i in mine] == \
        [(i.type, i.body_a, i.body_b, i.broken) for i in theirs], f"{label}: joint kinds, ends or broken flags differ"
    # Values, forces and torques per joint: each row is compared on its own scale.
    for k, (m, t) in enumerate(zip(_joint_rows(mine), _joint_rows(theirs))):
        assert rel_err(m[None, :], t[None, :]) <= TOL, f"{label}: joint {k} differs by {rel_err(m[None, :], t[None, :])}"


@needs_oracle
@pytest.mark.parametrize("seed", range(3))
def test_jointed_world_matches_reference(seed):
    w = scenes.jointed(seed)
    sc = scenes.Scene("jointed", [w])
    b = Batch.from_scene(sc)
    r = R.RefWorld(w, sc.settings, lib=R.ROUNDED_LIB)
    nj = len(w.joints)
    broke = 0
    for s in range(240):
        b.step_checked(sc.dt)
        r.step(sc.dt)
        bm, br = b.broken_joints(0), r.broken_joints()
        assert bm == br, f"seed {seed} step {s + 1}: broken joints {bm} vs {br}"
        broke += len(br)
        if s < 10 or s % 10 == 9:
            _compare(b, 0, r, nj, f"seed {seed} step {s + 1}")
        if s in (0, 59, 239):
            cm, cr = b.candidates(0), r.candidates()
            assert np.array_equal(cm, cr), f"seed {seed} step {s + 1}: candidates differ at {first_difference(list(cm), list(cr))}"
            em, _ = contact_table(b.contacts(0, mode=1))
            er, _ = contact_table(r.contacts(mode=1))
            assert em == er, f"seed {seed} step {s + 1}: contacts differ at {first_difference(em, er)}"
    assert broke == 2
    assert b.profile(0).awake_bodies == r.profile().awake_bodies


@needs_oracle
def test_jointed_worlds_in_a_batch_match_reference():
    """Jointed worlds among uneven worlds without joints, in one batch: each matches its own reference world."""
    worlds = [scenes.jointed(3), *scenes.config4(n_worlds=3, max_bodies=64).worlds, scenes.jointed(4)]
    sc = scenes.Scene("mixed", worlds)
    b = Batch.from_scene(sc)
    refs = [R.RefWorld(w, sc.settings, lib=R.ROUNDED_LIB) for w in worlds]
    for s in range(90):
        b.step_checked(sc.dt, 1, graph=True)
        for r in refs:
            r.step(sc.dt)
    for wi, (w, r) in enumerate(zip(worlds, refs)):
        _compare(b, wi, r, len(w.joints), f"world {wi} after 90 steps")


@needs_oracle
def test_joint_changes_match_reference():
    """The joint setters and destroyJoint between steps (src/world.cpp:2341-2397, 399-406): limits, motor,
    spring, friction, swing cone and break limits changed mid-run, a chain link destroyed and its slot reused by
    a new joint, each side stepped on; compared with the reference every 10th step."""
    w = scenes.jointed(1)
    sc = scenes.Scene("jointed", [w])
    b = Batch.from_scene(sc)
    r = R.RefWorld(w, sc.settings, lib=R.ROUNDED_LIB)
    for _ in range(20):
        b.step_checked(sc.dt)
        r.step(sc.dt)
    awake = r.states()["awake"]

    def ends_awake(k):
        info = r.joint_info(abi.tf_id(k, 0))
        return all(e == 0xFFFFFFFF or awake[e] for e in (info.body_a, info.body_b))

    changes = [(6, "limits", 1, -0.3, 0.3), (7, "motor", -3.0, 50.0), (10, "spring", 4.0, 0.1), (9, "friction", 0.0),
               (14, "swing", 0.2, 0.2), (11, "break", 0.01, float("inf"))]
    applied = 0
    for k, what, *values in changes:
        if not ends_awake(k):
            continue
        b.joint_set(0, abi.tf_id(k, 0), what, *values)
        r.joint_set(abi.tf_id(k, 0), what, *values)
        applied += 1
    assert applied >= 4
    # The last chain link lets go, and its slot comes back as a new joint holding that body where it is.
    assert ends_awake(5)
    last = r.joint_info(abi.tf_id(5, 0)).body_b
    b.joint_set(0, abi.tf_id(5, 0), "destroy")
    r.joint_set(abi.tf_id(5, 0), "destroy")
    pos = tuple(float(x) for x in r.states()["p"][last])
    desc = abi.joint_desc(abi.TF_JOINT_POINT, abi.tf_id(last, 0), anchor=pos)
    mine, theirs = b.joint_create(0, desc), r.joint_create(desc)
    assert (mine.index, mine.generation) == (theirs.index, theirs.generation) == (5, 1)
    n = len(w.joints)
    for s in range(60):
        b.step_checked(sc.dt)
        r.step(sc.dt)
        assert b.broken_joints(0) == r.broken_joints(), f"step {s + 21}"
        if s % 10 == 9:
            errs = state_errors(b.world_states(0), r.states())
            assert max(errs.values()) <= TOL, f"step {s + 21}: state error {errs}"
            for k in range(n):
                jid = abi.tf_id(k, 1 if k == 5 else 0)
                m, t = b.joint_info(0, jid), r.joint_info(jid)
                assert (m.type, m.body_a, m.body_b, m.broken) == (t.type, t.body_a, t.body_b, t.broken), f"joint {k}"
                mr, tr = _joint_rows([m]), _joint_rows([t])
                assert rel_err(mr, tr) <= TOL, f"step {s + 21}: joint {k} differs by {rel_err(mr, tr)}"
