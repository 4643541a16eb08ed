"""The World calls between steps (include/twofold/world.h:375-463) against the oracle: each call is made on both
sides at the same step of the same world, and the two then step on together. States, sleep, contacts and the
contact events (those the calls queue come first in the next step's list) are compared step by step.

Compared with the reference built with correctly rounded float functions, so that steps where the continuous
pass moves bodies stay comparable bit for bit (the library's continuous pass uses those values)."""
import numpy as np
import pytest

import reference as R
from parity import contact_table, first_difference, rel_err, state_errors
from twofold_b200 import abi, scenes
from twofold_b200.world import Batch

pytestmark = pytest.mark.gpu

TOL = 1e-5
needs_oracle = pytest.mark.skipif(not R.available(R.ROUNDED_LIB), reason="oracle library not built")

F32 = np.float32


def _world():
    """A floor, a kinematic paddle, two stacks of boxes and two spheres, with sleeping on."""
    n = 19
    b, s = scenes._bodies(n), scenes._shapes(n)
    b["type"][0] = abi.TF_STATIC
    b["position"][0] = (0.0, -0.5, 0.0)
    s["half_extents"][0] = (12.0, 0.5, 12.0)
    b["type"][1] = abi.TF_KINEMATIC
    b["position"][1] = (-6.0, 0.6, 0.0)
    s["half_extents"][1] = (0.4, 0.4, 1.5)
    k = 2
    for x in (-2.0, 2.0):
        for i in range(7):
            b["position"][k] = (x + 0.01 * i, 0.5 + 1.0 * i, 0.02 * (i % 3))
            s["half_extents"][k] = (0.5, 0.5, 0.5)
            k += 1
    for y in (3.0, 6.0):
        b["position"][k] = (0.0, y, 0.0)
        s["geometry"][k] = abi.TF_SPHERE
        s["radius"][k] = 0.4
        k += 1
    b["position"][k] = (5.0, 0.5, 3.0)
    s["half_extents"][k] = (0.5, 0.5, 0.5)
    s["friction"] = 0.6
    return scenes.World(b, s, np.arange(n))


def _id(i):
    return abi.tf_id(i, 0)


# (step, call, target index, values, a, b): a shape's index equals its body's here, one shape per body.
SCRIPT = [
    (45, "friction", 3, (0.1,), 0, 0),
    (45, "restitution", 4, (0.5,), 0, 0),
    (45, "rolling_resistance", 17, (0.05,), 0, 0),
    (45, "damping", 5, (0.3, 0.2), 0, 0),
    (45, "gravity_scale", 6, (0.5,), 0, 0),
    (50, "impulse", 8, (2.0, 0.0, 0.0), 1, 0),
    (50, "force_at", 9, (0.0, 40.0, 0.0, 2.1, 2.0, 0.3), 1, 0),
    (50, "torque", 10, (0.0, 5.0, 0.0), 0, 0),
    (50, "impulse_at", 11, (0.0, 0.0, 1.5, 2.0, 5.4, 0.0), 1, 0),
    (55, "force", 12, (0.0, 0.0, 30.0), 1, 0),
    (70, "transform", 13, (2.0, 9.0, 0.0, 0.0, 0.3826834, 0.0, 0.9238795), 0, 0),
    (80, "destroy_body", 4, (), 0, 0),
    (82, "remove_shape", 14, (), 0, 0),
    (90, "filter", 15, (), 2, 2),
    (100, "motion_type", 7, (), abi.TF_STATIC, 0),
    (100, "motion_type", 16, (), abi.TF_KINEMATIC, 0),
    (104, "motion_type", 16, (), abi.TF_DYNAMIC, 0),
    (110, "sleep", 5, (), 0, 0),
    (110, "can_sleep", 18, (), 0, 0),
    (112, "wake", 18, (), 0, 0),
    (120, "velocity", 2, (0.0, 3.0, 0.0), 0, 0),
    (120, "spin", 3, (0.0, 2.0, 0.0), 0, 0),
    (126, "transform", 0, (0.0, -0.45, 0.0, 0.0, 0.0, 0.0, 1.0), 0, 0),
]


def _compare(b, r, label):
    errs = state_errors(b.world_states(0), r.states())
    assert max(errs.values()) <= TOL, f"{label}: state error {errs}"
    assert np.array_equal(b.world_states(0)["awake"], r.states()["awake"]), f"{label}: sleep differs"
    em, pm = contact_table(b.contacts(0, mode=1))
    er, pr = contact_table(r.contacts(mode=1))
    assert em == er, f"{label}: contacts differ at {first_difference(em, er)}"
    assert rel_err(pm, pr) <= TOL, f"{label}: contact points differ by {rel_err(pm, pr)}"
    ev_m, ev_r = b.contact_events(0), r.contact_events()
    assert ev_m == ev_r, f"{label}: contact events differ: {ev_m} vs {ev_r}"


@needs_oracle
@pytest.mark.parametrize("graph", [False, True])
def test_calls_between_steps_match_reference(graph):
    w = _world()
    sc = scenes.Scene("calls", [w])
    b = Batch.from_scene(sc)
    r = R.RefWorld(w, sc.settings, lib=R.ROUNDED_LIB)
    slept = False
    for step in range(140):
        for (at, what, target, values, a, bb) in SCRIPT:
            if at == step:
                b.call(0, what, _id(target), values, a, bb)
                r.call(what, _id(target), values, a, bb)
        if 60 <= step < 80:
            # The paddle carried into the left stack, one target a step.
            x = F32(-6.0 + 0.25 * (step - 59))
            target = (x, 0.6, 0.0, 0.0, 0.0, 0.0, 1.0, sc.dt)
            b.call(0, "kinematic_target", _id(1), target)
            r.call("kinematic_target", _id(1), target)
        if step == 130:
            # A joint between two bodies that touch: their contacts go and the touching pair ends.
            d = abi.joint_desc(abi.TF_JOINT_POINT, _id(6), body_a=_id(5), anchor=(-2.0, 4.0, 0.0))
            b.joint_create(0, d)
            r.joint_create(d)
        b.step_checked(sc.dt, 1, graph=graph)
        r.step(sc.dt)
        slept = slept or not all(r.states()["awake"][2:])
        _compare(b, r, f"step {step + 1}")
    assert slept  # the script also ran on sleeping bodies


def test_default_mixes_only():
    lib = abi.load()
    b = Batch.from_scene(scenes.Scene("one", [scenes.single("box_on_ground")]))
    abi.check(lib.tf_world_set_mix(b.h, 0, 0), lib)
    assert lib.tf_world_set_mix(b.h, 0, 1) == abi.TF_E_UNSUPPORTED
    assert lib.tf_world_set_mix(b.h, 1, 2) == abi.TF_E_UNSUPPORTED
