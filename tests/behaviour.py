"""Known-answer scenarios restated from the reference's own test suite (tests/test_world.cpp), as descriptor
arrays both the oracle and the B200 library can step. Each scenario returns (world, steps, check) where
check(states_after, contacts_after) raises on a wrong answer.
"""
import numpy as np

from twofold_b200 import abi, scenes

DT = float(np.float32(1.0 / 60.0))


def _world(n):
    b, s = scenes._bodies(n), scenes._shapes(n)
    scenes._ground(b, s)
    s["friction"][1:] = 0.6
    return b, s


def box_rests_on_half_space():
    """tests/test_world.cpp:109-116: a box dropped from 2 m rests at 0.5 m, upright."""
    b, s = _world(2)
    b["position"][1] = (0, 2, 0)

    def check(st, _):
        assert abs(st["p"][1, 1] - 0.5) <= 0.02, st["p"][1]
        q = st["q"][1]
        # |rotate(q, y).y| > 0.999
        x, y, z, w = q
        up_y = 1 - 2 * (x * x + z * z)
        assert abs(up_y) > 0.999

    return scenes.World(b, s, np.arange(2)), 180, check


def box_stack_stays_upright():
    """tests/test_world.cpp:235-244: ten stacked unit boxes, the top stays at 9.5 m within 0.1 after 6 s."""
    b, s = _world(11)
    for i in range(10):
        b["position"][i + 1] = (0, 0.5 + i, 0)

    def check(st, _):
        top = st["p"][10]
        assert abs(top[1] - 9.5) <= 0.1 and abs(top[0]) <= 0.05 and abs(top[2]) <= 0.05, top

    return scenes.World(b, s, np.arange(11)), 360, check


def bounce_with_full_restitution():
    """tests/test_world.cpp:246-267: a sphere with restitution 1 on a restitution-1 floor bounces back above
    2.6 m. The check here is on the peak after the first landing, tracked by the caller."""
    b, s = _world(2)
    s["restitution"][0] = 1.0
    b["position"][1] = (0, 3, 0)
    s["geometry"][1] = abi.TF_SPHERE
    s["radius"][1] = 0.5
    s["restitution"][1] = 1.0
    s["friction"][1] = 0.5
    return scenes.World(b, s, np.arange(2)), 240, None


def contacts_are_reported():
    """tests/test_world.cpp:598-607: a resting box reports one contact of four points."""
    b, s = _world(2)
    b["position"][1] = (0, 0.5, 0)

    def check(_, contacts):
        touching = [c for c in contacts if any(c.separations[i] < 0 or c.normal_impulses[i] > 0
                                                for i in range(c.point_count))]
        assert len(touching) == 1 and touching[0].point_count == 4

    return scenes.World(b, s, np.arange(2)), 30, check


def body_falls_asleep():
    """tests/test_world.cpp:317-323: a box resting on the ground is asleep after 4 s."""
    b, s = _world(2)
    b["position"][1] = (0, 1, 0)

    def check(st, _):
        assert st["awake"][1] == 0

    return scenes.World(b, s, np.arange(2)), 240, check


def mixed_column():
    """tests/test_world.cpp:523-551: twenty alternating boxes and spheres dropped in a column, used for
    the run-twice determinism check."""
    b, s = _world(21)
    for i in range(20):
        b["position"][i + 1] = (0.3 * (i % 4), 1.0 + 1.1 * i, 0.2 * (i % 3))
        half = 0.05 * i  # axisAngle({1, 1, 0}, 0.1 i)
        ax = np.array([1.0, 1.0, 0.0]) / np.sqrt(2.0)
        b["rotation"][i + 1] = np.concatenate([ax * np.sin(half), [np.cos(half)]]).astype(np.float32)
        if i % 2:
            s["geometry"][i + 1] = abi.TF_SPHERE
            s["radius"][i + 1] = 0.4
        else:
            s["half_extents"][i + 1] = (0.4, 0.3, 0.5)
        s["friction"][i + 1] = 0.5
    return scenes.World(b, s, np.arange(21)), 180, None


SCENARIOS = {
    "box_rests_on_half_space": box_rests_on_half_space,
    "box_stack_stays_upright": box_stack_stays_upright,
    "contacts_are_reported": contacts_are_reported,
    "body_falls_asleep": body_falls_asleep,
}
