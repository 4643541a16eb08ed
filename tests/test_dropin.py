"""The drop-in C++ surface: the programs under tests/dropin/, written against the reference's public World API,
build unchanged against include/twofold_b200/world.hpp, and run on the GPU they print what the reference printed
(tests/golden/dropin_*.txt, made by tests/golden/make_dropin_golden.py) within 1e-5.
"""
import os
import subprocess

import numpy as np
import pytest

from parity import rel_err
from twofold_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PROGRAM = os.path.join(HERE, "dropin", "pyramid_step.cpp")
GOLDEN = os.path.join(HERE, "golden", "dropin_pyramid.txt")
JOINTS_PROGRAM = os.path.join(HERE, "dropin", "joints_step.cpp")
JOINTS_GOLDEN = os.path.join(HERE, "golden", "dropin_joints.txt")
SETTERS_PROGRAM = os.path.join(HERE, "dropin", "setters_step.cpp")
SETTERS_GOLDEN = os.path.join(HERE, "golden", "dropin_setters.txt")
TOL = 1e-5


def _compile(out, link, program=PROGRAM):
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", f"-I{os.path.join(ROOT, 'include')}",
           '-DTWOFOLD_HEADER="twofold_b200/world.hpp"', program]
    if link:
        libdir = os.path.dirname(abi.LIB_PATH)
        cmd += ["-o", out, f"-L{libdir}", "-l:" + os.path.basename(abi.LIB_PATH), f"-Wl,-rpath,{libdir}"]
    else:
        cmd += ["-fsyntax-only"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def _parse(text):
    lines = [l for l in text.splitlines() if l and not l.startswith("#")]
    manifolds = int(lines[0].split()[1])
    events = [float(x) for x in lines[1].split()[1:]]
    rows = np.array([[float(x) for x in l.split()] for l in lines[2:]])
    return (manifolds, events), rows


def test_dropin_program_compiles_against_the_facade():
    _compile(None, link=False)
    _compile(None, link=False, program=JOINTS_PROGRAM)
    _compile(None, link=False, program=SETTERS_PROGRAM)


def _parse_joints(text):
    lines = [l for l in text.splitlines() if l and not l.startswith("#")]
    broken = int(lines[0].split()[1])
    live = [int(l.split()[1]) for l in lines if l.startswith("live")]
    bodies = np.array([[float(x) for x in l.split()] for l in lines[1:] if not l.startswith(("joint", "live"))])
    joints = np.array([[float(x) for x in l.split()[1:]] for l in lines[1:] if l.startswith("joint")])
    return (broken, live), bodies, joints


@pytest.mark.gpu
def test_dropin_joints_program_matches_the_reference(tmp_path):
    """Every joint kind through the drop-in World::createJoint, jointInfo and brokenJoints."""
    exe = str(tmp_path / "joints_b200")
    _compile(exe, link=True, program=JOINTS_PROGRAM)
    out = subprocess.run([exe, "60"], check=True, capture_output=True, text=True).stdout
    b_mine, bodies_mine, joints_mine = _parse_joints(out)
    with open(JOINTS_GOLDEN) as f:
        b_ref, bodies_ref, joints_ref = _parse_joints(f.read())
    assert b_mine == b_ref
    assert np.array_equal(bodies_mine[:, 0], bodies_ref[:, 0])
    for name, cols in (("p", slice(1, 4)), ("q", slice(4, 8)), ("v", slice(8, 11)), ("w", slice(11, 14))):
        err = rel_err(bodies_mine[:, cols], bodies_ref[:, cols])
        assert err <= TOL, f"{name} differs by {err}"
    # index, type and broken flag exactly; value and force within the tolerance
    assert np.array_equal(joints_mine[:, [0, 1, 6]], joints_ref[:, [0, 1, 6]])
    for name, cols in (("value", slice(2, 3)), ("force", slice(3, 6))):
        err = rel_err(joints_mine[:, cols], joints_ref[:, cols])
        assert err <= TOL, f"joint {name} differs by {err}"


@pytest.mark.gpu
def test_dropin_program_matches_the_reference(tmp_path):
    exe = str(tmp_path / "pyramid_b200")
    _compile(exe, link=True)
    out = subprocess.run([exe, "6", "60"], check=True, capture_output=True, text=True).stdout
    m_mine, mine = _parse(out)
    with open(GOLDEN) as f:
        m_ref, ref = _parse(f.read())
    # manifolds; events summed over the run: began, ended, hits (counts exact), hit speeds, touching contacts
    assert m_mine[0] == m_ref[0]
    ev_mine, ev_ref = m_mine[1], m_ref[1]
    assert [ev_mine[i] for i in (0, 1, 2, 4)] == [ev_ref[i] for i in (0, 1, 2, 4)], (ev_mine, ev_ref)
    assert abs(ev_mine[3] - ev_ref[3]) <= TOL * max(1.0, abs(ev_ref[3]))
    assert np.array_equal(mine[:, 0], ref[:, 0])
    for name, cols in (("p", slice(1, 4)), ("q", slice(4, 8)), ("v", slice(8, 11)), ("w", slice(11, 14))):
        err = rel_err(mine[:, cols], ref[:, cols])
        assert err <= TOL, f"{name} differs by {err}"


def _parse_setters(text):
    """{step: rows of index, generation, awake, p, q, v, w} and the validity line."""
    snaps, valid, step = {}, None, None
    for line in text.splitlines():
        if not line or line.startswith("#"):
            continue
        if line.startswith("step"):
            step = int(line.split()[1])
            snaps[step] = []
        elif line.startswith("valid"):
            valid = [int(x) for x in line.split()[1:]]
        else:
            snaps[step].append([float(x) for x in line.split()])
    return {k: np.array(v) for k, v in snaps.items()}, valid


@pytest.mark.gpu
def test_dropin_setters_program_matches_the_reference(tmp_path):
    """destroyBody, removeShape, setTransform, setKinematicTarget, setMotionType, forces and impulses, friction,
    restitution, rolling resistance, filters, damping, gravity scale, sleep, wake and setCanSleep, each called
    mid-run through the drop-in World, print what the reference printed every 20 steps."""
    exe = str(tmp_path / "setters_b200")
    _compile(exe, link=True, program=SETTERS_PROGRAM)
    out = subprocess.run([exe, "160"], check=True, capture_output=True, text=True).stdout
    mine, valid_mine = _parse_setters(out)
    with open(SETTERS_GOLDEN) as f:
        ref, valid_ref = _parse_setters(f.read())
    assert valid_mine == valid_ref
    assert sorted(mine) == sorted(ref)
    for step in sorted(ref):
        m, r = mine[step], ref[step]
        assert m.shape == r.shape, step
        # index, generation and awake flag exactly
        assert np.array_equal(m[:, :3], r[:, :3]), step
        for name, cols in (("p", slice(3, 6)), ("q", slice(6, 10)), ("v", slice(10, 13)), ("w", slice(13, 16))):
            err = rel_err(m[:, cols], r[:, cols])
            assert err <= TOL, f"step {step}: {name} differs by {err}"
