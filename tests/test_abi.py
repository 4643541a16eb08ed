"""The C ABI library loads, exports every entry point include/twofold_b200.h declares, and behaves as the
reference's API does for invalid input, all without a GPU (CUDA is first touched by a step)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from twofold_b200 import abi, scenes
from twofold_b200.world import Batch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "twofold_b200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"TF_API\s+[\w\s\*]+?\b(tf_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = abi.load()
    names = declared()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(abi.EXPORTED) == names


def test_abi_version_and_defaults():
    lib = abi.load()
    assert lib.tf_abi_version() == 1
    s = abi.tf_settings()
    lib.tf_default_settings(C.byref(s))
    ref = abi.default_settings()
    for name, _ in abi.tf_settings._fields_:
        a, b = getattr(s, name), getattr(ref, name)
        if hasattr(a, "__len__"):
            assert list(a) == list(b), name
        else:
            assert a == b, name


def test_invalid_handles_read_as_zero_and_bad_calls_fail_cleanly():
    lib = abi.load()
    b = Batch([scenes.single("box_on_ground")])
    m, c, i = b.mass(0, 99)  # no such body: zeros, no error (src/world.cpp:352-371)
    assert m == 0 and not c.any() and not i.any()
    out = C.c_void_p()
    assert lib.tf_world_create(None, 0, 0, C.byref(out)) == abi.TF_OK - 1  # TF_E_INVALID
    assert b"bad arguments" in lib.tf_last_error()


def test_step_ignores_a_time_that_is_not_finite():
    """tests/test_world.cpp:553-565: dt <= 0 or non-finite does nothing (and touches no device)."""
    b = Batch([scenes.single("box_on_ground")])
    before = b.states()
    for dt in (float("nan"), float("inf"), -float("inf"), 0.0, -1.0):
        assert b.step(dt) == abi.TF_OK
    after = b.states()
    for k in before:
        assert np.array_equal(before[k], after[k])


def test_unsupported_shapes_are_refused():
    """Sensors and meshes on dynamic bodies are not run by this build; an unknown geometry is invalid."""
    lib = abi.load()
    h = C.c_void_p()
    abi.check(lib.tf_world_create(None, 1, 0, C.byref(h)))
    bid = abi.tf_id()
    abi.check(lib.tf_body_create(h, 0, C.byref(abi.body_desc()), C.byref(bid)))
    sid = abi.tf_id()
    assert lib.tf_shape_add(h, 0, bid, C.byref(abi.shape_desc(sensor=True)), C.byref(sid)) == abi.TF_E_UNSUPPORTED
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 0, 1]], np.float32)
    i = np.array([0, 2, 1], np.uint32)
    mesh = C.c_int32(-1)
    abi.check(lib.tf_mesh_create(h, v.ctypes.data, 3, i.ctypes.data, 3, C.byref(mesh)))
    assert lib.tf_shape_add(h, 0, bid, C.byref(abi.shape_desc(geometry=abi.TF_MESH, mesh=mesh.value)),
                            C.byref(sid)) == abi.TF_E_UNSUPPORTED
    assert lib.tf_shape_add(h, 0, bid, C.byref(abi.shape_desc(geometry=99)), C.byref(sid)) == abi.TF_E_INVALID
    abi.check(lib.tf_shape_add(h, 0, bid, C.byref(abi.shape_desc(geometry=abi.TF_CYLINDER)), C.byref(sid)))
    lib.tf_world_destroy(h)


def test_bodies_locked_to_two_planes_in_one_world_are_refused():
    """Bodies locked to a plane run when every one of a world is locked to the same plane."""
    lib = abi.load()
    h = C.c_void_p()
    abi.check(lib.tf_world_create(None, 2, 0, C.byref(h)))
    bid = abi.tf_id()
    planar = abi.body_desc(locks=abi.TF_LOCK_PLANAR)
    abi.check(lib.tf_body_create(h, 0, C.byref(planar), C.byref(bid)))
    abi.check(lib.tf_body_create(h, 0, C.byref(planar), C.byref(bid)))
    turned = abi.body_desc(locks=abi.TF_LOCK_PLANAR, lock_frame=(0.0, 0.70710677, 0.0, 0.70710677))
    assert lib.tf_body_create(h, 0, C.byref(turned), C.byref(bid)) == abi.TF_E_UNSUPPORTED
    abi.check(lib.tf_body_create(h, 1, C.byref(turned), C.byref(bid)))
    lib.tf_world_destroy(h)
