"""Test infrastructure only: Python access to the oracle (the unmodified AnvilFx/twofold World, built by
oracle/Makefile into oracle/_ref/libtwofold_ref.so). Only tests/, the smoke check and bench.py's
CPU-baseline leg use this module, and only as the checker or the timed CPU baseline.
"""
import ctypes as C
import os

import numpy as np

from twofold_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libtwofold_ref.so")
# The same reference with sinf, cosf, atan2f and asinf correctly rounded (oracle/rounded_libm.cpp).
ROUNDED_LIB = os.path.join(HERE, "_ref", "libtwofold_ref_rounded.so")

_libs = {}


def available(path=REF_LIB):
    return os.path.exists(path)


def load(path=REF_LIB):
    if path not in _libs:
        if not available(path):
            raise RuntimeError(f"{path} is missing; build it with `make -C oracle`")
        lib = C.CDLL(path)
        P = C.c_void_p
        sig = {
            "ref_world_create": ([C.POINTER(abi.tf_settings)], P),
            "ref_world_copy": ([P], P),
            "ref_world_destroy": ([P], None),
            "ref_body_create": ([P, C.POINTER(abi.tf_body_desc), C.POINTER(abi.tf_id)], C.c_int),
            "ref_shape_add": ([P, abi.tf_id, C.POINTER(abi.tf_shape_desc), C.POINTER(abi.tf_id)], C.c_int),
            "ref_scene_build": ([P, C.c_int, P, C.c_int, P, P], C.c_int),
            "ref_mesh_create": ([P, C.c_int, P, C.c_int], C.c_int),
            "ref_mesh_read": ([C.c_int, P, P, P, P, P, P, P], C.c_int),
            "ref_hull_compute": ([P, C.c_int32, C.c_int32, P, P, C.c_int32, P, C.c_int32], C.c_int),
            "ref_world_step": ([P, C.c_float, C.c_int], C.c_int),
            "ref_body_count": ([P], C.c_int),
            "ref_world_get_states": ([P, P, P, P, P, P], C.c_int),
            "ref_body_set_velocity": ([P, abi.tf_id, P, P], C.c_int),
            "ref_body_get_mass": ([P, abi.tf_id, P, P, P], C.c_int),
            "ref_world_candidates": ([P, P, C.c_int, C.POINTER(C.c_int)], C.c_int),
            "ref_world_contacts": ([P, C.c_int, C.POINTER(abi.tf_contact), C.c_int, C.POINTER(C.c_int)], C.c_int),
            "ref_world_profile": ([P, C.POINTER(abi.tf_profile)], C.c_int),
            "ref_joint_create": ([P, C.POINTER(abi.tf_joint_desc), C.POINTER(abi.tf_id)], C.c_int),
            "ref_joint_info": ([P, abi.tf_id, C.POINTER(abi.tf_joint_info)], C.c_int),
            "ref_joint_set": ([P, abi.tf_id, C.c_int, P], C.c_int),
            "ref_world_call": ([P, C.c_int, abi.tf_id, P, C.c_uint32, C.c_uint32], C.c_int),
            "ref_broken_joints": ([P, P, C.c_int, C.POINTER(C.c_int)], C.c_int),
            "ref_world_contact_events": ([P, C.POINTER(abi.tf_contact_event), C.c_int, C.POINTER(C.c_int)], C.c_int),
            "ref_world_hit_events": ([P, C.POINTER(abi.tf_hit_event), C.c_int, C.POINTER(C.c_int)], C.c_int),
            "ref_awake_dynamic": ([P], C.c_int),
            "ref_worlds_step_parallel": ([P, C.c_int, C.c_float, C.c_int, C.c_int, C.POINTER(C.c_int64)], C.c_int),
            "ref_hardware_threads": ([], C.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = res
        _libs[path] = lib
    return _libs[path]


def mesh_create(vertices, indices, lib=REF_LIB):
    """A reference TriangleMesh (include/twofold/mesh.h:13-30); returns its id in the harness."""
    lib = load(lib)
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
    i = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    return lib.ref_mesh_create(v.ctypes.data, len(v), i.ctypes.data, len(i))


def mesh_read(mesh):
    """The reference's built mesh, in the layout of twofold_b200.world.Batch.read_mesh."""
    lib = load()
    counts = np.zeros(3, np.int32)
    lib.ref_mesh_read(mesh, counts.ctypes.data, None, None, None, None, None, None)
    nv, nt, nn = (int(x) for x in counts)
    out = {"vertices": np.zeros((nv, 3), np.float32), "indices": np.zeros(3 * nt, np.uint32),
           "normals": np.zeros((nt, 3), np.float32), "edges": np.zeros(nt, np.uint8),
           "node_bounds": np.zeros((nn, 6), np.float32), "node_ranges": np.zeros((nn, 2), np.int32)}
    lib.ref_mesh_read(mesh, counts.ctypes.data, *(out[k].ctypes.data for k in
                      ("vertices", "indices", "normals", "edges", "node_bounds", "node_ranges")))
    return out


def hull_compute(points, max_vertices):
    """The reference's computeHull, in the layout of twofold_b200.abi.hull_compute."""
    return abi._hull_call(load().ref_hull_compute, points, max_vertices, lambda rc: None)


class RefWorld:
    """One reference World built from a scenes.World."""

    def __init__(self, world, settings=None, _handle=None, lib=REF_LIB):
        self.lib = load(lib)
        if _handle is not None:
            self.h = _handle
            return
        s = settings if settings is not None else abi.default_settings()
        self.h = self.lib.ref_world_create(C.byref(s))
        shapes = world.shapes
        if getattr(world, "meshes", None):
            ids = [mesh_create(v, i, lib) for v, i in world.meshes]
            shapes = world.shapes.copy()
            named = shapes["geometry"] == abi.TF_MESH
            shapes["mesh"][named] = np.asarray(ids, np.int32)[shapes["mesh"][named]]
        rc = self.lib.ref_scene_build(self.h, len(world.bodies), world.bodies.ctypes.data, len(shapes),
                                      world.body_of.ctypes.data, shapes.ctypes.data)
        if rc != 0:
            raise RuntimeError("reference scene build failed")
        for j in getattr(world, "joints", []):
            self.joint_create(j)

    def copy(self):
        r = RefWorld(None, _handle=self.lib.ref_world_copy(self.h))
        r.lib = self.lib
        return r

    def __del__(self):
        if getattr(self, "h", None) and getattr(self, "lib", None) is not None:
            self.lib.ref_world_destroy(self.h)
            self.h = None

    def step(self, dt, n=1):
        self.lib.ref_world_step(self.h, C.c_float(dt), n)

    def states(self):
        n = self.lib.ref_body_count(self.h)
        p = np.zeros((n, 3), np.float32)
        q = np.zeros((n, 4), np.float32)
        v = np.zeros((n, 3), np.float32)
        w = np.zeros((n, 3), np.float32)
        awake = np.zeros(n, np.int32)
        self.lib.ref_world_get_states(self.h, p.ctypes.data, q.ctypes.data, v.ctypes.data, w.ctypes.data,
                                      awake.ctypes.data)
        return {"p": p, "q": q, "v": v, "w": w, "awake": awake}

    def candidates(self):
        n = C.c_int(0)
        self.lib.ref_world_candidates(self.h, None, 0, C.byref(n))
        out = np.zeros(max(n.value, 1), np.uint64)
        self.lib.ref_world_candidates(self.h, out.ctypes.data, n.value, C.byref(n))
        return out[:n.value]

    def contacts(self, mode=1):
        n = C.c_int(0)
        self.lib.ref_world_contacts(self.h, mode, None, 0, C.byref(n))
        arr = (abi.tf_contact * max(n.value, 1))()
        self.lib.ref_world_contacts(self.h, mode, arr, n.value, C.byref(n))
        return list(arr)[:n.value]

    def joint_create(self, desc):
        out = abi.tf_id()
        if self.lib.ref_joint_create(self.h, C.byref(desc), C.byref(out)) != 0:
            raise ValueError("the reference refused the joint")
        return out

    def joint_set(self, joint, what, *values):
        """what: limits (limited, lower, upper), motor, spring, friction, swing, break, destroy."""
        kinds = ("limits", "motor", "spring", "friction", "swing", "break", "destroy")
        v = (C.c_float * 3)(*(list(values) + [0.0] * (3 - len(values))))
        self.lib.ref_joint_set(self.h, joint, kinds.index(what), v)

    def call(self, what, target, values=(), a=0, b=0):
        """A World call between steps (twofold_b200.world.CALLS names them) on a body or shape id."""
        from twofold_b200.world import CALLS

        v = (C.c_float * 8)(*(list(values) + [0.0] * (8 - len(values))))
        if self.lib.ref_world_call(self.h, CALLS.index(what), target, v, a, b) != 0:
            raise ValueError(f"unknown call {what}")

    def joint_info(self, joint):
        info = abi.tf_joint_info()
        self.lib.ref_joint_info(self.h, joint, C.byref(info))
        return info

    def broken_joints(self):
        n = C.c_int(0)
        self.lib.ref_broken_joints(self.h, None, 0, C.byref(n))
        arr = (abi.tf_id * max(n.value, 1))()
        self.lib.ref_broken_joints(self.h, arr, n.value, C.byref(n))
        return [(x.index, x.generation) for x in list(arr)[:n.value]]

    def contact_events(self):
        n = C.c_int(0)
        self.lib.ref_world_contact_events(self.h, None, 0, C.byref(n))
        arr = (abi.tf_contact_event * max(n.value, 1))()
        self.lib.ref_world_contact_events(self.h, arr, n.value, C.byref(n))
        return [(e.shape_a, e.shape_b, e.body_a, e.body_b, bool(e.begin)) for e in list(arr)[:n.value]]

    def hit_events(self):
        n = C.c_int(0)
        self.lib.ref_world_hit_events(self.h, None, 0, C.byref(n))
        arr = (abi.tf_hit_event * max(n.value, 1))()
        self.lib.ref_world_hit_events(self.h, arr, n.value, C.byref(n))
        return [(e.shape_a, e.shape_b, e.body_a, e.body_b, np.array(e.point[:], np.float32),
                 np.array(e.normal[:], np.float32), np.float32(e.speed)) for e in list(arr)[:n.value]]

    def profile(self):
        p = abi.tf_profile()
        self.lib.ref_world_profile(self.h, C.byref(p))
        return p

    def mass(self, index, generation=0):
        m = C.c_float(0)
        c = np.zeros(3, np.float32)
        i = np.zeros(9, np.float32)
        self.lib.ref_body_get_mass(self.h, abi.tf_id(index, generation), C.byref(m), c.ctypes.data, i.ctypes.data)
        return m.value, c, i.reshape(3, 3)

    def awake_dynamic(self):
        return self.lib.ref_awake_dynamic(self.h)


def step_parallel(ref_worlds, dt, steps, threads):
    """Steps independent reference worlds, each by one thread from a pool of `threads`. Returns the
    awake-dynamic body-steps summed over every step of every world. The worlds come from one build of the
    oracle, whose stepping code runs them."""
    if not ref_worlds:
        return 0
    lib = ref_worlds[0].lib
    arr = (C.c_void_p * len(ref_worlds))(*[r.h for r in ref_worlds])
    total = C.c_int64(0)
    lib.ref_worlds_step_parallel(arr, len(ref_worlds), C.c_float(dt), steps, threads, C.byref(total))
    return total.value


def hardware_threads():
    return load().ref_hardware_threads()
