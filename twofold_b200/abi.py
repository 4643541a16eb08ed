"""ctypes mirror of include/twofold_b200.h and the loader for the CUDA library.

The library is the product: `load()` raises when libtwofold_b200.so is missing instead of falling back
to anything else.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# TWOFOLD_B200_LIB selects another build of the same library (for instance the index-checking one).
LIB_PATH = os.environ.get("TWOFOLD_B200_LIB") or os.path.join(HERE, "libtwofold_b200.so")

TF_OK = 0
TF_E_INVALID, TF_E_CUDA, TF_E_CAPACITY, TF_E_NUMERIC, TF_E_TIMEOUT, TF_E_UNSUPPORTED = -1, -2, -3, -4, -5, -6
TF_PAIR_LIVE, TF_PAIR_DYNAMIC, TF_PAIR_MOVING = 1, 2, 4
TF_NOALLOC_MAX_BODIES, TF_NOALLOC_MAX_PAIRS = 4096, 32768
TF_STATIC, TF_KINEMATIC, TF_DYNAMIC = 0, 1, 2
TF_SPHERE, TF_BOX, TF_CYLINDER, TF_PRISM, TF_HULL, TF_HALFSPACE, TF_MESH = range(7)
TF_LOCK_PLANAR = (1 << 2) | (1 << 3) | (1 << 4)


class tf_id(C.Structure):
    _fields_ = [("index", C.c_uint32), ("generation", C.c_uint32)]


class tf_settings(C.Structure):
    _fields_ = [
        ("gravity", C.c_float * 3),
        ("length_unit", C.c_float),
        ("substeps", C.c_int32),
        ("contact_hertz", C.c_float),
        ("contact_damping_ratio", C.c_float),
        ("max_pushout_speed", C.c_float),
        ("max_linear_speed", C.c_float),
        ("max_angular_speed", C.c_float),
        ("restitution_threshold", C.c_float),
        ("hit_threshold", C.c_float),
        ("sleep_threshold", C.c_float),
        ("time_to_sleep", C.c_float),
        ("contact_reuse_distance", C.c_float),
        ("contact_reuse_angle", C.c_float),
        ("joint_hertz", C.c_float),
        ("joint_damping_ratio", C.c_float),
        ("continuous", C.c_int32),
    ]


def default_settings(**over):
    """WorldSettings defaults (include/twofold/world.h:216-241)."""
    s = tf_settings()
    s.gravity[:] = [0.0, -9.81, 0.0]
    s.length_unit = 1.0
    s.substeps = 4
    s.contact_hertz = 30.0
    s.contact_damping_ratio = 10.0
    s.max_pushout_speed = 3.0
    s.max_linear_speed = 1000.0
    s.max_angular_speed = 1000.0
    s.restitution_threshold = 1.0
    s.hit_threshold = 1.0
    s.sleep_threshold = 0.05
    s.time_to_sleep = 0.5
    s.contact_reuse_distance = 0.0005
    s.contact_reuse_angle = 0.035
    s.joint_hertz = 60.0
    s.joint_damping_ratio = 2.0
    s.continuous = 1
    for k, v in over.items():
        if k == "gravity":
            s.gravity[:] = list(v)
        else:
            setattr(s, k, v)
    return s


class tf_body_desc(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("position", C.c_float * 3),
        ("rotation", C.c_float * 4),
        ("linear_velocity", C.c_float * 3),
        ("angular_velocity", C.c_float * 3),
        ("linear_damping", C.c_float),
        ("angular_damping", C.c_float),
        ("gravity_scale", C.c_float),
        ("locks", C.c_uint32),
        ("lock_frame", C.c_float * 4),
        ("awake", C.c_int32),
        ("can_sleep", C.c_int32),
    ]


class tf_shape_desc(C.Structure):
    _fields_ = [
        ("geometry", C.c_int32),
        ("radius", C.c_float),
        ("half_extents", C.c_float * 3),
        ("half_height", C.c_float),
        ("points", C.POINTER(C.c_float)),
        ("point_count", C.c_int32),
        ("max_vertices", C.c_int32),
        ("z_min", C.c_float),
        ("z_max", C.c_float),
        ("position", C.c_float * 3),
        ("rotation", C.c_float * 4),
        ("density", C.c_float),
        ("friction", C.c_float),
        ("restitution", C.c_float),
        ("rolling_resistance", C.c_float),
        ("category", C.c_uint32),
        ("mask", C.c_uint32),
        ("sensor", C.c_int32),
        ("mesh", C.c_int32),
    ]


class tf_profile(C.Structure):
    _fields_ = [
        ("total", C.c_float),
        ("broadphase", C.c_float),
        ("narrowphase", C.c_float),
        ("solver", C.c_float),
        ("continuous", C.c_float),
        ("sleep", C.c_float),
        ("candidate_pairs", C.c_int32),
        ("swept_pairs", C.c_int32),
        ("impacts", C.c_int32),
        ("manifolds", C.c_int32),
        ("touching_contacts", C.c_int32),
        ("awake_bodies", C.c_int32),
        ("awake_islands", C.c_int32),
    ]


class tf_contact(C.Structure):
    _fields_ = [
        ("key", C.c_uint64),
        ("part", C.c_uint32),
        ("shape_a", C.c_uint32),
        ("shape_b", C.c_uint32),
        ("body_a", C.c_uint32),
        ("body_b", C.c_uint32),
        ("point_count", C.c_int32),
        ("feature_kind", C.c_int32),
        ("feature_a", C.c_int32),
        ("feature_b", C.c_int32),
        ("normal", C.c_float * 3),
        ("friction", C.c_float),
        ("restitution", C.c_float),
        ("rolling_resistance", C.c_float),
        ("rolling_impulse", C.c_float * 3),
        ("points", (C.c_float * 3) * 4),
        ("separations", C.c_float * 4),
        ("normal_impulses", C.c_float * 4),
        ("tangent_impulses", (C.c_float * 3) * 4),
    ]


TF_JOINT_POINT, TF_JOINT_FIXED, TF_JOINT_HINGE, TF_JOINT_SLIDER, TF_JOINT_DISTANCE, TF_JOINT_SWING_TWIST = range(6)


class tf_joint_desc(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("body_a", tf_id),
        ("body_b", tf_id),
        ("anchor", C.c_float * 3),
        ("anchor_b", C.c_float * 3),
        ("axis", C.c_float * 3),
        ("normal", C.c_float * 3),
        ("limited", C.c_int32),
        ("lower", C.c_float),
        ("upper", C.c_float),
        ("motor_speed", C.c_float),
        ("max_motor", C.c_float),
        ("friction", C.c_float),
        ("length", C.c_float),
        ("hertz", C.c_float),
        ("damping_ratio", C.c_float),
        ("swing_y", C.c_float),
        ("swing_z", C.c_float),
        ("collide_connected", C.c_int32),
        ("break_force", C.c_float),
        ("break_torque", C.c_float),
    ]


def joint_desc(type, body_b, body_a=None, **kw):
    """A tf_joint_desc with the reference's JointDesc defaults: no limits, no motor, unbreakable, a hinge or
    swing-twist axis along x (hinge: z), swing and twist free."""
    d = tf_joint_desc()
    d.type = type
    d.body_a = body_a if body_a is not None else tf_id(0xFFFFFFFF, 0)
    d.body_b = body_b
    d.axis[:] = [0.0, 0.0, 1.0] if type == TF_JOINT_HINGE else [1.0, 0.0, 0.0]
    d.normal[:] = [0.0, 1.0, 0.0]
    d.length = -1.0
    d.swing_y = d.swing_z = 3.14159265
    if type == TF_JOINT_SWING_TWIST:
        d.lower, d.upper = -3.14159265, 3.14159265
    d.break_force = d.break_torque = float("inf")
    for k, v in kw.items():
        if isinstance(v, (list, tuple)):
            getattr(d, k)[:] = list(v)
        else:
            setattr(d, k, v)
    return d


class tf_joint_info(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("body_a", C.c_uint32),
        ("body_b", C.c_uint32),
        ("anchor_a", C.c_float * 3),
        ("anchor_b", C.c_float * 3),
        ("axis", C.c_float * 3),
        ("value", C.c_float),
        ("force", C.c_float * 3),
        ("torque", C.c_float * 3),
        ("broken", C.c_int32),
    ]


class tf_contact_event(C.Structure):
    _fields_ = [
        ("shape_a", C.c_uint32),
        ("shape_b", C.c_uint32),
        ("body_a", C.c_uint32),
        ("body_b", C.c_uint32),
        ("begin", C.c_int32),
    ]


class tf_hit_event(C.Structure):
    _fields_ = [
        ("shape_a", C.c_uint32),
        ("shape_b", C.c_uint32),
        ("body_a", C.c_uint32),
        ("body_b", C.c_uint32),
        ("point", C.c_float * 3),
        ("normal", C.c_float * 3),
        ("speed", C.c_float),
    ]


def body_desc(type=TF_DYNAMIC, position=(0, 0, 0), rotation=(0, 0, 0, 1), linear_velocity=(0, 0, 0),
              angular_velocity=(0, 0, 0), linear_damping=0.0, angular_damping=0.0, gravity_scale=1.0, locks=0,
              lock_frame=(0, 0, 0, 1), awake=True, can_sleep=True):
    """BodyDesc defaults (include/twofold/world.h:108-123)."""
    d = tf_body_desc()
    d.type = type
    d.position[:] = list(position)
    d.rotation[:] = list(rotation)
    d.linear_velocity[:] = list(linear_velocity)
    d.angular_velocity[:] = list(angular_velocity)
    d.linear_damping = linear_damping
    d.angular_damping = angular_damping
    d.gravity_scale = gravity_scale
    d.locks = locks
    d.lock_frame[:] = list(lock_frame)
    d.awake = 1 if awake else 0
    d.can_sleep = 1 if can_sleep else 0
    return d


def shape_desc(geometry=TF_BOX, radius=0.5, half_extents=(0.5, 0.5, 0.5), half_height=0.5, points=None,
               max_vertices=64, z_min=-0.5, z_max=0.5, position=(0, 0, 0), rotation=(0, 0, 0, 1), density=1.0,
               friction=0.5, restitution=0.0, rolling_resistance=0.0, category=1, mask=0xFFFFFFFF, sensor=False,
               mesh=-1):
    """ShapeDesc defaults (include/twofold/world.h:90-106). `points` must stay alive until the shape is added."""
    d = tf_shape_desc()
    d.geometry = geometry
    d.radius = radius
    d.half_extents[:] = list(half_extents)
    d.half_height = half_height
    if points is not None:
        d.points = points.ctypes.data_as(C.POINTER(C.c_float))
        d.point_count = points.shape[0]
    d.max_vertices = max_vertices
    d.z_min = z_min
    d.z_max = z_max
    d.position[:] = list(position)
    d.rotation[:] = list(rotation)
    d.density = density
    d.friction = friction
    d.restitution = restitution
    d.rolling_resistance = rolling_resistance
    d.category = category
    d.mask = mask
    d.sensor = 1 if sensor else 0
    d.mesh = mesh
    return d


_lib = None


def _declare(lib):
    P = C.c_void_p
    sig = {
        "tf_abi_version": ([], C.c_int),
        "tf_last_error": ([], C.c_char_p),
        "tf_default_settings": ([C.POINTER(tf_settings)], None),
        "tf_world_create": ([C.POINTER(tf_settings), C.c_int32, C.c_int32, C.POINTER(P)], C.c_int),
        "tf_world_destroy": ([P], C.c_int),
        "tf_world_count": ([P, C.POINTER(C.c_int32)], C.c_int),
        "tf_world_set_settings": ([P, C.POINTER(tf_settings)], C.c_int),
        "tf_mesh_create": ([P, P, C.c_int32, P, C.c_int32, C.POINTER(C.c_int32)], C.c_int),
        "tf_mesh_read": ([P, C.c_int32, P, P, P, P, P, P, P], C.c_int),
        "tf_body_destroy": ([P, C.c_int32, tf_id], C.c_int),
        "tf_shape_remove": ([P, C.c_int32, tf_id], C.c_int),
        "tf_shape_set_friction": ([P, C.c_int32, tf_id, C.c_float], C.c_int),
        "tf_shape_set_restitution": ([P, C.c_int32, tf_id, C.c_float], C.c_int),
        "tf_shape_set_rolling_resistance": ([P, C.c_int32, tf_id, C.c_float], C.c_int),
        "tf_shape_set_filter": ([P, C.c_int32, tf_id, C.c_uint32, C.c_uint32], C.c_int),
        "tf_body_set_transform": ([P, C.c_int32, tf_id, P, P], C.c_int),
        "tf_body_set_kinematic_target": ([P, C.c_int32, tf_id, P, P, C.c_float], C.c_int),
        "tf_body_set_motion_type": ([P, C.c_int32, tf_id, C.c_int32], C.c_int),
        "tf_body_add_force": ([P, C.c_int32, tf_id, P, P, C.c_int32], C.c_int),
        "tf_body_add_torque": ([P, C.c_int32, tf_id, P, C.c_int32], C.c_int),
        "tf_body_add_impulse": ([P, C.c_int32, tf_id, P, P, C.c_int32], C.c_int),
        "tf_body_set_damping": ([P, C.c_int32, tf_id, C.c_float, C.c_float], C.c_int),
        "tf_body_set_gravity_scale": ([P, C.c_int32, tf_id, C.c_float], C.c_int),
        "tf_body_wake": ([P, C.c_int32, tf_id], C.c_int),
        "tf_body_sleep": ([P, C.c_int32, tf_id], C.c_int),
        "tf_body_set_can_sleep": ([P, C.c_int32, tf_id, C.c_int32], C.c_int),
        "tf_world_set_mix": ([P, C.c_int32, C.c_int32], C.c_int),
        "tf_hull_compute": ([P, C.c_int32, C.c_int32, P, P, C.c_int32, P, C.c_int32], C.c_int),
        "tf_body_create": ([P, C.c_int32, C.POINTER(tf_body_desc), C.POINTER(tf_id)], C.c_int),
        "tf_shape_add": ([P, C.c_int32, tf_id, C.POINTER(tf_shape_desc), C.POINTER(tf_id)], C.c_int),
        "tf_bodies_create": ([P, C.c_int32, P, C.POINTER(tf_body_desc), P], C.c_int),
        "tf_shapes_add": ([P, C.c_int32, P, P, C.POINTER(tf_shape_desc), P], C.c_int),
        "tf_joint_create": ([P, C.c_int32, C.POINTER(tf_joint_desc), C.POINTER(tf_id)], C.c_int),
        "tf_joint_get_info": ([P, C.c_int32, tf_id, C.POINTER(tf_joint_info)], C.c_int),
        "tf_world_broken_joints": ([P, C.c_int32, P, C.c_int32, C.POINTER(C.c_int32)], C.c_int),
        "tf_joint_set_limits": ([P, C.c_int32, tf_id, C.c_int32, C.c_float, C.c_float], C.c_int),
        "tf_joint_set_motor": ([P, C.c_int32, tf_id, C.c_float, C.c_float], C.c_int),
        "tf_joint_set_spring": ([P, C.c_int32, tf_id, C.c_float, C.c_float], C.c_int),
        "tf_joint_set_friction": ([P, C.c_int32, tf_id, C.c_float], C.c_int),
        "tf_joint_set_swing": ([P, C.c_int32, tf_id, C.c_float, C.c_float], C.c_int),
        "tf_joint_set_break_limits": ([P, C.c_int32, tf_id, C.c_float, C.c_float], C.c_int),
        "tf_joint_destroy": ([P, C.c_int32, tf_id], C.c_int),
        "tf_world_step": ([P, C.c_float, C.c_int32], C.c_int),
        "tf_world_step_graph": ([P, C.c_float, C.c_int32], C.c_int),
        "tf_world_synchronize": ([P], C.c_int),
        "tf_world_device_status": ([P, C.POINTER(C.c_uint32)], C.c_int),
        "tf_body_get_state": ([P, C.c_int32, tf_id, P, P, P, P], C.c_int),
        "tf_body_set_velocity": ([P, C.c_int32, tf_id, P, P], C.c_int),
        "tf_body_get_mass": ([P, C.c_int32, tf_id, P, P, P], C.c_int),
        "tf_body_is_awake": ([P, C.c_int32, tf_id, C.POINTER(C.c_int32)], C.c_int),
        "tf_world_body_count": ([P, C.POINTER(C.c_int64)], C.c_int),
        "tf_world_get_states": ([P, P, P, P, P, P], C.c_int),
        "tf_world_contacts": ([P, C.c_int32, C.c_int32, C.POINTER(tf_contact), C.c_int32, C.POINTER(C.c_int32)],
                              C.c_int),
        "tf_world_candidates": ([P, C.c_int32, P, C.c_int32, C.POINTER(C.c_int32)], C.c_int),
        "tf_world_contact_events": ([P, C.c_int32, C.POINTER(tf_contact_event), C.c_int32, C.POINTER(C.c_int32)],
                                    C.c_int),
        "tf_world_hit_events": ([P, C.c_int32, C.POINTER(tf_hit_event), C.c_int32, C.POINTER(C.c_int32)], C.c_int),
        "tf_world_profile": ([P, C.c_int32, C.POINTER(tf_profile)], C.c_int),
        "tf_world_awake_bodies": ([P, C.POINTER(C.c_int64)], C.c_int),
        "tf_world_launch_count": ([P, C.POINTER(C.c_int64)], C.c_int),
        "tf_world_elapsed_ms": ([P, C.POINTER(C.c_float)], C.c_int),
        "tf_world_body_steps": ([P, C.POINTER(C.c_int64)], C.c_int),
        "tf_world_add_forces": ([P, P, P], C.c_int),
        "tf_world_read_poses": ([P, P, P], C.c_int),
        "tf_world_read_poses_async": ([P, P, P], C.c_int),
        "tf_world_poses_wait": ([P], C.c_int),
        "tf_world_set_profiling": ([P, C.c_int32], C.c_int),
        "tf_world_kernel_times": ([P, P, P, C.c_int32, C.POINTER(C.c_int32)], C.c_int),
        "tf_kernel_name": ([C.c_int32], C.c_char_p),
        "tf_world_work_counts": ([P, P], C.c_int),
        "tf_world_solver_counts": ([P, C.c_int32, P], C.c_int),
        "tf_world_save_state": ([P, C.c_int32], C.c_int),
        "tf_world_restore_state": ([P, C.c_int32], C.c_int),
        "tf_world_autotune": ([P, C.c_float, C.c_int32, P], C.c_int),
        "tf_tape_record": ([P, C.c_float, C.c_int32], C.c_int),
        "tf_adjoint_forward": ([P, C.c_int32, P, P, P, P], C.c_int),
        "tf_adjoint_backward": ([P, P, P, P, P], C.c_int),
        "tf_adjoint_elapsed_ms": ([P, P], C.c_int),
        "tf_adjoint_branches": ([P, P], C.c_int),
        "tf_adjoint_backward_ms": ([P, P], C.c_int),
        "tf_world_set_launch": ([P, C.c_int32, C.c_int32, C.c_int32, C.c_int32], C.c_int),
        "tf_world_get_launch": ([P, C.c_int32, P], C.c_int),
        "tf_candidates_noalloc": ([P, P, P, P, C.c_int32, P, C.c_int32, P, P], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


# Every symbol include/twofold_b200.h declares.
EXPORTED = [
    "tf_abi_version", "tf_last_error", "tf_default_settings", "tf_world_create", "tf_world_destroy",
    "tf_world_count", "tf_world_set_settings", "tf_mesh_create", "tf_mesh_read", "tf_hull_compute", "tf_body_destroy", "tf_shape_remove",
    "tf_shape_set_friction", "tf_shape_set_restitution", "tf_shape_set_rolling_resistance", "tf_shape_set_filter",
    "tf_body_set_transform", "tf_body_set_kinematic_target", "tf_body_set_motion_type", "tf_body_add_force",
    "tf_body_add_torque", "tf_body_add_impulse", "tf_body_set_damping", "tf_body_set_gravity_scale", "tf_body_wake",
    "tf_body_sleep", "tf_body_set_can_sleep", "tf_world_set_mix", "tf_body_create", "tf_shape_add",
    "tf_bodies_create",
    "tf_shapes_add", "tf_joint_create", "tf_joint_get_info", "tf_world_broken_joints", "tf_joint_set_limits", "tf_joint_set_motor",
    "tf_joint_set_spring", "tf_joint_set_friction", "tf_joint_set_swing", "tf_joint_set_break_limits", "tf_joint_destroy", "tf_world_step", "tf_world_step_graph", "tf_world_synchronize", "tf_world_device_status",
    "tf_body_get_state", "tf_body_set_velocity", "tf_body_get_mass", "tf_body_is_awake", "tf_world_body_count",
    "tf_world_get_states", "tf_world_contacts", "tf_world_contact_events", "tf_world_hit_events", "tf_world_candidates", "tf_world_profile", "tf_world_awake_bodies",
    "tf_world_launch_count", "tf_world_elapsed_ms", "tf_world_body_steps", "tf_world_add_forces",
    "tf_world_read_poses", "tf_world_read_poses_async", "tf_world_poses_wait", "tf_world_set_profiling", "tf_world_kernel_times", "tf_kernel_name",
    "tf_world_work_counts", "tf_world_solver_counts", "tf_world_save_state", "tf_world_restore_state", "tf_world_autotune", "tf_tape_record", "tf_adjoint_forward",
    "tf_adjoint_backward", "tf_adjoint_elapsed_ms", "tf_adjoint_branches",
    "tf_adjoint_backward_ms", "tf_world_set_launch", "tf_world_get_launch", "tf_candidates_noalloc",
]


def load():
    """Loads the in-tree CUDA library. Raises if it was not built: there is no other implementation."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with twofold_b200.build.build()")
        _lib = _declare(C.CDLL(LIB_PATH))
    return _lib


def check(rc, lib=None):
    if rc != TF_OK:
        lib = lib or load()
        msg = lib.tf_last_error()
        raise RuntimeError(f"twofold_b200 error {rc}: {msg.decode() if msg else ''}")


def hull_compute(points, max_vertices, lib=None):
    """tf_hull_compute: (vertices (n, 3) float32, faces as lists of vertex indices) of a point cloud (m, 3)."""
    lib = lib or load()
    return _hull_call(lib.tf_hull_compute, points, max_vertices, check)


def _hull_call(fn, points, max_vertices, checker):
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    counts = np.zeros(2, np.int32)
    checker(fn(pts.ctypes.data, len(pts), int(max_vertices), counts.ctypes.data, None, 0, None, 0))
    verts = np.zeros((max(int(counts[0]), 1), 3), np.float32)
    words = np.zeros(max(int(counts[1]), 1), np.int32)
    checker(fn(pts.ctypes.data, len(pts), int(max_vertices), counts.ctypes.data, verts.ctypes.data, int(counts[0]),
               words.ctypes.data, int(counts[1])))
    faces, at = [], 0
    while at < int(counts[1]):
        k = int(words[at])
        faces.append(words[at + 1:at + 1 + k].tolist())
        at += 1 + k
    return verts[:int(counts[0])], faces
