"""Python view of the C ABI: a batch of worlds built from scenes.Scene descriptor arrays.

This is how tests and bench.py drive the library; every call goes through libtwofold_b200.so.
"""
import ctypes as C

import numpy as np

from . import abi


# The World calls between steps, by name (include/twofold/world.h:375-463), in the order the oracle's harness
# numbers them.
CALLS = ("destroy_body", "remove_shape", "friction", "restitution", "rolling_resistance", "filter", "transform",
         "kinematic_target", "motion_type", "force", "force_at", "torque", "impulse", "impulse_at", "damping",
         "gravity_scale", "wake", "sleep", "can_sleep", "velocity", "spin")


class Batch:
    """One tf_world handle holding len(worlds) independent worlds on one CUDA device."""

    def __init__(self, worlds, settings=None, device=0):
        self.lib = abi.load()
        self.settings = settings if settings is not None else abi.default_settings()
        self.n = len(worlds)
        h = C.c_void_p()
        abi.check(self.lib.tf_world_create(C.byref(self.settings), self.n, device, C.byref(h)), self.lib)
        self.h = h
        self.body_counts = []
        for wi, w in enumerate(worlds):
            nb, ns = len(w.bodies), len(w.shapes)
            world_of = np.full(nb, wi, np.int32)
            abi.check(self.lib.tf_bodies_create(self.h, nb, world_of.ctypes.data,
                                                w.bodies.ctypes.data_as(C.POINTER(abi.tf_body_desc)), None), self.lib)
            shapes = w.shapes
            if getattr(w, "meshes", None):
                # A world's shapes name its meshes by position; the handle names them by its own ids.
                ids = [self.create_mesh(v, i) for v, i in w.meshes]
                shapes = w.shapes.copy()
                named = shapes["geometry"] == abi.TF_MESH
                shapes["mesh"][named] = np.asarray(ids, np.int32)[shapes["mesh"][named]]
            world_of = np.full(ns, wi, np.int32)
            abi.check(self.lib.tf_shapes_add(self.h, ns, world_of.ctypes.data, w.body_of.ctypes.data,
                                             shapes.ctypes.data_as(C.POINTER(abi.tf_shape_desc)), None), self.lib)
            for j in getattr(w, "joints", []):
                self.joint_create(wi, j)
            self.body_counts.append(nb)
        self.offsets = np.concatenate([[0], np.cumsum(self.body_counts)]).astype(np.int64)

    def create_mesh(self, vertices, indices):
        """tf_mesh_create: a TriangleMesh every world of the batch may use; returns its id."""
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        i = np.ascontiguousarray(indices, np.uint32).reshape(-1)
        out = C.c_int32(-1)
        abi.check(self.lib.tf_mesh_create(self.h, v.ctypes.data, len(v), i.ctypes.data, len(i), C.byref(out)), self.lib)
        return out.value

    def read_mesh(self, mesh):
        """The built mesh: vertices, indices, normals, edge flags, node bounds (lo, hi) and ranges (first, count)."""
        counts = np.zeros(3, np.int32)
        abi.check(self.lib.tf_mesh_read(self.h, mesh, counts.ctypes.data, None, None, None, None, None, None), self.lib)
        nv, nt, nn = (int(x) for x in counts)
        out = {"vertices": np.zeros((nv, 3), np.float32), "indices": np.zeros(3 * nt, np.uint32),
               "normals": np.zeros((nt, 3), np.float32), "edges": np.zeros(nt, np.uint8),
               "node_bounds": np.zeros((nn, 6), np.float32), "node_ranges": np.zeros((nn, 2), np.int32)}
        abi.check(self.lib.tf_mesh_read(self.h, mesh, counts.ctypes.data, *(out[k].ctypes.data for k in
                                        ("vertices", "indices", "normals", "edges", "node_bounds", "node_ranges"))),
                  self.lib)
        return out

    @classmethod
    def from_scene(cls, scene, device=0):
        return cls(scene.worlds, scene.settings, device)

    def close(self):
        if self.h:
            self.lib.tf_world_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt, n=1, graph=False):
        fn = self.lib.tf_world_step_graph if graph else self.lib.tf_world_step
        return fn(self.h, C.c_float(dt), n)

    def step_checked(self, dt, n=1, graph=False):
        abi.check(self.step(dt, n, graph), self.lib)

    def states(self):
        total = int(self.offsets[-1])
        p = np.zeros((total, 3), np.float32)
        q = np.zeros((total, 4), np.float32)
        v = np.zeros((total, 3), np.float32)
        w = np.zeros((total, 3), np.float32)
        awake = np.zeros(total, np.int32)
        abi.check(self.lib.tf_world_get_states(self.h, p.ctypes.data, q.ctypes.data, v.ctypes.data, w.ctypes.data,
                                               awake.ctypes.data), self.lib)
        return {"p": p, "q": q, "v": v, "w": w, "awake": awake}

    def world_states(self, wi):
        s = self.states()
        a, b = self.offsets[wi], self.offsets[wi + 1]
        return {k: v[a:b] for k, v in s.items()}

    def candidates(self, wi=0):
        n = C.c_int32(0)
        abi.check(self.lib.tf_world_candidates(self.h, wi, None, 0, C.byref(n)), self.lib)
        out = np.zeros(max(n.value, 1), np.uint64)
        abi.check(self.lib.tf_world_candidates(self.h, wi, out.ctypes.data, n.value, C.byref(n)), self.lib)
        return out[:n.value]

    def contacts(self, wi=0, mode=1):
        n = C.c_int32(0)
        abi.check(self.lib.tf_world_contacts(self.h, wi, mode, None, 0, C.byref(n)), self.lib)
        arr = (abi.tf_contact * max(n.value, 1))()
        abi.check(self.lib.tf_world_contacts(self.h, wi, mode, arr, n.value, C.byref(n)), self.lib)
        return list(arr)[:n.value]

    def joint_create(self, wi, desc):
        out = abi.tf_id()
        abi.check(self.lib.tf_joint_create(self.h, wi, C.byref(desc), C.byref(out)), self.lib)
        return out

    def joint_info(self, wi, joint):
        info = abi.tf_joint_info()
        abi.check(self.lib.tf_joint_get_info(self.h, wi, joint, C.byref(info)), self.lib)
        return info

    def joint_set(self, wi, joint, what, *values):
        """World::setJointLimits (limited, lower, upper), setJointMotor (speed, max), setJointSpring (hertz,
        damping), setJointFriction (max), setJointSwing (y, z), setJointBreakLimits (force, torque) and
        destroyJoint, by name: limits, motor, spring, friction, swing, break, destroy."""
        fn = {"limits": self.lib.tf_joint_set_limits, "motor": self.lib.tf_joint_set_motor,
              "spring": self.lib.tf_joint_set_spring, "friction": self.lib.tf_joint_set_friction,
              "swing": self.lib.tf_joint_set_swing, "break": self.lib.tf_joint_set_break_limits,
              "destroy": self.lib.tf_joint_destroy}[what]
        if what == "limits":
            values = (int(values[0]), *values[1:])
        abi.check(fn(self.h, wi, joint, *values), self.lib)

    def broken_joints(self, wi=0):
        n = C.c_int32(0)
        abi.check(self.lib.tf_world_broken_joints(self.h, wi, None, 0, C.byref(n)), self.lib)
        arr = (abi.tf_id * max(n.value, 1))()
        abi.check(self.lib.tf_world_broken_joints(self.h, wi, arr, n.value, C.byref(n)), self.lib)
        return [(x.index, x.generation) for x in list(arr)[:n.value]]

    def contact_events(self, wi=0):
        """World::contactEvents of world wi's last step: (shape_a, shape_b, body_a, body_b, begin) tuples."""
        n = C.c_int32(0)
        abi.check(self.lib.tf_world_contact_events(self.h, wi, None, 0, C.byref(n)), self.lib)
        arr = (abi.tf_contact_event * max(n.value, 1))()
        abi.check(self.lib.tf_world_contact_events(self.h, wi, arr, n.value, C.byref(n)), self.lib)
        return [(e.shape_a, e.shape_b, e.body_a, e.body_b, bool(e.begin)) for e in list(arr)[:n.value]]

    def hit_events(self, wi=0):
        """World::hitEvents of world wi's last step: (shape_a, shape_b, body_a, body_b, point, normal, speed)."""
        n = C.c_int32(0)
        abi.check(self.lib.tf_world_hit_events(self.h, wi, None, 0, C.byref(n)), self.lib)
        arr = (abi.tf_hit_event * max(n.value, 1))()
        abi.check(self.lib.tf_world_hit_events(self.h, wi, arr, n.value, C.byref(n)), self.lib)
        return [(e.shape_a, e.shape_b, e.body_a, e.body_b, np.array(e.point[:], np.float32),
                 np.array(e.normal[:], np.float32), np.float32(e.speed)) for e in list(arr)[:n.value]]

    def profile(self, wi=0):
        p = abi.tf_profile()
        abi.check(self.lib.tf_world_profile(self.h, wi, C.byref(p)), self.lib)
        return p

    def mass(self, wi, index, generation=0):
        m = C.c_float(0)
        c = np.zeros(3, np.float32)
        i = np.zeros(9, np.float32)
        abi.check(self.lib.tf_body_get_mass(self.h, wi, abi.tf_id(index, generation), C.byref(m), c.ctypes.data,
                                            i.ctypes.data), self.lib)
        return m.value, c, i.reshape(3, 3)

    def awake_bodies(self):
        n = C.c_int64(0)
        abi.check(self.lib.tf_world_awake_bodies(self.h, C.byref(n)), self.lib)
        return n.value

    def launches(self):
        n = C.c_int64(0)
        abi.check(self.lib.tf_world_launch_count(self.h, C.byref(n)), self.lib)
        return n.value

    def device_flags(self):
        f = C.c_uint32(0)
        abi.check(self.lib.tf_world_device_status(self.h, C.byref(f)), self.lib)
        return f.value

    # Timing and host traffic of a running batch.

    def elapsed_ms(self):
        ms = C.c_float(0)
        abi.check(self.lib.tf_world_elapsed_ms(self.h, C.byref(ms)), self.lib)
        return ms.value

    def body_steps(self):
        n = C.c_int64(0)
        abi.check(self.lib.tf_world_body_steps(self.h, C.byref(n)), self.lib)
        return n.value

    def add_forces(self, forces=None, torques=None):
        """forces/torques: float32 arrays (total_bodies, 3), ideally in pinned host memory."""
        f = forces.ctypes.data if forces is not None else None
        t = torques.ctypes.data if torques is not None else None
        abi.check(self.lib.tf_world_add_forces(self.h, f, t), self.lib)

    def read_poses(self, positions, rotations):
        abi.check(self.lib.tf_world_read_poses(self.h, positions.ctypes.data, rotations.ctypes.data), self.lib)

    def read_poses_async(self, positions, rotations):
        """Queues a pose read into (pinned) host arrays that must stay alive until poses_wait returns."""
        abi.check(self.lib.tf_world_read_poses_async(self.h, positions.ctypes.data, rotations.ctypes.data), self.lib)

    def poses_wait(self):
        abi.check(self.lib.tf_world_poses_wait(self.h), self.lib)

    def set_profiling(self, on=True):
        abi.check(self.lib.tf_world_set_profiling(self.h, 1 if on else 0), self.lib)

    def kernel_times(self):
        """{kernel name: (total ms, launches)} since profiling was turned on."""
        ms = np.zeros(16, np.float32)
        n = np.zeros(16, np.int64)
        cnt = C.c_int32(0)
        abi.check(self.lib.tf_world_kernel_times(self.h, ms.ctypes.data, n.ctypes.data, 16, C.byref(cnt)), self.lib)
        return {self.lib.tf_kernel_name(k).decode(): (float(ms[k]), int(n[k])) for k in range(cnt.value)}

    def work_counts(self):
        """Work of the last step: bodies, awake, candidates, contacts, active contacts, active points."""
        out = np.zeros(6, np.int64)
        abi.check(self.lib.tf_world_work_counts(self.h, out.ctypes.data), self.lib)
        keys = ("bodies", "awake", "candidates", "contacts", "active_contacts", "active_points")
        return dict(zip(keys, (int(x) for x in out)))

    def solver_counts(self, wi):
        """Solver work of world wi in the last step."""
        out = np.zeros(8, np.int32)
        abi.check(self.lib.tf_world_solver_counts(self.h, wi, out.ctypes.data), self.lib)
        keys = ("active", "colors", "rest", "impact", "impact_colors", "impact_rest", "fast", "fast_solid")
        return dict(zip(keys, (int(x) for x in out)))

    KERNELS = ("broadphase", "narrowphase", "wake", "prepare", "refresh", "substep", "finish", "collide")

    def set_launch(self, kernel, threads, big_bodies, smem_bytes):
        """Launch shape of one kernel (name or index; None for all): threads per CTA, the world size above
        which a world gets the whole CTA, and the CTA's staging bytes."""
        k = -1 if kernel is None else (self.KERNELS.index(kernel) if isinstance(kernel, str) else int(kernel))
        abi.check(self.lib.tf_world_set_launch(self.h, k, int(threads), int(big_bodies), int(smem_bytes)), self.lib)

    def call(self, wi, what, target, values=(), a=0, b=0):
        """A World call between steps on world wi (CALLS names them): target is a body or shape id (tf_id), values
        the call's floats (position then rotation x, y, z, w then dt; force then point; ...), a and b its
        integers (category and mask, motion type, wake)."""
        L, h = self.lib, self.h
        f = (C.c_float * 8)(*(list(values) + [0.0] * (8 - len(values))))
        P = C.c_void_p(C.addressof(f))
        at = C.c_void_p(C.addressof(f) + 12)  # values[3:]: a rotation, or a point
        rc = {
            "destroy_body": lambda: L.tf_body_destroy(h, wi, target),
            "remove_shape": lambda: L.tf_shape_remove(h, wi, target),
            "friction": lambda: L.tf_shape_set_friction(h, wi, target, f[0]),
            "restitution": lambda: L.tf_shape_set_restitution(h, wi, target, f[0]),
            "rolling_resistance": lambda: L.tf_shape_set_rolling_resistance(h, wi, target, f[0]),
            "filter": lambda: L.tf_shape_set_filter(h, wi, target, a, b),
            "transform": lambda: L.tf_body_set_transform(h, wi, target, P, at),
            "kinematic_target": lambda: L.tf_body_set_kinematic_target(h, wi, target, P, at, f[7]),
            "motion_type": lambda: L.tf_body_set_motion_type(h, wi, target, a),
            "force": lambda: L.tf_body_add_force(h, wi, target, P, None, a),
            "force_at": lambda: L.tf_body_add_force(h, wi, target, P, at, a),
            "torque": lambda: L.tf_body_add_torque(h, wi, target, P, a),
            "impulse": lambda: L.tf_body_add_impulse(h, wi, target, P, None, a),
            "impulse_at": lambda: L.tf_body_add_impulse(h, wi, target, P, at, a),
            "damping": lambda: L.tf_body_set_damping(h, wi, target, f[0], f[1]),
            "gravity_scale": lambda: L.tf_body_set_gravity_scale(h, wi, target, f[0]),
            "wake": lambda: L.tf_body_wake(h, wi, target),
            "sleep": lambda: L.tf_body_sleep(h, wi, target),
            "can_sleep": lambda: L.tf_body_set_can_sleep(h, wi, target, a),
            "velocity": lambda: L.tf_body_set_velocity(h, wi, target, P, None),
            "spin": lambda: L.tf_body_set_velocity(h, wi, target, None, P),
        }[what]()
        abi.check(rc, L)

    def save_state(self, slot=0):
        """Snapshot of the batch's dynamic state on the device."""
        abi.check(self.lib.tf_world_save_state(self.h, slot), self.lib)

    def restore_state(self, slot=0):
        abi.check(self.lib.tf_world_restore_state(self.h, slot), self.lib)

    def autotune(self, dt, trial_steps=2):
        """Picks each kernel's launch shape by timing candidates on the current state (left as it was).
        Returns {kernel: (threads, big-world threshold, shared bytes)}."""
        out = np.zeros(3 * len(self.KERNELS), np.uint32)
        abi.check(self.lib.tf_world_autotune(self.h, C.c_float(dt), trial_steps, out.ctypes.data), self.lib)
        # A substep shape whose threshold is all ones is the flat solve, which set_launch takes as -1.
        as_int = lambda x: -1 if int(x) == 0xFFFFFFFF else int(x)
        return {k: tuple(as_int(x) for x in out[3 * i:3 * i + 3]) for i, k in enumerate(self.KERNELS)}

    # ---- differentiation ----

    def tape_record(self, dt, n_steps):
        """Steps n_steps times, recording each step's contact set for the differentiable model."""
        abi.check(self.lib.tf_tape_record(self.h, C.c_float(dt), n_steps), self.lib)

    def adjoint_forward(self, precision=64, initial=None, mass=None, friction=None):
        """The model from the recorded initial state; returns the final state, (bodies, 13) float64:
        center of mass, rotation (x, y, z, w), linear and angular velocity."""
        total = int(self.offsets[-1])
        out = np.zeros((total, 13), np.float64)
        args = []
        for a in (initial, mass, friction):
            args.append(None if a is None else np.ascontiguousarray(a, np.float64))
        ptr = [None if a is None else a.ctypes.data for a in args]
        abi.check(self.lib.tf_adjoint_forward(self.h, precision, ptr[0], ptr[1], ptr[2], out.ctypes.data), self.lib)
        return out

    def adjoint_backward(self, grad_final, n_shapes):
        """d loss / d (initial state, mass, friction) from d loss / d final state (bodies, 13)."""
        total = int(self.offsets[-1])
        g = np.ascontiguousarray(grad_final, np.float64)
        gi = np.zeros((total, 13), np.float64)
        gm = np.zeros(total, np.float64)
        gf = np.zeros(n_shapes, np.float64)
        abi.check(self.lib.tf_adjoint_backward(self.h, g.ctypes.data, gi.ctypes.data, gm.ctypes.data, gf.ctypes.data),
                  self.lib)
        return gi, gm, gf

    def adjoint_branches(self):
        """Per world, the branch signature of the last adjoint_forward run (uint64)."""
        out = np.zeros(len(self.offsets) - 1, np.uint64)
        abi.check(self.lib.tf_adjoint_branches(self.h, out.ctypes.data), self.lib)
        return out

    def adjoint_backward_ms(self):
        """The last backward's recomputation and reverse walk, each summed over its chunks (ms)."""
        ms = np.zeros(2, np.float32)
        abi.check(self.lib.tf_adjoint_backward_ms(self.h, ms.ctypes.data), self.lib)
        return float(ms[0]), float(ms[1])

    def adjoint_ms(self):
        ms = np.zeros(2, np.float32)
        abi.check(self.lib.tf_adjoint_elapsed_ms(self.h, ms.ctypes.data), self.lib)
        return float(ms[0]), float(ms[1])

    def launch(self, kernel):
        """The launch shape in use for one kernel, after the batch was laid out on the device."""
        k = self.KERNELS.index(kernel) if isinstance(kernel, str) else int(kernel)
        out = np.zeros(6, np.uint32)
        abi.check(self.lib.tf_world_get_launch(self.h, k, out.ctypes.data), self.lib)
        keys = ("threads", "big_bodies", "smem_bytes", "grid", "stage_big", "stage_small")
        return dict(zip(keys, (int(x) for x in out)))
