"""Seeded synthetic scenes for the five benchmark configurations, as descriptor arrays.

Both the B200 library and the reference oracle are built from exactly these arrays, so both sides step
identical input. No public dataset exists for this path; every scene is generated from a seed.

A `Scene` is a list of worlds. Each world holds numpy structured arrays laid out like tf_body_desc and
tf_shape_desc (include/twofold_b200.h) plus `body_of`, the index of each shape's body in its world.
"""
import ctypes as C
import math

import numpy as np

from . import abi


def _dtype_of(struct):
    names, formats, offsets = [], [], []
    for name, ctype in struct._fields_:
        off = getattr(struct, name).offset
        if isinstance(ctype, type) and issubclass(ctype, C._Pointer):
            fmt = np.uint64
        else:
            fmt = np.dtype(ctype)
        names.append(name)
        formats.append(fmt)
        offsets.append(off)
    return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": C.sizeof(struct)})


BODY_DTYPE = _dtype_of(abi.tf_body_desc)
SHAPE_DTYPE = _dtype_of(abi.tf_shape_desc)

F32 = np.float32


def _f(x):
    return np.float32(x)


def from_to_z_to_y():
    """Quat::fromTo({0,0,1}, {0,1,0}) in float arithmetic (include/twofold/math.h:150-156)."""
    # d = 0, c = cross(z, y) = (-1, 0, 0), s = sqrt((1 + d) * 2)
    s = np.sqrt(_f(2.0), dtype=F32)
    return (_f(-1.0) / s, _f(0.0), _f(0.0), _f(0.5) * s)


GROUND_ROTATION = from_to_z_to_y()


class World:
    def __init__(self, bodies, shapes, body_of, meta=None):
        self.bodies = bodies
        self.shapes = shapes
        self.body_of = np.ascontiguousarray(body_of, dtype=np.uint32)
        self.meta = meta or {}
        self.keepalive = []
        # Joints as tf_joint_desc, created after the bodies and shapes; body ids are positions in `bodies`.
        self.joints = []
        # TriangleMeshes as (vertices (n, 3), indices (3 m,)); a TF_MESH shape's "mesh" is a position here.
        self.meshes = []

    @property
    def dynamic_count(self):
        return int(np.count_nonzero(self.bodies["type"] == abi.TF_DYNAMIC))


class Scene:
    def __init__(self, name, worlds, settings=None, dt=1.0 / 60.0, steps=1):
        self.name = name
        self.worlds = worlds
        self.settings = settings if settings is not None else abi.default_settings()
        self.dt = float(np.float32(dt))
        self.steps = steps

    @property
    def body_count(self):
        return sum(len(w.bodies) for w in self.worlds)

    @property
    def dynamic_count(self):
        return sum(w.dynamic_count for w in self.worlds)


def _bodies(n):
    b = np.zeros(n, dtype=BODY_DTYPE)
    b["type"] = abi.TF_DYNAMIC
    b["rotation"][:, 3] = 1.0
    b["lock_frame"][:, 3] = 1.0
    b["gravity_scale"] = 1.0
    b["awake"] = 1
    b["can_sleep"] = 1
    return b


def _shapes(n):
    s = np.zeros(n, dtype=SHAPE_DTYPE)
    s["geometry"] = abi.TF_BOX
    s["radius"] = 0.5
    s["half_extents"] = 0.5
    s["half_height"] = 0.5
    s["max_vertices"] = 64
    s["z_min"] = -0.5
    s["z_max"] = 0.5
    s["rotation"][:, 3] = 1.0
    s["density"] = 1.0
    s["friction"] = 0.5
    s["category"] = 1
    s["mask"] = 0xFFFFFFFF
    s["mesh"] = -1
    return s


def _ground(bodies, shapes, friction=0.6, restitution=0.0):
    """A static half-space y <= 0, as tests/test_world.cpp:16-26 adds it."""
    bodies["type"][0] = abi.TF_STATIC
    bodies["rotation"][0] = GROUND_ROTATION
    shapes["geometry"][0] = abi.TF_HALFSPACE
    shapes["friction"][0] = friction
    shapes["restitution"][0] = restitution


def _uniform_quats(rng, n):
    """Shoemake's uniform random rotations."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
    q = np.stack([a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2), b * np.sin(2 * np.pi * u3),
                  b * np.cos(2 * np.pi * u3)], axis=1)
    return q.astype(F32)


def pyramid(rows=20, pitch=1.0, jitter=1e-4, seed=0, friction=0.6, sleep=False):
    """Box pyramid: `rows` layers of unit boxes (half extents 0.5, density 1) on a static half-space,
    row r holding rows - r boxes at pitch spacing, every coordinate jittered by U[-jitter, jitter]."""
    n = rows * (rows + 1) // 2
    rng = np.random.default_rng(seed)
    bodies, shapes = _bodies(n + 1), _shapes(n + 1)
    _ground(bodies, shapes, friction=friction)
    k = 1
    for r in range(rows):
        for i in range(rows - r):
            x = (i - (rows - 1 - r) / 2.0) * pitch
            y = 0.5 + r * pitch
            bodies["position"][k] = (x, y, 0.0)
            k += 1
    bodies["position"][1:] += rng.uniform(-jitter, jitter, size=(n, 3)).astype(F32)
    bodies["can_sleep"][1:] = 1 if sleep else 0
    shapes["friction"][1:] = friction
    return World(bodies, shapes, np.arange(n + 1), meta={"kind": "pyramid"})


def config1():
    """Box pyramid, plain method: 20 layers, 210 dynamic unit boxes, sleeping off, 300 steps."""
    return Scene("box_pyramid_210", [pyramid(20)], steps=300)


def _world_c4(rng, n_bodies):
    bodies, shapes = _bodies(n_bodies + 1), _shapes(n_bodies + 1)
    friction = _f(rng.uniform(0.2, 1.0))
    restitution = _f(rng.uniform(0.0, 0.3))
    _ground(bodies, shapes, friction=friction, restitution=restitution)
    is_box = rng.random(n_bodies) < 0.7
    half = rng.uniform(0.2, 0.6, size=(n_bodies, 3)).astype(F32)
    radius = rng.uniform(0.2, 0.5, size=n_bodies).astype(F32)
    g = np.where(is_box, abi.TF_BOX, abi.TF_SPHERE)
    shapes["geometry"][1:] = g
    shapes["half_extents"][1:] = half
    shapes["radius"][1:] = radius
    shapes["friction"][1:] = friction
    shapes["restitution"][1:] = restitution
    if rng.random() < 0.5:
        # Stack: columns on a 1.3 m grid over the 10 x 10 m footprint, layers 1.3 m apart.
        cols = 7
        idx = np.arange(n_bodies)
        layer, cell = idx // (cols * cols), idx % (cols * cols)
        cx, cz = cell % cols, cell // cols
        pos = np.stack([(cx - (cols - 1) / 2.0) * 1.3, 0.65 + 1.3 * layer, (cz - (cols - 1) / 2.0) * 1.3], axis=1)
        bodies["position"][1:] = pos.astype(F32)
        kind = "stack"
    else:
        # Scatter: jittered cells over the footprint, rising from 1 m, randomly turned. Cells are wide enough
        # that bounding spheres (at most 1.04 m for the largest box) never overlap.
        cols, pitch = 5, 2.1
        idx = np.arange(n_bodies)
        layer, cell = idx // (cols * cols), idx % (cols * cols)
        cx, cz = cell % cols, cell // cols
        jit = rng.uniform(-0.02, 0.02, size=(n_bodies, 3))
        pos = np.stack([(cx - (cols - 1) / 2.0) * pitch, 1.1 + pitch * layer, (cz - (cols - 1) / 2.0) * pitch],
                       axis=1) + jit
        bodies["position"][1:] = pos.astype(F32)
        bodies["rotation"][1:] = _uniform_quats(rng, n_bodies)
        kind = "scatter"
    return World(bodies, shapes, np.arange(n_bodies + 1), meta={"kind": kind})


def _c4_count(rng, min_bodies, max_bodies):
    n = int(math.floor(math.exp(rng.uniform(math.log(min_bodies), math.log(max_bodies + 1)))))
    return max(min_bodies, min(max_bodies, n))


def config4(n_worlds=4096, seed=0, min_bodies=8, max_bodies=512, only=None):
    """Batched uneven worlds: body counts log-uniform in [8, 512], 70% boxes and 30% spheres in a random
    stack or scatter above a half-space, per-world friction U[0.2, 1] and restitution U[0, 0.3]. Each world
    comes from its own seed (seed, world), so `only` (world numbers of the n_worlds set, in the order given)
    builds a shard of the set with the very worlds the whole set has."""
    worlds = []
    for w in (range(n_worlds) if only is None else only):
        rng = np.random.default_rng([seed, int(w)])
        worlds.append(_world_c4(rng, _c4_count(rng, min_bodies, max_bodies)))
    return Scene("batched_uneven_4096", worlds, steps=240)


def config4_bodies(n_worlds=4096, seed=0, min_bodies=8, max_bodies=512):
    """The dynamic body count of each world of config4 (the ground is not counted), without building them."""
    return np.array([_c4_count(np.random.default_rng([seed, w]), min_bodies, max_bodies) for w in range(n_worlds)],
                    np.int64)


def impact_world(rng):
    """One world of the differentiable impact: a 4x4x4 wall of 0.25 m boxes hit by a dense sphere."""
    n = 64
    bodies, shapes = _bodies(n + 2), _shapes(n + 2)
    friction = _f(rng.uniform(0.3, 0.9))
    _ground(bodies, shapes, friction=friction)
    mass = rng.uniform(0.5, 2.0, size=n).astype(F32)
    k = 1
    for i in range(4):
        for j in range(4):
            for kk in range(4):
                bodies["position"][k] = (3.0 + 0.5 * (i - 1.5), 0.25 + 0.5 * j, 0.5 * (kk - 1.5))
                k += 1
    shapes["half_extents"][1:n + 1] = 0.25
    shapes["density"][1:n + 1] = mass / _f(0.125)
    shapes["friction"][1:] = friction
    bodies["position"][n + 1] = (0.0, 0.5, 0.0)
    bodies["linear_velocity"][n + 1] = (np.array([10.0, 2.0, 0.0]) + rng.normal(0.0, 1.0, size=3)).astype(F32)
    shapes["geometry"][n + 1] = abi.TF_SPHERE
    shapes["radius"][n + 1] = 0.25
    shapes["density"][n + 1] = 8.0
    return World(bodies, shapes, np.arange(n + 2), meta={"kind": "impact", "mass": mass})


def config5(n_worlds=1024, seed=0):
    """Differentiable batched impact: 1024 walls of 64 boxes hit by a sphere, 120 steps."""
    worlds = [impact_world(np.random.default_rng([seed, 5, w])) for w in range(n_worlds)]
    return Scene("impact_1024", worlds, steps=120)


def _set_points(world, index, pts):
    """Points of shape `index` (prism outline as (x, y) pairs, or hull points), kept alive with the world."""
    arr = np.ascontiguousarray(pts, dtype=F32)
    world.keepalive.append(arr)
    world.shapes["points"][index] = arr.ctypes.data
    world.shapes["point_count"][index] = len(arr)


def prisms(n=24, seed=0, degenerate=True):
    """Prisms of 3-8 vertices and boxes, randomly turned, dropped in a loose column onto a half-space. With
    `degenerate`, some outlines are clockwise, repeat a point, hold a nearly collinear point, or are flat, so
    the outline cleaning runs on every path."""
    rng = np.random.default_rng([seed, 3])
    b, s = _bodies(n + 1), _shapes(n + 1)
    _ground(b, s, friction=0.6)
    w = World(b, s, np.arange(n + 1))
    b["rotation"][1:] = _uniform_quats(rng, n)
    for i in range(1, n + 1):
        b["position"][i] = (rng.uniform(-1.5, 1.5), 0.8 + 0.9 * i, rng.uniform(-1.5, 1.5))
        s["friction"][i] = _f(rng.uniform(0.3, 0.9))
        if i % 4 == 0:
            s["half_extents"][i] = rng.uniform(0.2, 0.5, size=3).astype(F32)
            continue
        k = int(rng.integers(3, 9))
        r = rng.uniform(0.2, 0.6)
        ang = np.sort(rng.uniform(0.0, 2 * math.pi, size=k))
        pts = np.stack([r * np.cos(ang), r * np.sin(ang)], 1).astype(F32)
        if degenerate and i % 5 == 1:
            pts = pts[::-1]                                  # clockwise
        if degenerate and i % 7 == 2:
            pts = np.concatenate([pts, pts[:1]])             # a repeated point
        if degenerate and i % 9 == 3:
            mid = (pts[0] + pts[1]) * F32(0.5)
            pts = np.concatenate([pts[:1], mid[None], pts[1:]])  # a point on an edge
        s["geometry"][i] = abi.TF_PRISM
        _set_points(w, i, pts)
        z = rng.uniform(0.15, 0.5)
        s["z_min"][i] = _f(-z)
        s["z_max"][i] = _f(z)
        if degenerate and i % 11 == 4:
            s["z_max"][i] = s["z_min"][i]                    # flat: thickened to a slab
    return w


def _sphere_points(rng, n, r):
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True) * r).astype(F32)


def hulls(n=24, seed=0, degenerate=True, max_vertices=16):
    """Hulls of 16 points uniform on a 0.5 m sphere (vertex limit 16), some boxes and spheres, randomly turned
    and dropped in a loose column onto a half-space. With `degenerate`, some clouds are flat, collinear, a
    single point, or repeat points, so the hull's thickening and tolerance paths run."""
    rng = np.random.default_rng([seed, 2])
    b, s = _bodies(n + 1), _shapes(n + 1)
    _ground(b, s, friction=0.6)
    w = World(b, s, np.arange(n + 1))
    b["rotation"][1:] = _uniform_quats(rng, n)
    for i in range(1, n + 1):
        b["position"][i] = (rng.uniform(-1.5, 1.5), 0.8 + 1.0 * i, rng.uniform(-1.5, 1.5))
        s["friction"][i] = _f(rng.uniform(0.3, 0.9))
        s["density"][i] = _f(rng.uniform(0.5, 2.0))
        if i % 6 == 0:
            s["half_extents"][i] = rng.uniform(0.2, 0.5, size=3).astype(F32)
            continue
        if i % 6 == 3:
            s["geometry"][i] = abi.TF_SPHERE
            s["radius"][i] = _f(rng.uniform(0.2, 0.5))
            continue
        pts = _sphere_points(rng, 16, 0.5)
        if degenerate and i % 7 == 1:
            pts[:, 2] = 0.0                                          # flat
        if degenerate and i % 11 == 2:
            pts = (np.outer(rng.uniform(-0.5, 0.5, 16), [1, 2, 3]) / 4).astype(F32)  # collinear
        if degenerate and i % 13 == 4:
            pts = np.zeros((3, 3), F32)                              # one point
        if degenerate and i % 5 == 2:
            pts = np.concatenate([pts, pts[:4]])                     # repeated points
        s["geometry"][i] = abi.TF_HULL
        s["max_vertices"][i] = max_vertices
        _set_points(w, i, pts)
    return w


def planar(n=16384, cols=46, spheres=256, seed=0, sphere_height=(10.0, 600.0), floor="box", restitution=0.0,
           discs=False):
    """Bodies locked to the z = 0 plane (lock frame identity): half boxes with half extents x, y ~ U[0.2, 0.6]
    and z = 0.5, half prisms of 3-8 vertices at sorted random angles on a circle of radius U[0.2, 0.6] with z in
    [-0.5, 0.5]; friction U[0.3, 0.9], a random turn in the plane; laid out on a `cols`-column grid of 1.7 m
    centred on x = 0, rows from y = 2 at 1.7 m. Static container: a floor box reaching 1.9 m past the grid
    (41 m half width at 46 columns) with 0.5 m walls 60 m tall at its ends, or a half-space floor alone
    (`floor="halfspace"`). `spheres` free spheres (r 0.5, density 4, not locked) at x ~ U over the grid,
    y ~ U[sphere_height], z = 0. With `discs`, every third prism is a cylinder of radius U[0.2, 0.6] and half
    height 0.5 standing on the plane (a circle profile)."""
    rng = np.random.default_rng([seed, 3, 3])
    n_static = 3 if floor == "box" else 1
    total = n_static + n + spheres
    b, s = _bodies(total), _shapes(total)
    w = World(b, s, np.arange(total), meta={"kind": "planar", "floor": floor})
    half = 0.85 * cols + 1.9
    b["type"][:n_static] = abi.TF_STATIC
    if floor == "box":
        b["position"][0] = (0.0, -0.5, 0.0)
        s["half_extents"][0] = (half, 0.5, 2.0)
        for k, side in ((1, -1.0), (2, 1.0)):
            b["position"][k] = (side * (half - 0.5), 30.0, 0.0)
            s["half_extents"][k] = (0.5, 30.0, 2.0)
        s["friction"][:n_static] = 0.6
    else:
        _ground(b, s, friction=0.6)
    s["restitution"][:] = restitution
    first = n_static
    idx = np.arange(n)
    row, col = idx // cols, idx % cols
    b["position"][first:first + n, 0] = (-0.85 * (cols - 1) + 1.7 * col).astype(F32)
    b["position"][first:first + n, 1] = (2.0 + 1.7 * row).astype(F32)
    angle = rng.uniform(0.0, 2 * math.pi, size=n)
    b["rotation"][first:first + n] = np.stack(
        [np.zeros(n), np.zeros(n), np.sin(0.5 * angle), np.cos(0.5 * angle)], 1).astype(F32)
    b["locks"][first:first + n] = abi.TF_LOCK_PLANAR
    s["friction"][first:first + n] = rng.uniform(0.3, 0.9, size=n).astype(F32)
    for i in range(n):
        k = first + i
        if i % 2 == 0:
            s["half_extents"][k] = (rng.uniform(0.2, 0.6), rng.uniform(0.2, 0.6), 0.5)
            continue
        m = int(rng.integers(3, 9))
        r = rng.uniform(0.2, 0.6)
        ang = np.sort(rng.uniform(0.0, 2 * math.pi, size=m))
        if discs and i % 6 == 1:
            s["geometry"][k] = abi.TF_CYLINDER
            s["radius"][k] = r
            s["half_height"][k] = 0.5
            continue
        s["geometry"][k] = abi.TF_PRISM
        _set_points(w, k, np.stack([r * np.cos(ang), r * np.sin(ang)], 1))
        s["z_min"][k] = -0.5
        s["z_max"][k] = 0.5
    first += n
    if spheres:
        sl = slice(first, first + spheres)
        b["position"][sl, 0] = rng.uniform(-0.85 * (cols - 1), 0.85 * (cols - 1), size=spheres).astype(F32)
        b["position"][sl, 1] = rng.uniform(sphere_height[0], sphere_height[1], size=spheres).astype(F32)
        s["geometry"][sl] = abi.TF_SPHERE
        s["radius"][sl] = 0.5
        s["density"][sl] = 4.0
    return w


def bullets(n=24, seed=0, speed=(40.0, 80.0)):
    """Fast small bodies that the continuous pass must catch: spheres of radius U[0.03, 0.08], thin boxes
    (half extents 0.02 x 0.1 x 0.1) and small boxes, shot at U[speed] m/s along x, half of them at a static
    thin wall (half thickness 0.05) at x = 6 and half at a kinematic wall at x = -6 moving at 1 m/s in +x,
    past three dynamic thin plates (half thickness 0.02) standing on a half-space between them."""
    rng = np.random.default_rng([seed, 7])
    plates = 3
    total = 3 + plates + n
    b, s = _bodies(total), _shapes(total)
    w = World(b, s, np.arange(total), meta={"kind": "bullets"})
    _ground(b, s, friction=0.6)
    b["type"][1] = abi.TF_STATIC
    b["position"][1] = (6.0, 1.5, 0.0)
    s["half_extents"][1] = (0.05, 1.5, 1.5)
    b["type"][2] = abi.TF_KINEMATIC
    b["position"][2] = (-6.0, 1.5, 0.0)
    b["linear_velocity"][2] = (1.0, 0.0, 0.0)
    s["half_extents"][2] = (0.1, 1.5, 1.5)
    for k in range(plates):
        i = 3 + k
        b["position"][i] = (-3.0 + 3.0 * k, 0.5, rng.uniform(-0.2, 0.2))
        s["half_extents"][i] = (0.02, 0.5, 0.5)
    first = 3 + plates
    for k in range(n):
        i = first + k
        side = 1.0 if k % 2 == 0 else -1.0
        b["position"][i] = (rng.uniform(-1.5, 1.5), rng.uniform(0.3, 2.6), rng.uniform(-1.2, 1.2))
        b["linear_velocity"][i] = (side * rng.uniform(*speed), rng.uniform(-2.0, 2.0), rng.uniform(-2.0, 2.0))
        b["angular_velocity"][i] = rng.uniform(-5.0, 5.0, size=3)
        b["rotation"][i] = _uniform_quats(rng, 1)[0]
        kind = k % 3
        if kind == 0:
            s["geometry"][i] = abi.TF_SPHERE
            s["radius"][i] = rng.uniform(0.03, 0.08)
        elif kind == 1:
            s["half_extents"][i] = (0.02, 0.1, 0.1)
        else:
            s["half_extents"][i] = rng.uniform(0.05, 0.1, size=3)
        s["density"][i] = 2.0
    s["friction"][3:] = 0.5
    return w


def terrain_mesh(cells=256, cell=0.5, seed=0):
    """A height field of cells x cells squares of `cell` m, centred on the origin, two triangles a square
    facing +y: h = sum over k < 8 of 0.25 sin(a_k x + b_k z + phi_k), (a_k, b_k) = f_k (cos t_k, sin t_k),
    f_k ~ U[0.05, 0.5] rad/m, t_k and phi_k ~ U[0, 2 pi). Returns (vertices, indices)."""
    rng = np.random.default_rng([seed, 2, 1])
    f = rng.uniform(0.05, 0.5, size=8)
    t = rng.uniform(0.0, 2 * math.pi, size=8)
    phi = rng.uniform(0.0, 2 * math.pi, size=8)
    a, b = f * np.cos(t), f * np.sin(t)
    g = (np.arange(cells + 1) - cells / 2.0) * cell
    x, z = np.meshgrid(g, g, indexing="ij")
    h = sum(0.25 * np.sin(a[k] * x + b[k] * z + phi[k]) for k in range(8))
    vertices = np.stack([x, h, z], axis=-1).reshape(-1, 3).astype(F32)
    i, j = np.meshgrid(np.arange(cells), np.arange(cells), indexing="ij")
    v00 = (i * (cells + 1) + j).reshape(-1)
    v01, v10, v11 = v00 + 1, v00 + cells + 1, v00 + cells + 2
    indices = np.stack([v00, v01, v11, v00, v11, v10], axis=1).reshape(-1).astype(np.uint32)
    return vertices, indices


def terrain(cells=256, cell=0.5, cols=32, levels=32, pitch=2.0, top=60.0, seed=0, flat_hulls=False, spin=0.0,
            cylinders=False):
    """Bodies dropped on a static terrain mesh (terrain_mesh): cols x cols columns at `pitch` m, `levels`
    levels from y = 2 to `top`, positions jittered by U[-0.1, 0.1], cycling through a sphere of radius
    U[0.25, 0.75], a box of half extents U[0.2, 0.8] and a hull of 16 points uniform on a 0.5 m sphere (at most
    16 vertices); density U[0.5, 2], uniformly random rotations, default sleeping. With `flat_hulls` the hulls
    are 12 points in a plane instead, thickened to slabs a few millimetres thin; with `spin` the terrain is a
    kinematic body turning about y at that many rad/s."""
    rng = np.random.default_rng([seed, 2, 2])
    n = cols * cols * levels
    b, s = _bodies(n + 1), _shapes(n + 1)
    w = World(b, s, np.arange(n + 1), meta={"kind": "terrain"})
    w.meshes.append(terrain_mesh(cells, cell, seed))
    b["type"][0] = abi.TF_STATIC
    s["geometry"][0] = abi.TF_MESH
    s["mesh"][0] = 0
    s["friction"][0] = 0.6
    idx = np.arange(n)
    level, col = idx // (cols * cols), idx % (cols * cols)
    cx, cz = col % cols, col // cols
    y = 2.0 + (top - 2.0) / max(levels - 1, 1) * level
    pos = np.stack([(cx - (cols - 1) / 2.0) * pitch, y, (cz - (cols - 1) / 2.0) * pitch], axis=1)
    b["position"][1:] = (pos + rng.uniform(-0.1, 0.1, size=(n, 3))).astype(F32)
    b["rotation"][1:] = _uniform_quats(rng, n)
    s["density"][1:] = rng.uniform(0.5, 2.0, size=n).astype(F32)
    for k in range(n):
        i = k + 1
        kind = k % 3
        if kind == 0:
            s["geometry"][i] = abi.TF_SPHERE
            s["radius"][i] = rng.uniform(0.25, 0.75)
        elif kind == 1:
            s["half_extents"][i] = rng.uniform(0.2, 0.8, size=3).astype(F32)
        else:
            s["geometry"][i] = abi.TF_HULL
            s["max_vertices"][i] = 16
            _set_points(w, i, _sphere_points(rng, 16, 0.5))
    if flat_hulls:
        flat = np.random.default_rng([seed, 2, 3])
        for i in range(1, n + 1):
            if s["geometry"][i] == abi.TF_HULL:
                pts = flat.uniform(-0.5, 0.5, size=(12, 3)).astype(F32)
                pts[:, 1] = 0.0
                _set_points(w, i, pts)
    if cylinders:
        # Every fourth body a cylinder of radius U[0.15, 0.6] and half height U[0.05, 0.6].
        cyl = np.random.default_rng([seed, 2, 4])
        for i in range(4, n + 1, 4):
            s["geometry"][i] = abi.TF_CYLINDER
            s["radius"][i] = cyl.uniform(0.15, 0.6)
            s["half_height"][i] = cyl.uniform(0.05, 0.6)
    if spin:
        b["type"][0] = abi.TF_KINEMATIC
        b["angular_velocity"][0] = (0.0, spin, 0.0)
    return w


def config2():
    """Terrain: 32,768 spheres, boxes and hulls dropped on a 256 x 256 cell terrain mesh, 600 steps."""
    return Scene("terrain_32768", [terrain()], steps=600)


def cylinders(n=24, seed=0):
    """Cylinders of every proportion (discs, rods, squat drums; radius U[0.08, 0.5], half height U[0.03, 0.6])
    with boxes, spheres and hulls, randomly turned, dropped in a loose column onto a half-space: cylinder
    against cylinder, box, hull, sphere and half-space."""
    rng = np.random.default_rng([seed, 9])
    b, s = _bodies(n + 1), _shapes(n + 1)
    _ground(b, s, friction=0.6)
    w = World(b, s, np.arange(n + 1), meta={"kind": "cylinders"})
    b["rotation"][1:] = _uniform_quats(rng, n)
    for i in range(1, n + 1):
        b["position"][i] = (rng.uniform(-1.2, 1.2), 0.8 + 0.8 * i, rng.uniform(-1.2, 1.2))
        b["angular_velocity"][i] = rng.uniform(-2.0, 2.0, size=3)
        s["friction"][i] = _f(rng.uniform(0.3, 0.9))
        kind = i % 5
        if kind in (0, 1, 2):
            s["geometry"][i] = abi.TF_CYLINDER
            s["radius"][i] = rng.uniform(0.08, 0.5)
            s["half_height"][i] = rng.uniform(0.03, 0.6)
        elif kind == 3:
            s["half_extents"][i] = rng.uniform(0.15, 0.45, size=3).astype(F32)
        elif i % 2:
            s["geometry"][i] = abi.TF_SPHERE
            s["radius"][i] = rng.uniform(0.15, 0.4)
        else:
            s["geometry"][i] = abi.TF_HULL
            s["max_vertices"][i] = 16
            _set_points(w, i, _sphere_points(rng, 16, 0.4))
    return w


def config3():
    """Planar pile: 16,384 bodies locked to the z = 0 plane in a static box container, with 256 free spheres
    dropped among them, 600 steps."""
    return Scene("planar_16384", [planar()], steps=600)


def jointed(seed=0):
    """Every joint kind in one world over a half-space, each with its limits, motor, spring or friction: a
    swinging chain of point joints from the world, a limited door with hinge friction, a hinge motor driving a
    paddle off a kinematic body that moves, a limited slider with a motor and a tilted one with friction, a
    spring, a rod and a rope with distance limits (one end on a body with locked rotation), a fixed pair that
    falls and comes to rest (its two boxes touch but do not collide), a swing-twist chain with cone and twist
    limits, two joints that break under load, and loose boxes dropped onto the chain and the door. Seeded
    jitter moves every body and anchor."""
    rng = np.random.default_rng(seed)
    b, s, joints = [], [], []

    def body(pos, half=(0.2, 0.2, 0.2), type=abi.TF_DYNAMIC, vel=(0, 0, 0), spin=(0, 0, 0), density=1.0, locks=0,
             rot=None, geometry=abi.TF_BOX, radius=0.25):
        bd = _bodies(1)
        bd["type"][0] = type
        bd["position"][0] = np.asarray(pos, np.float32) + rng.uniform(-0.02, 0.02, 3).astype(np.float32)
        if rot is not None:
            bd["rotation"][0] = rot
        bd["linear_velocity"][0] = vel
        bd["angular_velocity"][0] = spin
        bd["locks"][0] = locks
        sd = _shapes(1)
        sd["geometry"][0] = geometry
        sd["half_extents"][0] = half
        sd["radius"][0] = radius
        sd["density"][0] = density
        sd["friction"][0] = 0.5
        b.append(bd)
        s.append(sd)
        return len(b) - 1

    def joint(type, bb, ba=None, **kw):
        kw = dict(kw)
        for k in ("anchor", "anchor_b"):
            if k in kw:
                kw[k] = tuple(np.asarray(kw[k], np.float32) + rng.uniform(-0.01, 0.01, 3).astype(np.float32))
        joints.append((type, ba, bb, kw))

    ground = body((0, 0, 0), type=abi.TF_STATIC)
    # A chain of point joints, held out sideways from a world anchor so that it swings.
    prev = None
    for i in range(6):
        k = body((-6.0 + 0.45 * (i + 1), 6.0, 0.0), half=(0.2, 0.1, 0.1))
        joint(abi.TF_JOINT_POINT, k, prev, anchor=(-6.0 + 0.45 * i + 0.225, 6.0, 0.0))
        prev = k
    # A door on a limited hinge about y with friction, pushed open.
    door = body((-2.0, 1.2, 0.55), half=(0.05, 1.0, 0.5), spin=(0, 3.0, 0))
    joint(abi.TF_JOINT_HINGE, door, anchor=(-2.0, 1.2, 0.05), axis=(0, 1, 0), limited=1, lower=-0.8, upper=0.6,
          friction=0.5)
    # A paddle driven by a hinge motor off a kinematic body that moves along z.
    hub = body((1.0, 2.0, 0.0), half=(0.1, 0.1, 0.1), type=abi.TF_KINEMATIC, vel=(0, 0, 0.5))
    paddle = body((1.0, 2.0, 0.6), half=(0.05, 0.05, 0.5))
    joint(abi.TF_JOINT_HINGE, paddle, hub, anchor=(1.0, 2.0, 0.0), axis=(1, 0, 0), motor_speed=2.0, max_motor=30.0)
    # Sliders: limited with a motor, and tilted with friction.
    sl = body((3.0, 1.5, 0.0), half=(0.25, 0.15, 0.15))
    joint(abi.TF_JOINT_SLIDER, sl, anchor=(3.0, 1.5, 0.0), axis=(1, 0, 0), limited=1, lower=-0.5, upper=0.7,
          motor_speed=1.0, max_motor=20.0)
    tilt = body((5.0, 2.0, 0.0), half=(0.2, 0.2, 0.2))
    joint(abi.TF_JOINT_SLIDER, tilt, anchor=(5.0, 2.0, 0.0), axis=(0.6, -0.8, 0.0), friction=1.5)
    # Distance joints: a spring from the world, a rod between two boxes, a rope with limits to a body whose
    # rotation is locked.
    spring = body((7.0, 3.0, 0.0))
    joint(abi.TF_JOINT_DISTANCE, spring, anchor=(7.0, 4.5, 0.0), anchor_b=(7.0, 3.2, 0.0), hertz=2.0,
          damping_ratio=0.3)
    r1 = body((9.0, 3.0, 0.0), vel=(0, 0, 1.0))
    r2 = body((9.8, 3.0, 0.0))
    joint(abi.TF_JOINT_DISTANCE, r2, r1, anchor=(9.0, 3.0, 0.0), anchor_b=(9.8, 3.0, 0.0))
    rope = body((11.0, 2.5, 0.0), locks=(1 << 3) | (1 << 4) | (1 << 5))
    joint(abi.TF_JOINT_DISTANCE, rope, anchor=(11.0, 4.0, 0.0), anchor_b=(11.0, 2.7, 0.0), limited=1, lower=0.5,
          upper=1.6, length=1.0)
    # A fixed pair, touching but not colliding, falling to rest.
    f1 = body((13.0, 1.0, 0.0), half=(0.3, 0.3, 0.3))
    f2 = body((13.55, 1.1, 0.0), half=(0.25, 0.25, 0.25), spin=(0, 0, 1.0))
    joint(abi.TF_JOINT_FIXED, f2, f1, anchor=(13.3, 1.05, 0.0))
    # A swing-twist chain with cone and twist limits and friction.
    prev = None
    for i in range(3):
        k = body((15.0, 5.0 - 0.6 * (i + 1), 0.0), half=(0.1, 0.25, 0.1), spin=(1.0, 0.5, 2.0))
        joint(abi.TF_JOINT_SWING_TWIST, k, prev, anchor=(15.0, 5.0 - 0.6 * i - 0.3, 0.0), axis=(0, -1, 0),
              normal=(1, 0, 0), swing_y=0.5, swing_z=0.3, lower=-0.3, upper=0.3, friction=0.05)
        prev = k
    # Joints that break under load: a point joint with a small force limit, a fixed joint with a torque limit.
    heavy = body((17.0, 3.0, 0.0), density=8.0)
    joint(abi.TF_JOINT_POINT, heavy, anchor=(17.0, 3.2, 0.0), break_force=4.9)
    lever = body((18.5, 3.0, 0.0), half=(0.6, 0.1, 0.1))
    joint(abi.TF_JOINT_FIXED, lever, anchor=(18.0, 3.0, 0.0), break_torque=0.2)
    # Loose boxes dropped onto the chain and onto the door.
    for x, y in ((-4.8, 8.0), (-2.3, 3.5), (-5.2, 9.5)):
        body((x, y, 0.0), half=(0.15, 0.15, 0.15))
    bodies, shapes = _bodies(len(b)), _shapes(len(s))
    for i in range(len(b)):
        bodies[i] = b[i][0]
        shapes[i] = s[i][0]
    _ground(bodies, shapes)
    w = World(bodies, shapes, np.arange(len(bodies)))
    for type, ba, bb, kw in joints:
        w.joints.append(abi.joint_desc(type, abi.tf_id(bb, 0), None if ba is None else abi.tf_id(ba, 0), **kw))
    return w


def single(kind="box_on_ground", **kw):
    """Small hand-checkable worlds used by the unit parity tests."""
    if kind == "box_on_ground":
        b, s = _bodies(2), _shapes(2)
        _ground(b, s)
        b["position"][1] = kw.get("position", (0.0, 2.0, 0.0))
        b["rotation"][1] = kw.get("rotation", (0, 0, 0, 1))
        s["friction"][1] = 0.6
        return World(b, s, np.arange(2))
    if kind == "sphere_on_ground":
        b, s = _bodies(2), _shapes(2)
        _ground(b, s)
        b["position"][1] = kw.get("position", (0.0, 2.0, 0.0))
        s["geometry"][1] = abi.TF_SPHERE
        s["radius"][1] = kw.get("radius", 0.5)
        s["restitution"][1] = kw.get("restitution", 0.0)
        return World(b, s, np.arange(2))
    if kind == "boxes":
        # n randomly turned boxes dropped in a column onto a static box floor.
        n = kw.get("n", 8)
        rng = np.random.default_rng(kw.get("seed", 0))
        b, s = _bodies(n + 1), _shapes(n + 1)
        b["type"][0] = abi.TF_STATIC
        b["position"][0] = (0.0, -0.5, 0.0)
        s["half_extents"][0] = (10.0, 0.5, 10.0)
        for i in range(1, n + 1):
            b["position"][i] = (rng.uniform(-0.3, 0.3), 0.6 + 1.2 * i, rng.uniform(-0.3, 0.3))
        b["rotation"][1:] = _uniform_quats(rng, n)
        s["half_extents"][1:] = rng.uniform(0.2, 0.5, size=(n, 3)).astype(F32)
        s["friction"] = 0.6
        return World(b, s, np.arange(n + 1))
    raise ValueError(kind)
