"""tf_candidates_noalloc, the candidate-pair entry point that allocates no device memory, against the step's
own broadphase as tf_world_candidates reports it, on the same world of single-shape bodies.

The inputs the entry point takes (shape bounds, growth, flags) are rebuilt here in float32 with the step's
operation order: a sphere's bounds are its center -/+ its radius, and a body's growth is the speculative
distance plus (|v| + |w| * extent) * dt for a moving body (src/world.cpp:754-765). Keys are integers, so
the comparison is exact. Every call is made twice in a row, to show that the fixed scratch starts clean.
"""
import ctypes as C

import numpy as np
import pytest

from twofold_b200 import abi, scenes
from twofold_b200.world import Batch

F32 = np.float32
DT = F32(1.0 / 60.0)


def _sphere_world(n, span, seed):
    rng = np.random.default_rng(seed)
    b, s = scenes._bodies(n), scenes._shapes(n)
    b["position"] = rng.uniform(-span, span, size=(n, 3)).astype(F32)
    b["linear_velocity"] = rng.uniform(-3.0, 3.0, size=(n, 3)).astype(F32)
    b["angular_velocity"] = rng.uniform(-4.0, 4.0, size=(n, 3)).astype(F32)
    b["linear_velocity"][::3] = 0.0
    b["angular_velocity"][::2] = 0.0
    b["type"][::7] = abi.TF_STATIC
    b["linear_velocity"][::7] = 0.0
    b["angular_velocity"][::7] = 0.0
    s["geometry"] = abi.TF_SPHERE
    s["radius"] = rng.uniform(0.2, 0.6, size=n).astype(F32)
    return scenes.World(b, s, np.arange(n))


def _length(v):
    return np.sqrt(((v[:, 0] * v[:, 0]) + (v[:, 1] * v[:, 1])) + (v[:, 2] * v[:, 2])).astype(F32)


def _pair_inputs(world, settings):
    b, s = world.bodies, world.shapes
    p = b["position"].astype(F32)
    r = s["radius"].astype(F32)[:, None]
    lo, hi = (p - r).astype(F32), (p + r).astype(F32)
    spec = F32(4.0) * (F32(0.005) * F32(settings.length_unit))
    dynamic = b["type"] == abi.TF_DYNAMIC
    v, w = b["linear_velocity"].astype(F32), b["angular_velocity"].astype(F32)
    still = ((v * v).sum(1) == 0) & ((w * w).sum(1) == 0)
    travel = ((_length(v) + _length(w) * s["radius"].astype(F32)) * DT).astype(F32)
    grow = np.where(dynamic & ~still, spec + travel, spec).astype(F32)
    flags = (abi.TF_PAIR_LIVE | np.where(dynamic, abi.TF_PAIR_DYNAMIC | abi.TF_PAIR_MOVING, 0)).astype(np.uint32)
    return lo, hi, grow, flags


def _noalloc(lib, torch, lo, hi, grow, flags, capacity):
    dev = torch.device("cuda:0")
    t_lo = torch.from_numpy(lo.reshape(-1)).to(dev)
    t_hi = torch.from_numpy(hi.reshape(-1)).to(dev)
    t_grow = torch.from_numpy(grow).to(dev)
    t_flags = torch.from_numpy(flags.view(np.int32)).to(dev)
    keys = torch.full((capacity,), -1, dtype=torch.int64, device=dev)
    count = torch.full((1,), -7, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.tf_candidates_noalloc(t_lo.data_ptr(), t_hi.data_ptr(), t_grow.data_ptr(), t_flags.data_ptr(), len(grow),
                                   keys.data_ptr(), capacity, count.data_ptr(), C.c_void_p(stream))
    abi.check(rc, lib)
    torch.cuda.synchronize()
    n = int(count.item())
    return n, keys.cpu().numpy().view(np.uint64)[:max(n, 0)]


@pytest.mark.gpu
@pytest.mark.parametrize("n,span,seed", [(300, 3.0, 0), (1500, 7.0, 1), (4096, 12.0, 2)])
def test_noalloc_candidates_match_the_step(n, span, seed):
    torch = pytest.importorskip("torch")
    world = _sphere_world(n, span, seed)
    sc = scenes.Scene("spheres", [world])
    batch = Batch.from_scene(sc)
    batch.step_checked(float(DT))
    expected = batch.candidates(0)
    assert len(expected) > 0
    lo, hi, grow, flags = _pair_inputs(world, sc.settings)
    for call in range(2):
        got_n, got = _noalloc(batch.lib, torch, lo, hi, grow, flags, capacity=len(expected) + 16)
        assert got_n == len(expected), f"call {call}: {got_n} pairs, the step found {len(expected)}"
        assert np.array_equal(got, expected), f"call {call}: pair keys differ"


@pytest.mark.gpu
def test_noalloc_reports_short_capacity():
    torch = pytest.importorskip("torch")
    world = _sphere_world(300, 3.0, 0)
    lo, hi, grow, flags = _pair_inputs(world, abi.default_settings())
    full_n, full = _noalloc(abi.load(), torch, lo, hi, grow, flags, capacity=20000)
    assert full_n > 8
    for call in range(2):
        n, _ = _noalloc(abi.load(), torch, lo, hi, grow, flags, capacity=8)
        assert n == full_n


def test_noalloc_refuses_more_bodies_than_its_scratch():
    lib = abi.load()
    n = abi.TF_NOALLOC_MAX_BODIES + 1
    cnt = C.c_int32(0)
    rc = lib.tf_candidates_noalloc(None, None, None, None, n, None, 0, C.byref(cnt), None)
    assert rc == abi.TF_E_CAPACITY
    assert b"4096" in lib.tf_last_error()


@pytest.mark.gpu
def test_noalloc_reports_too_many_raw_pairs_and_recovers():
    """300 bodies in one overlapping cluster make n(n-1)/2 = 44850 raw pair hits, more than the scratch holds:
    the count is -1 and the keys keep their fill value. A normal call afterwards gives the full answer again."""
    torch = pytest.importorskip("torch")
    lib = abi.load()
    n = 300
    assert n * (n - 1) // 2 > abi.TF_NOALLOC_MAX_PAIRS
    lo = np.zeros((n, 3), F32)
    hi = np.ones((n, 3), F32)
    grow = np.full(n, F32(0.02), F32)
    flags = np.full(n, abi.TF_PAIR_LIVE | abi.TF_PAIR_DYNAMIC | abi.TF_PAIR_MOVING, np.uint32)
    dev = torch.device("cuda:0")
    keys = torch.full((64,), -1, dtype=torch.int64, device=dev)
    count = torch.zeros((1,), dtype=torch.int32, device=dev)
    t = [torch.from_numpy(x.reshape(-1).view(np.int32) if x.dtype == np.uint32 else x.reshape(-1)).to(dev)
         for x in (lo, hi, grow, flags)]
    rc = lib.tf_candidates_noalloc(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), t[3].data_ptr(), n,
                                   keys.data_ptr(), 64, count.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    abi.check(rc, lib)
    torch.cuda.synchronize()
    assert int(count.item()) == -1
    assert bool((keys == -1).all()), "keys were written although the raw hits overflowed"
    world = _sphere_world(300, 3.0, 0)
    lo2, hi2, grow2, flags2 = _pair_inputs(world, abi.default_settings())
    full_n, full = _noalloc(lib, torch, lo2, hi2, grow2, flags2, capacity=20000)
    assert full_n > 8
    again_n, again = _noalloc(lib, torch, lo2, hi2, grow2, flags2, capacity=20000)
    assert again_n == full_n and np.array_equal(again, full)
