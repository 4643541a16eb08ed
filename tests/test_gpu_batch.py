"""Batched-form behaviour that has no reference counterpart: launch shapes never change results, device
snapshots put the state back exactly, and the autotuner leaves the batch as it found it."""
import numpy as np
import pytest

from parity import states_bitwise_equal
from twofold_b200 import scenes
from twofold_b200.world import Batch

pytestmark = pytest.mark.gpu


def _scene(n=64, seed=3):
    return scenes.config4(n_worlds=n, seed=seed)


@pytest.mark.parametrize("shape", [(128, 0, 48 * 1024), (512, 256, 96 * 1024), (256, 32, 0), (64, 0, 0)])
def test_launch_shapes_do_not_change_results(shape):
    sc = _scene()
    ref = Batch.from_scene(sc)
    ref.step_checked(sc.dt, 30)
    other = Batch.from_scene(sc)
    threads, big, smem = shape
    for k in Batch.KERNELS:
        flat = k in ("refresh", "collide")
        other.set_launch(k, min(threads, 256) if flat else max(threads, 128), big, smem)
    other.step_checked(sc.dt, 30)
    assert states_bitwise_equal(ref.states(), other.states())
    for w in range(0, sc.worlds.__len__(), 7):
        assert np.array_equal(ref.candidates(w), other.candidates(w))


def test_snapshot_restores_exactly():
    sc = _scene(48, 5)
    b = Batch.from_scene(sc)
    b.step_checked(sc.dt, 20)
    b.save_state(3)
    b.step_checked(sc.dt, 15)
    first = b.states()
    b.restore_state(3)
    b.step_checked(sc.dt, 15)
    assert states_bitwise_equal(first, b.states())
    b.restore_state(3)
    b.step_checked(sc.dt, 15, graph=True)
    assert states_bitwise_equal(first, b.states())


def test_autotune_leaves_the_state_alone():
    sc = _scene(96, 7)
    plain = Batch.from_scene(sc)
    tuned = Batch.from_scene(sc)
    plain.step_checked(sc.dt, 25)
    tuned.step_checked(sc.dt, 25)
    choice = tuned.autotune(sc.dt, trial_steps=1)
    assert set(choice) == set(Batch.KERNELS)
    assert states_bitwise_equal(plain.states(), tuned.states())
    plain.step_checked(sc.dt, 20)
    tuned.step_checked(sc.dt, 20, graph=True)
    assert states_bitwise_equal(plain.states(), tuned.states())


def _mixed_scene():
    """Uneven worlds with restitution, impact walls (impact colors), planar piles (contacts solved one at a time by
    level) and jointed worlds in one batch: every path of the flat solve."""
    worlds = list(scenes.config4(n_worlds=40, seed=11).worlds)
    worlds += list(scenes.config5(n_worlds=6).worlds)
    worlds += [scenes.planar(n=48, cols=8, spheres=4, sphere_height=(3.0, 8.0), seed=s, restitution=0.2) for s in range(3)]
    worlds += [scenes.jointed(s) for s in range(2)]
    return scenes.Scene("mixed", worlds)


@pytest.mark.parametrize("threads", [128, 256])
def test_flat_solve_matches_the_world_kernels(threads):
    """The flat solve (every world's contacts of a color at once across the device, a grid barrier between
    colors) gives the world kernels' bits: states, contacts and candidate pairs, by direct launches and by graph."""
    sc = _mixed_scene()
    worlds_kernel = Batch.from_scene(sc)
    flat = Batch.from_scene(sc)
    worlds_kernel.set_launch("substep", 128, 128, 32 * 1024)
    flat.set_launch("substep", threads, -1, 0)
    assert flat.launch("substep")["big_bodies"] == 0xFFFFFFFF
    for steps, graph in ((20, False), (20, True), (40, True)):
        worlds_kernel.step_checked(sc.dt, steps)
        flat.step_checked(sc.dt, steps, graph=graph)
        assert states_bitwise_equal(worlds_kernel.states(), flat.states())
    for w in range(len(sc.worlds)):
        assert np.array_equal(worlds_kernel.candidates(w), flat.candidates(w))
    assert flat.device_flags() == 0


def test_flat_solve_is_the_default_for_many_worlds_and_autotuned():
    sc = _scene(1024, 2)
    b = Batch.from_scene(sc)
    b.step_checked(sc.dt, 8)
    assert b.launch("substep")["big_bodies"] == 0xFFFFFFFF
    ref = Batch.from_scene(sc)
    ref.set_launch("substep", 128, 128, 32 * 1024)
    ref.step_checked(sc.dt, 8)
    choice = b.autotune(sc.dt, trial_steps=1)
    assert "substep" in choice
    b.step_checked(sc.dt, 12, graph=True)
    ref.step_checked(sc.dt, 12)
    assert states_bitwise_equal(ref.states(), b.states())


def test_queued_pose_reads_match_direct_reads():
    """tf_world_read_poses_async into two host buffers in turn, waited on every other step, gives the poses
    tf_world_read_poses gives for the same steps of an identical batch, with per-body forces added each step."""
    sc = scenes.config4(n_worlds=32)
    queued, direct = Batch.from_scene(sc), Batch.from_scene(sc)
    total = int(queued.offsets[-1])
    forces = np.zeros((total, 3), np.float32)
    forces[:, 0] = 2.0
    pq = [np.zeros((total, 3), np.float32) for _ in range(2)]
    qq = [np.zeros((total, 4), np.float32) for _ in range(2)]
    seen = []
    for k in range(8):
        queued.add_forces(forces)
        queued.step_checked(sc.dt, 1, graph=True)
        queued.read_poses_async(pq[k % 2], qq[k % 2])
        direct.add_forces(forces)
        direct.step_checked(sc.dt, 1, graph=True)
        p, q = np.zeros((total, 3), np.float32), np.zeros((total, 4), np.float32)
        direct.read_poses(p, q)
        seen.append((p, q))
        if k % 2 == 1:
            queued.poses_wait()
            for j in (k - 1, k):
                assert np.array_equal(pq[j % 2], seen[j][0]) and np.array_equal(qq[j % 2], seen[j][1]), j
    queued.poses_wait()
    assert not np.array_equal(seen[0][0], seen[-1][0])
