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
