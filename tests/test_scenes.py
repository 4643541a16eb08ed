"""The seeded synthetic scenes: sizes the benchmark configurations name, and reproducibility."""
import numpy as np

from twofold_b200 import abi, scenes


def test_pyramid_has_210_boxes_on_a_half_space():
    sc = scenes.config1()
    w = sc.worlds[0]
    assert w.dynamic_count == 210
    assert w.shapes["geometry"][0] == abi.TF_HALFSPACE
    assert sc.steps == 300
    assert not w.bodies["can_sleep"][1:].any()


def test_uneven_worlds_are_log_uniform_between_8_and_512():
    sc = scenes.config4(n_worlds=512)
    counts = np.array([w.dynamic_count for w in sc.worlds])
    assert counts.min() >= 8 and counts.max() <= 512
    # log-uniform on [8, 513): the median is near sqrt(8 * 513) ~ 64
    assert 40 <= np.median(counts) <= 100
    kinds = {w.meta["kind"] for w in sc.worlds}
    assert kinds == {"stack", "scatter"}


def test_impact_worlds_have_64_boxes_and_a_sphere():
    sc = scenes.config5(n_worlds=4)
    for w in sc.worlds:
        assert w.dynamic_count == 65
        assert w.shapes["geometry"][-1] == abi.TF_SPHERE


def test_scenes_are_reproducible():
    a, b = scenes.config4(n_worlds=8), scenes.config4(n_worlds=8)
    for x, y in zip(a.worlds, b.worlds):
        assert np.array_equal(x.bodies, y.bodies) and np.array_equal(x.shapes, y.shapes)
