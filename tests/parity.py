"""Comparison helpers shared by the parity tests: the B200 library against the oracle."""
import numpy as np


def rel_err(a, b):
    """Normwise relative error max|a - b| / max|b| (1e-6 floor), the measure the 1e-5 bound applies to."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if a.size == 0:
        return 0.0
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-6))


def state_errors(mine, ref):
    return {k: rel_err(mine[k], ref[k]) for k in ("p", "q", "v", "w")}


def states_bitwise_equal(mine, ref):
    return all(np.array_equal(mine[k].view(np.uint32), ref[k].view(np.uint32)) for k in ("p", "q", "v", "w"))


def contact_table(contacts):
    """Exact fields (key, part, point count, feature) and the float fields of a contact list."""
    exact = [(c.key, c.part, c.point_count, c.feature_kind, c.feature_a, c.feature_b) for c in contacts]
    pts = []
    for c in contacts:
        for i in range(c.point_count):
            pts.append(list(c.points[i]) + [c.separations[i], c.normal_impulses[i]] + list(c.tangent_impulses[i]))
    return exact, np.array(pts, np.float32).reshape(-1, 8)


def first_difference(xs, ys):
    for i, (x, y) in enumerate(zip(xs, ys)):
        if x != y:
            return i, x, y
    if len(xs) != len(ys):
        return min(len(xs), len(ys)), None, None
    return None
