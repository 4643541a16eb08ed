"""The adjoint of the substepped solve, through the C ABI and a thin torch.autograd.Function (the only torch
wrapper; it lives here, in the test harness).

Scene: the differentiable impact (a 4x4x4 wall of boxes hit by a sphere) for a few worlds and enough steps
for the sphere to reach the wall. Loss: the sum of the boxes' squared final x. Gradients with respect to the
sphere's initial velocity, a world's friction and box masses are checked against central finite
differences of the double-precision model, within 1e-3 relative.

The model is piecewise smooth: contacts switch on and off and friction moves between stick and slip, and a
step of h = 1e-3 in a velocity often crosses such an event, where the difference quotient measures the jump
and not the slope (one sphere velocity here gives 0.143 at h = 1e-3 against 0.0154 for h <= 1e-5). Each
check therefore starts at h = 1e-3 and takes the first step size whose quotient agrees with the next
smaller one's (a converged estimate); the adjoint must match that estimate. The float instantiation of the
same kernels must agree with the double one.
"""
import numpy as np
import pytest

from twofold_b200 import scenes
from twofold_b200.world import Batch

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

STEPS = 30
TOL = 1e-3


class RecordedRun(torch.autograd.Function):
    """The recorded run as a function of (initial state, masses, frictions) -> final state (bodies x 13)."""

    @staticmethod
    def forward(ctx, batch, n_shapes, precision, initial, mass, friction):
        out = batch.adjoint_forward(precision, initial.detach().numpy(), mass.detach().numpy(),
                                    friction.detach().numpy())
        ctx.batch, ctx.n_shapes = batch, n_shapes
        return torch.from_numpy(out)

    @staticmethod
    def backward(ctx, grad):
        gi, gm, gf = ctx.batch.adjoint_backward(grad.contiguous().numpy(), ctx.n_shapes)
        return None, None, None, torch.from_numpy(gi), torch.from_numpy(gm), torch.from_numpy(gf)


def _setup(n_worlds=3, seed=0):
    sc = scenes.config5(n_worlds=n_worlds, seed=seed)
    b = Batch.from_scene(sc)
    s = b.states()
    initial = np.concatenate([s["p"], s["q"], s["v"], s["w"]], axis=1).astype(np.float64)
    mass = np.array([b.mass(wi, i)[0] for wi, w in enumerate(sc.worlds) for i in range(len(w.bodies))], np.float64)
    mass[mass == 0] = 1.0
    friction = np.concatenate([w.shapes["friction"] for w in sc.worlds]).astype(np.float64)
    b.tape_record(sc.dt, STEPS)
    boxes = np.zeros(len(initial), bool)
    for wi, w in enumerate(sc.worlds):
        boxes[b.offsets[wi] + 1:b.offsets[wi] + 65] = True
    return sc, b, initial, mass, friction, boxes


def _loss(final, boxes):
    return (final[boxes, 0] ** 2).sum()


def _grads(b, n_shapes, precision, initial, mass, friction, boxes):
    ti = torch.tensor(initial, requires_grad=True)
    tm = torch.tensor(mass, requires_grad=True)
    tf = torch.tensor(friction, requires_grad=True)
    final = RecordedRun.apply(b, n_shapes, precision, ti, tm, tf)
    loss = (final[torch.from_numpy(boxes), 0] ** 2).sum()
    loss.backward()
    return float(loss.detach()), ti.grad.numpy(), tm.grad.numpy(), tf.grad.numpy()


STEPS_H = (1e-3, 1e-4, 1e-5, 1e-6, 1e-7)


def _fd(b, boxes, initial, mass, friction, which, index):
    """Central difference at the largest step (from 1e-3 down) that agrees with the next smaller step."""
    def at(delta):
        i, m, f = initial.copy(), mass.copy(), friction.copy()
        if which == "initial":
            i[index] += delta
        elif which == "mass":
            m[index] += delta
        else:
            f[index] += delta
        return _loss(b.adjoint_forward(64, i, m, f), boxes)

    q = [(at(h) - at(-h)) / (2 * h) for h in STEPS_H]
    for k in range(len(q) - 1):
        if abs(q[k] - q[k + 1]) <= TOL * max(abs(q[k + 1]), 1e-6):
            return q[k]
    return q[-1]


def test_adjoint_matches_finite_differences():
    sc, b, initial, mass, friction, boxes = _setup()
    n_shapes = len(friction)
    loss, gi, gm, gf = _grads(b, n_shapes, 64, initial, mass, friction, boxes)
    assert loss > 0
    sphere = int(b.offsets[0]) + 65
    checks = [("initial", (sphere, 7), gi[sphere, 7]), ("initial", (sphere, 8), gi[sphere, 8]),
              ("mass", 5, gm[5]), ("mass", 40, gm[40])]
    # A world's friction: every shape of world 0 moves together.
    w0 = slice(0, len(sc.worlds[0].shapes))
    f_idx = np.zeros(n_shapes, bool)
    f_idx[w0] = True
    for which, index, g in checks:
        fd = _fd(b, boxes, initial, mass, friction, which, index)
        assert abs(g - fd) <= TOL * max(abs(fd), 1e-6) + 1e-9, f"{which} {index}: adjoint {g} vs difference {fd}"
    fd = _fd(b, boxes, initial, mass, friction, "friction", f_idx)
    g = gf[w0].sum()
    assert abs(g - fd) <= TOL * max(abs(fd), 1e-6) + 1e-9, f"friction of world 0: adjoint {g} vs difference {fd}"


def test_float_adjoint_agrees_with_double():
    sc, b, initial, mass, friction, boxes = _setup(n_worlds=2, seed=1)
    n_shapes = len(friction)
    l64, gi64, gm64, gf64 = _grads(b, n_shapes, 64, initial, mass, friction, boxes)
    l32, gi32, gm32, gf32 = _grads(b, n_shapes, 32, initial, mass, friction, boxes)
    assert abs(l32 - l64) <= 1e-4 * abs(l64)
    # Normwise (2-norm) relative difference: a float run may take the other side of a contact event that the
    # double run only just reaches, which moves single entries more than the gradient as a whole.
    for a32, a64 in ((gi32[:, 7:10], gi64[:, 7:10]), (gm32, gm64), (gf32, gf64)):
        err = np.linalg.norm(a32 - a64) / max(np.linalg.norm(a64), 1e-12)
        assert err <= 1e-2, err


def test_model_forward_tracks_the_pipeline():
    """With contacts held fixed per step the model is not the pipeline, but over a short run it stays close."""
    sc, b, initial, mass, friction, boxes = _setup(n_worlds=2, seed=2)
    final = b.adjoint_forward(64, initial, mass, friction)
    s = b.states()
    assert np.max(np.abs(final[boxes, :3] - s["p"][boxes])) < 0.05
