"""The adjoint of the substepped solve, through the C ABI and a thin torch.autograd.Function (the only torch
wrapper; it lives here, in the test harness).

Scene: the differentiable impact (a 4x4x4 wall of boxes hit by a sphere) for a few worlds and enough steps
for the sphere to reach the wall. Loss: the sum of the boxes' squared final x. Gradients with respect to the
sphere's initial velocity, a world's friction and box masses are checked against central finite
differences of the double-precision model, within 1e-3 relative.

The model is piecewise smooth: contacts switch on and off and friction moves between stick and slip, and a
step of h = 1e-3 in a velocity often crosses such an event, where the difference quotient measures the jump
and not the slope (one sphere velocity here gives 0.143 at h = 1e-3 against 0.0154 for h <= 1e-5). Two checks
follow from that. On 64 worlds over 120 steps, central differences at h = 1e-3 are compared with the adjoint
for the entries whose +h and -h runs take every branch the unperturbed run takes (the forward's branch
signature, tf_adjoint_branches), which is asserted, not assumed. On a few worlds over 30 steps, each check
starts at h = 1e-3 and takes the first step size whose quotient agrees with the next smaller one's (a
converged estimate), so entries whose runs do cross an event are covered too. The float instantiation of
the same kernels must agree with the double one, and one step of the model must stay close to the step of
the pipeline it was recorded from wherever the pipeline did not collide again mid-step.
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


def test_adjoint_matches_differences_on_64_worlds_for_120_steps():
    """64 impact worlds, 120 steps, double precision. For each checked entry (a sphere's initial velocity, box
    masses, a world's friction) the central difference starts at h = 1e-3; where its +h and -h runs keep every
    branch of the unperturbed run (tf_adjoint_branches) that quotient is compared directly, and otherwise the
    quotient at the first step size from 1e-3 down that agrees with the one before it within 1e-4 (a converged
    estimate, an order closer than the tolerance). The adjoint matches within 1e-3 every entry whose quotients
    converge, and at least three quarters of the entries converge."""
    n_worlds, steps = 64, 120
    sc = scenes.config5(n_worlds=n_worlds, seed=3)
    b = Batch.from_scene(sc)
    s = b.states()
    initial = np.concatenate([s["p"], s["q"], s["v"], s["w"]], axis=1).astype(np.float64)
    mass = np.array([b.mass(wi, i)[0] for wi, w in enumerate(sc.worlds) for i in range(len(w.bodies))], np.float64)
    mass[mass == 0] = 1.0
    friction = np.concatenate([w.shapes["friction"] for w in sc.worlds]).astype(np.float64)
    b.tape_record(sc.dt, steps)
    boxes = np.zeros(len(initial), bool)
    for wi in range(n_worlds):
        boxes[b.offsets[wi] + 1:b.offsets[wi] + 65] = True
    n_shapes = len(friction)
    loss, gi, gm, gf = _grads(b, n_shapes, 64, initial, mass, friction, boxes)
    assert loss > 0
    b.adjoint_forward(64, initial, mass, friction)
    base_sig = b.adjoint_branches()
    shape_first = np.concatenate([[0], np.cumsum([len(w.shapes) for w in sc.worlds])])
    entries = []
    for wi in range(0, n_worlds, 8):
        sphere = int(b.offsets[wi]) + 65
        for k in (7, 8, 9):
            entries.append((wi, "initial", (sphere, k), gi[sphere, k]))
        for box in (1, 64):
            entries.append((wi, "mass", int(b.offsets[wi]) + box, gm[int(b.offsets[wi]) + box]))
        f_idx = np.zeros(n_shapes, bool)
        f_idx[shape_first[wi]:shape_first[wi + 1]] = True
        entries.append((wi, "friction", f_idx, gf[f_idx].sum()))

    def run(which, index, delta):
        i, m, f = initial.copy(), mass.copy(), friction.copy()
        if which == "initial":
            i[index] += delta
        elif which == "mass":
            m[index] += delta
        else:
            f[index] += delta
        return _loss(b.adjoint_forward(64, i, m, f), boxes), b.adjoint_branches()

    kept, converged, report = 0, 0, []
    for wi, which, index, g in entries:
        q = []
        for h in STEPS_H:
            lp, sp = run(which, index, h)
            lm, sm = run(which, index, -h)
            # Worlds are independent: the others see nothing of the change.
            others = np.arange(n_worlds) != wi
            assert np.array_equal(sp[others], base_sig[others]) and np.array_equal(sm[others], base_sig[others])
            q.append((lp - lm) / (2 * h))
            if h == STEPS_H[0] and sp[wi] == base_sig[wi] and sm[wi] == base_sig[wi]:
                kept += 1
                break
        fd = None
        if len(q) == 1:
            fd = q[0]
        else:
            # Converged: two successive quotients agree ten times closer than the tolerance they are held to.
            for k in range(len(q) - 1):
                if abs(q[k] - q[k + 1]) <= 0.1 * TOL * max(abs(q[k + 1]), 1e-6):
                    fd = q[k + 1]
                    break
        report.append((wi, which, float(g), None if fd is None else float(fd)))
        if fd is None:
            continue
        converged += 1
        assert abs(g - fd) <= TOL * max(abs(fd), 1e-6) + 1e-9, f"world {wi} {which} {index}: adjoint {g} vs difference {fd}"
    print(f"{kept} of {len(entries)} entries kept every branch at h = 1e-3; {converged} converged")
    assert converged >= 3 * len(entries) // 4, report


def test_model_step_stays_close_to_the_pipeline_step():
    """Each of 40 steps recorded on its own: where the pipeline did not collide any contact again mid-step,
    the model's step (double precision) from the recorded start ends within a millimetre and 1 cm/s of the
    pipeline's."""
    sc = scenes.config5(n_worlds=4, seed=2)
    b = Batch.from_scene(sc)
    compared, worst_p, worst_v = 0, 0.0, 0.0
    for step in range(40):
        b.tape_record(sc.dt, 1)
        model = b.adjoint_forward(64)
        s = b.states()
        for wi in range(len(sc.worlds)):
            if b.solver_counts(wi)["fast"] > 0:
                continue
            lo, hi = int(b.offsets[wi]), int(b.offsets[wi + 1])
            dp = np.max(np.abs(model[lo:hi, :3] - s["p"][lo:hi]))
            dv = np.max(np.abs(model[lo:hi, 7:10] - s["v"][lo:hi]))
            worst_p, worst_v = max(worst_p, dp), max(worst_v, dv)
            compared += 1
    assert compared >= 40, compared
    assert worst_p <= 1e-3 and worst_v <= 1e-2, (worst_p, worst_v)


def test_reverse_walk_layouts_give_the_same_gradients():
    """The reverse walk keeps each world's body arrays in shared memory when the largest world's fit there, and in
    global memory when one world is too large (a 325-box pyramid beside the impact walls): the impact worlds'
    gradients are the same bits either way, in float and in double."""
    impact = list(scenes.config5(n_worlds=4, seed=4).worlds)
    alone = Batch.from_scene(scenes.Scene("impact", impact))
    mixed = Batch.from_scene(scenes.Scene("impact and pyramid", impact + [scenes.pyramid(25)]))
    n = int(alone.offsets[-1])
    shapes = sum(len(w.shapes) for w in impact)
    for b in (alone, mixed):
        b.tape_record(1.0 / 60.0, 12)
    for precision in (32, 64):
        runs = []
        for b, n_shapes in ((alone, shapes), (mixed, shapes + 326)):
            final = b.adjoint_forward(precision)
            grad = np.zeros_like(final)
            grad[:n, 0] = 2 * final[:n, 0]
            gi, gm, gf = b.adjoint_backward(grad, n_shapes)
            runs.append((final[:n], gi[:n], gm[:n], gf[:shapes]))
        for a, c in zip(*runs):
            assert np.array_equal(a, c)
        assert np.any(runs[0][1] != 0)
