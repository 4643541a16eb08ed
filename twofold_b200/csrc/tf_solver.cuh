// Contact preparation, solve, restitution and integration for one contact or one body.
//
// The reference solves colored contacts four at a time in SSE/NEON lanes and the rest one at a time; both
// give the same bits (src/lanes.h:16-17, src/lanes.cpp:220-315 against src/solver.cpp:360-421). Here one
// thread solves one contact with the scalar sequence, which is therefore exact for laned and rest contacts
// alike. Contacts of one color move no body in common, so a color's contacts run in parallel with results
// identical to any sequential order.
//
// Each point's three axes (lever arms, velocity change per unit impulse, effective mass) are built where the
// reference builds them, at the step's start and after a mid-step refresh, and read by every pass between.
#pragma once

#include "tf_body.cuh"
#include "tf_collide.cuh"

namespace tfb {

// One direction at a contact point (src/internal.h:508-520, src/solver.cpp:5-17).
struct alignas(16) Axis {
    Vec3 armA, armB;
    Vec3 linearA, angularA;
    Vec3 linearB, angularB;
    float mass;
    float pad;
};

// A contact's axes are built once per step and again after a mid-step refresh, as the reference builds them
// (src/lanes.cpp:66-110, src/solver.cpp:43-50), and stored 3 per point: normal, tangent1, tangent2.
constexpr int kAxesPerContact = 12;

// The body fields an axis is built from, read once into registers before a contact's axes are written.
struct AxisBody {
    Mat3 invMassWorld, invInertiaWorld;
    float invMass;
    float planeInvMass, planeInvInertia;
};

template <class BodyT>
TF_HD AxisBody axisBodyOf(const BodyT& b) {
    return { b.invMassWorld, b.invInertiaWorld, b.invMass, b.planeInvMass, b.planeInvInertia };
}

// A planar contact's point axes (DPlanarAxes) live in the point's normal axis slot: normalA, normalB and
// normalMass in armA, tangentA, tangentB and tangentMass in armB.
TF_HD void putPlanarAxes(Axis& x, const DPlanarAxes& p) {
    x.armA = Vec3{ p.normalA, p.normalB, p.normalMass };
    x.armB = Vec3{ p.tangentA, p.tangentB, p.tangentMass };
}

TF_HD DPlanarAxes planarAxesOf(const Axis& x) {
    return { x.armA.x, x.armA.y, x.armA.z, x.armB.x, x.armB.y, x.armB.z };
}

// src/solver.cpp:83-86.
template <class BodyT>
TF_HD float planarMass(const BodyT& a, const BodyT& b, float armA, float armB) {
    const float k = a.planeInvMass + b.planeInvMass + a.planeInvInertia * armA * armA + b.planeInvInertia * armB * armB;
    return k > 1e-6f * (a.invMass + b.invMass) ? 1.0f / k : 0.0f;
}

// The planar axes of point i (src/solver.cpp:88-101).
template <class BodyT>
TF_HD DPlanarAxes makePlanarAxes(const BodyT& a, const BodyT& b, const DContact& c, int i) {
    const Vec3 n = c.plane;
    const DPoint& p = c.points[i];
    DPlanarAxes x;
    x.normalA = dot(n, cross(p.anchorA, c.normal));
    x.normalB = dot(n, cross(p.anchorB, c.normal));
    x.normalMass = planarMass(a, b, x.normalA, x.normalB);
    x.tangentA = dot(n, cross(p.anchorA, c.tangent1));
    x.tangentB = dot(n, cross(p.anchorB, c.tangent1));
    x.tangentMass = planarMass(a, b, x.tangentA, x.tangentB);
    return x;
}

// The velocities of a planar contact's bodies, with spin about the plane normal, held while its points are
// solved (src/solver.cpp:104-134).
struct PlanarState {
    Vec3 va, vb;
    float wa, wb;
    float ma, mb, ia, ib;

    template <class BodyT>
    TF_HD PlanarState(const BodyT& a, const BodyT& b, const Vec3& n)
        : va(a.v), vb(b.v), wa(dot(a.w, n)), wb(dot(b.w, n)), ma(a.planeInvMass), mb(b.planeInvMass),
          ia(a.planeInvInertia), ib(b.planeInvInertia) {}

    TF_HD float speed(const Vec3& d, float armA, float armB) const { return dot(d, vb - va) + armB * wb - armA * wa; }

    TF_HD void push(const Vec3& d, float armA, float armB, float impulse) {
        va -= d * (ma * impulse);
        wa -= ia * armA * impulse;
        vb += d * (mb * impulse);
        wb += ib * armB * impulse;
    }

    template <class BodyT>
    TF_HD void store(BodyT& a, BodyT& b, const Vec3& n, bool moveA, bool moveB) const {
        if (moveA) {
            a.v = va;
            a.w = n * wa;
        }
        if (moveB) {
            b.v = vb;
            b.w = n * wb;
        }
    }
};

template <class BodyT>
TF_HD Axis makeAxis(const BodyT& a, const BodyT& b, const Vec3& ra, const Vec3& rb, const Vec3& d) {
    Axis x;
    x.armA = cross(ra, d);
    x.armB = cross(rb, d);
    x.linearA = a.invMassWorld * d;
    x.angularA = a.invInertiaWorld * x.armA;
    x.linearB = b.invMassWorld * d;
    x.angularB = b.invInertiaWorld * x.armB;
    const float k = dot(d, x.linearA) + dot(d, x.linearB) + dot(x.armA, x.angularA) + dot(x.armB, x.angularB);
    x.mass = k > 1e-6f * (a.invMass + b.invMass) ? 1.0f / k : 0.0f;
    return x;
}

template <class BodyT>
TF_HD float speedAlong(const BodyT& a, const BodyT& b, const Vec3& d, const Axis& x) {
    return dot(d, b.v - a.v) + dot(x.armB, b.w) - dot(x.armA, a.w);
}

template <class BodyT>
TF_HD void pushMoving(BodyT& a, BodyT& b, const Axis& x, float impulse, bool moveA, bool moveB) {
    if (moveA) {
        a.v -= x.linearA * impulse;
        a.w -= x.angularA * impulse;
    }
    if (moveB) {
        b.v += x.linearB * impulse;
        b.w += x.angularB * impulse;
    }
}

// Where the body has turned r since the substep's base pose (src/solver.cpp:58-61).
template <class BodyT>
TF_HD Vec3 turned(const BodyT& b, const Vec3& r) {
    return b.dq.x == 0.0f && b.dq.y == 0.0f && b.dq.z == 0.0f ? r : rotate(b.dq, r);
}

template <class BodyT>
TF_HD bool anchored(const BodyT& b) { return b.type != kDynamic || !b.awake; }

TF_HD Softness makeSoft(float hertz, float zeta, float h) {
    if (hertz == 0.0f) { return { 0.0f, 1.0f, 0.0f }; }
    const float omega = 2.0f * 3.14159265358979f * hertz;
    const float a1 = 2.0f * zeta + h * omega;
    const float a2 = h * omega * a1;
    const float a3 = 1.0f / (1.0f + a2);
    return { omega / a1, a2 * a3, a3 };
}

// Whether every body the contact moves is a dynamic body locked to one plane n holding the normal
// (src/solver.cpp:66-81).
TF_HD bool planarContact(const DBody& a, const DBody& b, const Vec3& normal, Vec3& n) {
    const DBody* first = nullptr;
    const DBody* both[2] = { &a, &b };
    for (int k = 0; k < 2; ++k) {
        const DBody* x = both[k];
        if (x->type == kStatic) { continue; }
        if (x->type == kKinematic || !isPlanar(*x)) { return false; }
        if (!first) {
            first = x;
            n = planeNormal(*x);
        } else if (fabsf(dot(n, planeNormal(*x))) < 0.9999f) {
            return false;
        }
    }
    return first && fabsf(dot(normal, n)) < 1e-3f;
}

// Adjusted separation, approach speed and rolling radius at the step's start (src/solver.cpp:264-291). A
// planar contact's normal is laid in the plane first, with the tangent in the plane and the plane normal as
// the second tangent.
TF_HD void prepareContact(const DBody& a, const DBody& b, DContact& c) {
    Vec3 plane = c.plane;
    const bool planar = planarContact(a, b, c.normal, plane);
    c.plane = plane;
    c.flags = planar ? (c.flags | kCPlanar) : (c.flags & ~kCPlanar);
    if (planar) {
        c.normal = normalize(c.normal - c.plane * dot(c.normal, c.plane));
        c.tangent1 = cross(c.plane, c.normal);
        c.tangent2 = c.plane;
    }
    const PlanarState st(a, b, c.plane);
    for (int i = 0; i < c.count; ++i) {
        DPoint& p = c.points[i];
        p.adjustedSeparation = p.separation - dot(p.anchorB - p.anchorA, c.normal);
        if (planar) {
            const DPlanarAxes x = makePlanarAxes(a, b, c, i);
            p.relativeVelocity = st.speed(c.normal, x.normalA, x.normalB);
        } else {
            p.relativeVelocity = dot(c.normal, b.v - a.v) + dot(cross(p.anchorB, c.normal), b.w) -
                                 dot(cross(p.anchorA, c.normal), a.w);
        }
        p.maxNormalImpulse = 0.0f;
    }
    if (c.rollingResistance > 0.0f && c.count > 0) {
        float ha = 0.0f, hb = 0.0f;
        for (int i = 0; i < c.count; ++i) {
            ha += fabsf(dot(c.points[i].anchorA, c.normal));
            hb += fabsf(dot(c.points[i].anchorB, c.normal));
        }
        if (a.type != kDynamic) { ha = 0.0f; }
        if (b.type != kDynamic) { hb = 0.0f; }
        c.rollingRadius = maxf(ha, hb) / (float)c.count;
    }
}

// The axes of every point of a contact (src/solver.cpp:43-50), from the bodies' current world inverse mass
// and inertia; a planar contact's planar axes (src/solver.cpp:88-101), which the reference builds in
// prepareContact and rebaseContact from the same body state.
template <class BodyT>
TF_HD void makeContactAxes(const BodyT& a, const BodyT& b, const DContact& c, Axis* __restrict__ out) {
    if (c.flags & kCPlanar) {
        for (int i = 0; i < c.count; ++i) { putPlanarAxes(out[3 * i], makePlanarAxes(a, b, c, i)); }
        return;
    }
    for (int i = 0; i < c.count; ++i) {
        const DPoint& p = c.points[i];
        out[3 * i] = makeAxis(a, b, p.anchorA, p.anchorB, c.normal);
        out[3 * i + 1] = makeAxis(a, b, p.anchorA, p.anchorB, c.tangent1);
        out[3 * i + 2] = makeAxis(a, b, p.anchorA, p.anchorB, c.tangent2);
    }
}

// Re-expresses anchors as the bodies' current lever arms before their dp and dq are reset
// (src/solver.cpp:293-306).
TF_HD void rebaseContact(const DBody& a, const DBody& b, DContact& c) {
    const float shift = dot(b.dp - a.dp, c.normal);
    for (int i = 0; i < c.count; ++i) {
        DPoint& p = c.points[i];
        p.anchorA = rotate(a.dq, p.anchorA);
        p.anchorB = rotate(b.dq, p.anchorB);
        p.adjustedSeparation += shift;
    }
}

// Applies the stored impulses (src/solver.cpp:319-358 and src/lanes.cpp:195-217). A laned contact pushes only
// the bodies that move; a contact solved on its own pushes both, as the reference's scalar warm start does
// (the anchored body's zero inverse mass leaves it unchanged). Contacts solved on their own run one at a
// time, so the unmasked push never races.
template <class BodyT>
TF_HD void warmStartContact(BodyT& a, BodyT& b, const DContact& c, bool laned, const Axis* __restrict__ ax) {
    if (c.flags & kCPlanar) {
        // src/solver.cpp:325-344: a planar contact holding nothing leaves its bodies as they are.
        bool held = c.rollingResistance > 0.0f;
        for (int i = 0; i < c.count; ++i) {
            held = held || c.points[i].normalImpulse != 0.0f || lengthSquared(c.points[i].tangentImpulse) != 0.0f;
        }
        if (!held) { return; }
        PlanarState st(a, b, c.plane);
        for (int i = 0; i < c.count; ++i) {
            const DPoint& p = c.points[i];
            const DPlanarAxes x = planarAxesOf(ax[3 * i]);
            st.push(c.normal, x.normalA, x.normalB, p.normalImpulse);
            st.push(c.tangent1, x.tangentA, x.tangentB, dot(p.tangentImpulse, c.tangent1));
        }
        if (c.rollingResistance > 0.0f) {
            const float r = dot(c.rollingImpulse, c.plane);
            st.wa -= st.ia * r;
            st.wb += st.ib * r;
        }
        st.store(a, b, c.plane, !anchored(a), !anchored(b));
        return;
    }
    const bool moveA = !laned || !anchored(a), moveB = !laned || !anchored(b);
    for (int i = 0; i < c.count; ++i) {
        const DPoint& p = c.points[i];
        const Axis xn = ax[3 * i], x1 = ax[3 * i + 1], x2 = ax[3 * i + 2];
        pushMoving(a, b, xn, p.normalImpulse, moveA, moveB);
        pushMoving(a, b, x1, dot(p.tangentImpulse, c.tangent1), moveA, moveB);
        pushMoving(a, b, x2, dot(p.tangentImpulse, c.tangent2), moveA, moveB);
    }
    if (c.rollingResistance > 0.0f) {
        a.w -= a.invInertiaWorld * c.rollingImpulse;
        b.w += b.invInertiaWorld * c.rollingImpulse;
    }
}

// One step along the relative spin, held to the rolling limit (src/solver.cpp:225-251). Rolling contacts are
// never laned, so this runs one contact at a time and pushes both bodies as the reference does.
template <class BodyT>
TF_HD void resistTurning(BodyT& a, BodyT& b, DContact& c) {
    const Vec3 spin = b.w - a.w;
    const float speed = length(spin);
    Vec3 total = c.rollingImpulse;
    if (speed > 0.0f) {
        const Vec3 d = spin * (1.0f / speed);
        const Vec3 ia = a.invInertiaWorld * d, ib = b.invInertiaWorld * d;
        const float k = dot(d, ia) + dot(d, ib);
        if (k > 0.0f) {
            const float lambda = -speed / k;
            total += d * lambda;
            a.w -= ia * lambda;
            b.w += ib * lambda;
        }
    }
    float normal = 0.0f;
    for (int i = 0; i < c.count; ++i) { normal += c.points[i].normalImpulse; }
    const float limit = c.rollingResistance * c.rollingRadius * normal;
    const float mag = length(total);
    if (mag > limit) {
        const Vec3 fix = total * (limit / mag) - total;
        a.w -= a.invInertiaWorld * fix;
        b.w += b.invInertiaWorld * fix;
        total += fix;
    }
    c.rollingImpulse = total;
}

// The cosine and sine of a body's turn about n since the substep's base pose (src/solver.cpp:137-141).
template <class BodyT>
TF_HD Vec2 planarTurn(const BodyT& b, const Vec3& n) {
    const Quat& q = b.dq;
    return Vec2{ q.w * q.w - (q.x * q.x + q.y * q.y + q.z * q.z), 2.0f * q.w * dot(n, Vec3{ q.x, q.y, q.z }) };
}

// A planar contact's rows in the plane: soft normal rows, one friction row per point along the in-plane
// tangent, and the rolling row about the plane normal (src/solver.cpp:143-209).
template <class BodyT>
TF_HD void solvePlanar(BodyT& a, BodyT& b, DContact& c, const StepParams& P, bool useBias, const Axis* __restrict__ ax) {
    const bool moveA = !anchored(a), moveB = !anchored(b);
    const Softness soft = (!moveA || !moveB) ? P.staticSoft : P.contactSoft;
    const float shift = dot(b.dp - a.dp, c.normal);
    const Vec2 ta = planarTurn(a, c.plane), tb = planarTurn(b, c.plane);
    PlanarState st(a, b, c.plane);
    bool changed = false;
    for (int i = 0; i < c.count; ++i) {
        DPoint& p = c.points[i];
        const DPlanarAxes x = planarAxesOf(ax[3 * i]);
        // A turned anchor reaches along the normal by its tangent arm times the cosine plus its normal arm
        // times the sine.
        const float reachA = ta.x * x.tangentA + ta.y * x.normalA;
        const float reachB = tb.x * x.tangentB + tb.y * x.normalB;
        const float sep = shift + reachB - reachA + p.adjustedSeparation;
        float bias = 0.0f, massScale = 1.0f, impulseScale = 0.0f;
        if (sep > 0.0f) {
            bias = sep * P.invH;
        } else if (useBias) {
            bias = maxf(soft.biasRate * sep, -P.maxPushout);
            massScale = soft.massScale;
            impulseScale = soft.impulseScale;
        }
        const float vn = st.speed(c.normal, x.normalA, x.normalB);
        float impulse = -x.normalMass * massScale * (vn + bias) - impulseScale * p.normalImpulse;
        const float total = maxf(p.normalImpulse + impulse, 0.0f);
        impulse = total - p.normalImpulse;
        p.normalImpulse = total;
        p.maxNormalImpulse = maxf(p.maxNormalImpulse, impulse);
        if (impulse != 0.0f) {
            st.push(c.normal, x.normalA, x.normalB, impulse);
            changed = true;
        }
    }
    for (int j = 0; j < c.count; ++j) {
        const int i = useBias ? j : c.count - 1 - j;
        DPoint& p = c.points[i];
        const DPlanarAxes x = planarAxesOf(ax[3 * i]);
        const float old = dot(p.tangentImpulse, c.tangent1);
        // With no normal impulse the friction limit is zero, so a point holding no friction keeps none.
        if (p.normalImpulse == 0.0f && old == 0.0f) { continue; }
        changed = true;
        const float limit = c.friction * p.normalImpulse;
        const float t = minf(maxf(old - x.tangentMass * st.speed(c.tangent1, x.tangentA, x.tangentB), -limit), limit);
        p.tangentImpulse = c.tangent1 * t;
        st.push(c.tangent1, x.tangentA, x.tangentB, t - old);
    }
    if (c.rollingResistance > 0.0f) {
        changed = true;
        float total = dot(c.rollingImpulse, c.plane);
        const float spin = st.wb - st.wa;
        const float k = st.ia + st.ib;
        if (spin != 0.0f && k > 0.0f) {
            const float lambda = -spin / k;
            total += lambda;
            st.wa -= st.ia * lambda;
            st.wb += st.ib * lambda;
        }
        float normal = 0.0f;
        for (int i = 0; i < c.count; ++i) { normal += c.points[i].normalImpulse; }
        const float limit = c.rollingResistance * c.rollingRadius * normal;
        const float held = minf(maxf(total, -limit), limit);
        st.wa -= st.ia * (held - total);
        st.wb += st.ib * (held - total);
        c.rollingImpulse = c.plane * held;
    }
    if (changed) { st.store(a, b, c.plane, moveA, moveB); }
}

// The soft normal rows, then friction (forward in the biased pass, reverse in relax), then rolling
// (src/solver.cpp:360-421).
template <class BodyT>
TF_HD void solveContact(BodyT& a, BodyT& b, DContact& c, const StepParams& P, bool useBias, const Axis* __restrict__ ax) {
    if (c.flags & kCPlanar) {
        solvePlanar(a, b, c, P, useBias, ax);
        return;
    }
    const bool moveA = !anchored(a), moveB = !anchored(b);
    const Softness soft = (!moveA || !moveB) ? P.staticSoft : P.contactSoft;
    const Vec3 dp = b.dp - a.dp;
    for (int i = 0; i < c.count; ++i) {
        DPoint& p = c.points[i];
        const Vec3 d = dp + turned(b, p.anchorB) - turned(a, p.anchorA);
        const float sep = dot(d, c.normal) + p.adjustedSeparation;
        float bias = 0.0f, massScale = 1.0f, impulseScale = 0.0f;
        if (sep > 0.0f) {
            bias = sep * P.invH;
        } else if (useBias) {
            bias = maxf(soft.biasRate * sep, -P.maxPushout);
            massScale = soft.massScale;
            impulseScale = soft.impulseScale;
        }
        const Axis x = ax[3 * i];
        const float vn = speedAlong(a, b, c.normal, x);
        float impulse = -x.mass * massScale * (vn + bias) - impulseScale * p.normalImpulse;
        const float total = maxf(p.normalImpulse + impulse, 0.0f);
        impulse = total - p.normalImpulse;
        p.normalImpulse = total;
        p.maxNormalImpulse = maxf(p.maxNormalImpulse, impulse);
        pushMoving(a, b, x, impulse, moveA, moveB);
    }
    for (int j = 0; j < c.count; ++j) {
        const int i = useBias ? j : c.count - 1 - j;
        DPoint& p = c.points[i];
        const Axis x1 = ax[3 * i + 1], x2 = ax[3 * i + 2];
        const float old1 = dot(p.tangentImpulse, c.tangent1), old2 = dot(p.tangentImpulse, c.tangent2);
        float t1 = old1 - x1.mass * speedAlong(a, b, c.tangent1, x1);
        float t2 = old2 - x2.mass * speedAlong(a, b, c.tangent2, x2);
        const float limit = c.friction * p.normalImpulse;
        const float mag = sqrtf(t1 * t1 + t2 * t2);
        if (mag > limit) {
            const float scale = mag > 0.0f ? limit / mag : 0.0f;
            t1 *= scale;
            t2 *= scale;
        }
        p.tangentImpulse = c.tangent1 * t1 + c.tangent2 * t2;
        pushMoving(a, b, x1, t1 - old1, moveA, moveB);
        pushMoving(a, b, x2, t2 - old2, moveA, moveB);
    }
    if (c.rollingResistance > 0.0f) { resistTurning(a, b, c); }
}

// The solver state a laned contact reads and writes: velocities, the substep's displacement and turn, and
// the flags that say whether the body moves. Laned contacts are never planar or rolling, so they need no
// inertia.
struct LanedBody {
    Vec3 v, w, dp;
    Quat dq;
    uint32_t type, awake;
};

// warmStartContact for a laned contact, its points' impulses read into registers before any body is pushed.
template <class BodyT>
TF_HD void warmStartLaned(BodyT& a, BodyT& b, const DContact& c, const Axis* __restrict__ ax) {
    const bool moveA = !anchored(a), moveB = !anchored(b);
    const int n = c.count;
    const Vec3 t1 = c.tangent1, t2 = c.tangent2;
    float ni[4] = { 0, 0, 0, 0 };
    Vec3 ti[4] = {};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (i < n) {
            ni[i] = c.points[i].normalImpulse;
            ti[i] = c.points[i].tangentImpulse;
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (i < n) {
            const Axis xn = ax[3 * i], x1 = ax[3 * i + 1], x2 = ax[3 * i + 2];
            pushMoving(a, b, xn, ni[i], moveA, moveB);
            pushMoving(a, b, x1, dot(ti[i], t1), moveA, moveB);
            pushMoving(a, b, x2, dot(ti[i], t2), moveA, moveB);
        }
    }
}

// solveContact for a laned contact (no rolling row): the same operations in the same order, with the points'
// state read into registers first and written back once at the end.
template <class BodyT>
TF_HD void solveLaned(BodyT& a, BodyT& b, DContact& c, const StepParams& P, bool useBias, const Axis* __restrict__ ax) {
    const bool moveA = !anchored(a), moveB = !anchored(b);
    const Softness soft = (!moveA || !moveB) ? P.staticSoft : P.contactSoft;
    const int n = c.count;
    const Vec3 normal = c.normal, t1 = c.tangent1, t2 = c.tangent2;
    const float friction = c.friction;
    Vec3 rA[4] = {}, rB[4] = {}, ti[4] = {};
    float adj[4] = { 0, 0, 0, 0 }, ni[4] = { 0, 0, 0, 0 }, mi[4] = { 0, 0, 0, 0 };
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (i < n) {
            const DPoint& p = c.points[i];
            rA[i] = p.anchorA;
            rB[i] = p.anchorB;
            adj[i] = p.adjustedSeparation;
            ni[i] = p.normalImpulse;
            mi[i] = p.maxNormalImpulse;
            ti[i] = p.tangentImpulse;
        }
    }
    const Vec3 dp = b.dp - a.dp;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (i < n) {
            const Vec3 d = dp + turned(b, rB[i]) - turned(a, rA[i]);
            const float sep = dot(d, normal) + adj[i];
            float bias = 0.0f, massScale = 1.0f, impulseScale = 0.0f;
            if (sep > 0.0f) {
                bias = sep * P.invH;
            } else if (useBias) {
                bias = maxf(soft.biasRate * sep, -P.maxPushout);
                massScale = soft.massScale;
                impulseScale = soft.impulseScale;
            }
            const Axis x = ax[3 * i];
            const float vn = speedAlong(a, b, normal, x);
            float impulse = -x.mass * massScale * (vn + bias) - impulseScale * ni[i];
            const float total = maxf(ni[i] + impulse, 0.0f);
            impulse = total - ni[i];
            ni[i] = total;
            mi[i] = maxf(mi[i], impulse);
            pushMoving(a, b, x, impulse, moveA, moveB);
        }
    }
    auto row = [&](int i) {
        const Axis x1 = ax[3 * i + 1], x2 = ax[3 * i + 2];
        const float old1 = dot(ti[i], t1), old2 = dot(ti[i], t2);
        float f1 = old1 - x1.mass * speedAlong(a, b, t1, x1);
        float f2 = old2 - x2.mass * speedAlong(a, b, t2, x2);
        const float limit = friction * ni[i];
        const float mag = sqrtf(f1 * f1 + f2 * f2);
        if (mag > limit) {
            const float scale = mag > 0.0f ? limit / mag : 0.0f;
            f1 *= scale;
            f2 *= scale;
        }
        ti[i] = t1 * f1 + t2 * f2;
        pushMoving(a, b, x1, f1 - old1, moveA, moveB);
        pushMoving(a, b, x2, f2 - old2, moveA, moveB);
    };
    if (useBias) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (i < n) { row(i); }
        }
    } else {
#pragma unroll
        for (int i = 3; i >= 0; --i) {
            if (i < n) { row(i); }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (i < n) {
            DPoint& p = c.points[i];
            p.normalImpulse = ni[i];
            p.maxNormalImpulse = mi[i];
            p.tangentImpulse = ti[i];
        }
    }
}

// One restitution pass over the points that approached fast (src/solver.cpp:423-460, src/lanes.cpp:318-352),
// pushing as warmStartContact does.
template <class BodyT>
TF_HD void restituteContact(BodyT& a, BodyT& b, DContact& c, const StepParams& P, bool laned, const Axis* __restrict__ ax) {
    if (c.restitution == 0.0f) { return; }
    if (c.flags & kCPlanar) {
        // src/solver.cpp:430-445: the bodies are stored back whether or not a point took an impulse.
        PlanarState st(a, b, c.plane);
        for (int i = 0; i < c.count; ++i) {
            DPoint& p = c.points[i];
            if (p.relativeVelocity > -P.restitutionThreshold || p.maxNormalImpulse == 0.0f) { continue; }
            const DPlanarAxes x = planarAxesOf(ax[3 * i]);
            const float vn = st.speed(c.normal, x.normalA, x.normalB);
            float impulse = -x.normalMass * (vn + c.restitution * p.relativeVelocity);
            const float total = maxf(p.normalImpulse + impulse, 0.0f);
            impulse = total - p.normalImpulse;
            p.normalImpulse = total;
            p.maxNormalImpulse = maxf(p.maxNormalImpulse, impulse);
            st.push(c.normal, x.normalA, x.normalB, impulse);
        }
        st.store(a, b, c.plane, !anchored(a), !anchored(b));
        return;
    }
    const bool moveA = !laned || !anchored(a), moveB = !laned || !anchored(b);
    for (int i = 0; i < c.count; ++i) {
        DPoint& p = c.points[i];
        if (p.relativeVelocity > -P.restitutionThreshold || p.maxNormalImpulse == 0.0f) { continue; }
        const Axis x = ax[3 * i];
        const float vn = speedAlong(a, b, c.normal, x);
        float impulse = -x.mass * (vn + c.restitution * p.relativeVelocity);
        const float total = maxf(p.normalImpulse + impulse, 0.0f);
        impulse = total - p.normalImpulse;
        p.normalImpulse = total;
        p.maxNormalImpulse = maxf(p.maxNormalImpulse, impulse);
        pushMoving(a, b, x, impulse, moveA, moveB);
    }
}

// restituteContact for a laned contact, whose axes are not stored: each point's normal axis is built again from
// the bodies' world inverse mass and inertia, unchanged since the contact's record was last built, which gives
// the bits the stored axis had. Laned contacts are never planar.
template <class BodyT>
TF_HD void restituteLaned(BodyT& a, BodyT& b, DContact& c, const StepParams& P) {
    if (c.restitution == 0.0f) { return; }
    const bool moveA = !anchored(a), moveB = !anchored(b);
    for (int i = 0; i < c.count; ++i) {
        DPoint& p = c.points[i];
        if (p.relativeVelocity > -P.restitutionThreshold || p.maxNormalImpulse == 0.0f) { continue; }
        const Axis x = makeAxis(a, b, p.anchorA, p.anchorB, c.normal);
        const float vn = speedAlong(a, b, c.normal, x);
        float impulse = -x.mass * (vn + c.restitution * p.relativeVelocity);
        const float total = maxf(p.normalImpulse + impulse, 0.0f);
        impulse = total - p.normalImpulse;
        p.normalImpulse = total;
        p.maxNormalImpulse = maxf(p.maxNormalImpulse, impulse);
        pushMoving(a, b, x, impulse, moveA, moveB);
    }
}

// Gravity, forces, damping, locks and the speed limits (src/world.cpp:1141-1151).
template <class BodyT>
TF_HD void integrateVelocity(BodyT& b, const StepParams& P) {
    if (!b.alive || b.type != kDynamic || !b.awake) { return; }
    const float h = P.h;
    b.v = b.v + (P.gravity * b.gravityScale + b.force * b.invMass) * h;
    b.v = b.linearProj * (b.v * (1.0f / (1.0f + h * b.linearDamping)));
    b.w = b.w + b.invInertiaWorld * b.torque * h;
    b.w = b.angularProj * (b.w * (1.0f / (1.0f + h * b.angularDamping)));
    limitSpeed(b, P.maxLinearSpeed, P.maxAngularSpeed);
}

// The speed limits, then the pose update (src/world.cpp:1161-1172).
template <class BodyT>
TF_HD void integratePosition(BodyT& b, const StepParams& P) {
    if (b.alive) { limitSpeed(b, P.maxLinearSpeed, P.maxAngularSpeed); }
    if (!b.alive || b.type == kStatic) { return; }
    if (b.type == kDynamic && !b.awake) { return; }
    const float h = P.h;
    b.com += b.v * h;
    b.dp += b.v * h;
    b.xf.q = integrate(b.xf.q, b.w, h);
    b.dq = b.xf.q * conjugate(b.qBase);
    b.xf.p = b.com - rotate(b.xf.q, b.localCenter);
}

}
