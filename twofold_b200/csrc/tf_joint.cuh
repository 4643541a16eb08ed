// Joints in the substep loop (src/joint.cpp): warm start, the biased and relaxing solves, the reaction each
// relaxing solve adds, the position-level settle after the step and the speed-limit scaling of warm starts.
// Every function restates its reference counterpart's arithmetic in order; the world end of a joint is a
// static body at the origin. Joints of a world run one after another in index order on one thread, before
// the world's contacts in each pass, as the reference solves them.
#pragma once

#include "tf_continuous.cuh"
#include "tf_solver.cuh"

namespace tfb {

constexpr float kJointPi = 3.14159265358979f;
constexpr int kSettleIterations = 2;  // src/world.cpp:16

// The fields of a body a joint reads and writes.
struct JBody {
    Vec3 v, w, com;
    Transform xf;
    Vec3 localCenter;
    Mat3 invMassWorld, invInertiaWorld;
    float invMass, kept;
    uint32_t type, awake, locks;
};

TF_HD JBody worldEnd() {
    JBody b;
    b.v = zero3();
    b.w = zero3();
    b.com = zero3();
    b.xf = Transform{ zero3(), qid() };
    b.localCenter = zero3();
    b.invMassWorld = mzero();
    b.invInertiaWorld = mzero();
    b.invMass = 0.0f;
    b.kept = 1.0f;
    b.type = kStatic;
    b.awake = 1;
    b.locks = 0;
    return b;
}

TF_HD JBody jointBodyOf(const DBody& d) {
    JBody b;
    b.v = d.v;
    b.w = d.w;
    b.com = d.com;
    b.xf = d.xf;
    b.localCenter = d.localCenter;
    b.invMassWorld = d.invMassWorld;
    b.invInertiaWorld = d.invInertiaWorld;
    b.invMass = d.invMass;
    b.kept = d.kept;
    b.type = d.type;
    b.awake = d.awake;
    b.locks = d.locks;
    return b;
}

TF_HD Mat3 skewOf(const Vec3& v) {
    Mat3 m;
    m.r[0] = { 0.0f, -v.z, v.y };
    m.r[1] = { v.z, 0.0f, -v.x };
    m.r[2] = { -v.y, v.x, 0.0f };
    return m;
}

TF_HD float traceOf(const Mat3& m) { return m.r[0].x + m.r[1].y + m.r[2].z; }

// The inverse of m on the directions it acts in (src/joint.cpp:21-70): the plain inverse when m is well
// conditioned, else cyclic Jacobi rotations of its symmetric part and the reciprocals of its eigenvalues above
// a relative floor.
TF_HD Mat3 pseudoInverse(const Mat3& m) {
    const float tr = traceOf(m);
    if (tr <= 0.0f) { return mzero(); }
    const float third = tr / 3.0f;
    if (dot(m.r[0], cross(m.r[1], m.r[2])) > 1e-3f * third * third * third) { return inverse(m); }
    float a[3][3], v[3][3];
    for (int i = 0; i < 3; ++i) {
        for (int k = 0; k < 3; ++k) {
            a[i][k] = 0.5f * (comp(m.r[i], k) + comp(m.r[k], i));
            v[i][k] = i == k ? 1.0f : 0.0f;
        }
    }
    for (int sweep = 0; sweep < 8; ++sweep) {
        if (a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2] <= 1e-14f * tr * tr) { break; }
        for (int p = 0; p < 2; ++p) {
            for (int q = p + 1; q < 3; ++q) {
                if (a[p][q] == 0.0f) { continue; }
                const float theta = (a[q][q] - a[p][p]) / (2.0f * a[p][q]);
                const float t = (theta >= 0.0f ? 1.0f : -1.0f) / (fabsf(theta) + sqrtf(theta * theta + 1.0f));
                const float c = 1.0f / sqrtf(t * t + 1.0f), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    const float kp = a[k][p], kq = a[k][q];
                    a[k][p] = c * kp - s * kq;
                    a[k][q] = s * kp + c * kq;
                }
                for (int k = 0; k < 3; ++k) {
                    const float pk = a[p][k], qk = a[q][k];
                    a[p][k] = c * pk - s * qk;
                    a[q][k] = s * pk + c * qk;
                }
                for (int k = 0; k < 3; ++k) {
                    const float kp = v[k][p], kq = v[k][q];
                    v[k][p] = c * kp - s * kq;
                    v[k][q] = s * kp + c * kq;
                }
            }
        }
    }
    const float top = maxf(a[0][0], maxf(a[1][1], a[2][2]));
    Mat3 out = mzero();
    for (int i = 0; i < 3; ++i) {
        if (a[i][i] <= 1e-6f * top) { continue; }
        const Vec3 e{ v[0][i], v[1][i], v[2][i] };
        out = out + outer(e, e) * (1.0f / a[i][i]);
    }
    return out;
}

// The rotation of an orthonormal frame (include/twofold/math.h:197-214), for a swing-twist joint's frame.
TF_HD Quat quatOfMat3(const Mat3& m) {
    const float tr = m.r[0].x + m.r[1].y + m.r[2].z;
    Quat q;
    if (tr > 0.0f) {
        const float s = sqrtf(tr + 1.0f) * 2.0f;
        q = { (m.r[2].y - m.r[1].z) / s, (m.r[0].z - m.r[2].x) / s, (m.r[1].x - m.r[0].y) / s, 0.25f * s };
    } else if (m.r[0].x > m.r[1].y && m.r[0].x > m.r[2].z) {
        const float s = sqrtf(1.0f + m.r[0].x - m.r[1].y - m.r[2].z) * 2.0f;
        q = { 0.25f * s, (m.r[0].y + m.r[1].x) / s, (m.r[0].z + m.r[2].x) / s, (m.r[2].y - m.r[1].z) / s };
    } else if (m.r[1].y > m.r[2].z) {
        const float s = sqrtf(1.0f + m.r[1].y - m.r[0].x - m.r[2].z) * 2.0f;
        q = { (m.r[0].y + m.r[1].x) / s, 0.25f * s, (m.r[1].z + m.r[2].y) / s, (m.r[0].z - m.r[2].x) / s };
    } else {
        const float s = sqrtf(1.0f + m.r[2].z - m.r[0].x - m.r[1].y) * 2.0f;
        q = { (m.r[0].z + m.r[2].x) / s, (m.r[1].z + m.r[2].y) / s, 0.25f * s, (m.r[1].x - m.r[0].y) / s };
    }
    return normalize(q);
}

// src/joint.cpp:74.
TF_HD Vec3 jointArm(const JBody& b, const Vec3& local) { return rotate(b.xf.q, local - b.localCenter); }

// A pure turn about d (src/joint.cpp:76-84).
TF_HD Axis makeTurn(const JBody& a, const JBody& b, const Vec3& d) {
    Axis x;
    x.armA = d;
    x.armB = d;
    x.linearA = zero3();
    x.linearB = zero3();
    x.angularA = a.invInertiaWorld * d;
    x.angularB = b.invInertiaWorld * d;
    const float k = dot(d, x.angularA) + dot(d, x.angularB);
    x.mass = k > 1e-6f * (traceOf(a.invInertiaWorld) + traceOf(b.invInertiaWorld)) ? 1.0f / k : 0.0f;
    return x;
}

TF_HD Axis flipped(const Axis& x) {
    Axis f = x;
    f.armA = -x.armA;
    f.armB = -x.armB;
    f.linearA = -x.linearA;
    f.angularA = -x.angularA;
    f.linearB = -x.linearB;
    f.angularB = -x.angularB;
    return f;
}

// How a point at r from the centre moves per unit impulse there (src/joint.cpp:98-101).
TF_HD Mat3 pointResponse(const JBody& b, const Vec3& r) {
    const Mat3 s = skewOf(r);
    return b.invMassWorld - s * b.invInertiaWorld * s;
}

// A turn about axis through the anchors, with the point impulse per unit turn that holds them
// (src/joint.cpp:104-117).
TF_HD Axis anchoredTurn(const JBody& a, const JBody& b, const Vec3& ra, const Vec3& rb, const Vec3& axis,
                        Vec3& pointImpulse) {
    const Vec3 drift = cross(b.invInertiaWorld * axis, rb) + cross(a.invInertiaWorld * axis, ra);
    pointImpulse = pseudoInverse(pointResponse(a, ra) + pointResponse(b, rb)) * -drift;
    Axis x;
    x.armA = axis + cross(ra, pointImpulse);
    x.armB = axis + cross(rb, pointImpulse);
    x.linearA = a.invMassWorld * pointImpulse;
    x.angularA = a.invInertiaWorld * x.armA;
    x.linearB = b.invMassWorld * pointImpulse;
    x.angularB = b.invInertiaWorld * x.armB;
    const float k = dot(pointImpulse, x.linearA + x.linearB) + dot(x.armA, x.angularA) + dot(x.armB, x.angularB);
    x.mass = k > 1e-6f * (traceOf(a.invInertiaWorld) + traceOf(b.invInertiaWorld)) ? 1.0f / k : 0.0f;
    return x;
}

// A slide along axis with the turn impulse that keeps the relative rotation (src/joint.cpp:120-130).
TF_HD Axis lockedSlide(const JBody& a, const JBody& b, const Vec3& ra, const Vec3& rb, const Vec3& axis) {
    Axis x = makeAxis(a, b, ra, rb, axis);
    const Vec3 twist = pseudoInverse(a.invInertiaWorld + b.invInertiaWorld) * -(x.angularA + x.angularB);
    x.armA += twist;
    x.armB += twist;
    x.angularA = a.invInertiaWorld * x.armA;
    x.angularB = b.invInertiaWorld * x.armB;
    const float k = dot(axis, x.linearA + x.linearB) + dot(x.armA, x.angularA) + dot(x.armB, x.angularB);
    x.mass = k > 1e-6f * (a.invMass + b.invMass) ? 1.0f / k : 0.0f;
    return x;
}

// The share of a distance error locked bodies can correct (src/joint.cpp:134-138).
TF_HD float reachable(const JBody& a, const JBody& b, const Axis& x) {
    const float invMass = a.invMass + b.invMass;
    if ((!a.locks && !b.locks) || x.mass <= 0.0f || invMass <= 0.0f) { return 1.0f; }
    return minf(1.0f, 1.0f / (x.mass * invMass));
}

TF_HD void pushAxis(JBody& a, JBody& b, const Axis& x, float impulse) {
    a.v -= x.linearA * impulse;
    a.w -= x.angularA * impulse;
    b.v += x.linearB * impulse;
    b.w += x.angularB * impulse;
}

TF_HD void pushPoint(JBody& a, JBody& b, const Vec3& ra, const Vec3& rb, const Vec3& impulse) {
    a.v -= a.invMassWorld * impulse;
    a.w -= a.invInertiaWorld * cross(ra, impulse);
    b.v += b.invMassWorld * impulse;
    b.w += b.invInertiaWorld * cross(rb, impulse);
}

TF_HD void pushTurn(JBody& a, JBody& b, const Vec3& impulse) {
    a.w -= a.invInertiaWorld * impulse;
    b.w += b.invInertiaWorld * impulse;
}

// src/joint.cpp:155-163.
TF_HD void solvePoint(JBody& a, JBody& b, const Vec3& ra, const Vec3& rb, const Mat3& proj, const Vec3& error, Vec3& total,
                      const Softness& soft) {
    const Mat3 k = proj * (pointResponse(a, ra) + pointResponse(b, rb)) * proj;
    const Vec3 speed = proj * (b.v + cross(b.w, rb) - a.v - cross(a.w, ra));
    const Vec3 old = proj * total;
    const Vec3 impulse = pseudoInverse(k) * (speed + error * soft.biasRate) * -soft.massScale - old * soft.impulseScale;
    total = old + impulse;
    pushPoint(a, b, ra, rb, impulse);
}

// src/joint.cpp:166-173.
TF_HD void solveTurn(JBody& a, JBody& b, const Mat3& proj, const Vec3& error, Vec3& total, const Softness& soft) {
    const Mat3 k = proj * (a.invInertiaWorld + b.invInertiaWorld) * proj;
    const Vec3 speed = proj * (b.w - a.w);
    const Vec3 old = proj * total;
    const Vec3 impulse = pseudoInverse(k) * (speed + error * soft.biasRate) * -soft.massScale - old * soft.impulseScale;
    total = old + impulse;
    pushTurn(a, b, impulse);
}

TF_HD void solveEqual(JBody& a, JBody& b, const Axis& x, const Vec3& d, float error, float& total, const Softness& soft) {
    const float impulse =
        -x.mass * soft.massScale * (speedAlong(a, b, d, x) + soft.biasRate * error) - soft.impulseScale * total;
    total += impulse;
    pushAxis(a, b, x, impulse);
}

// Keeps error at or above zero (src/joint.cpp:183-198).
TF_HD void solveLimit(JBody& a, JBody& b, const Axis& x, const Vec3& d, float error, float& total, const StepParams& P,
                      const Softness& jointSoft, bool useBias) {
    float bias = 0.0f, massScale = 1.0f, impulseScale = 0.0f;
    if (error > 0.0f) {
        bias = error * P.invH;
    } else if (useBias) {
        bias = jointSoft.biasRate * error;
        massScale = jointSoft.massScale;
        impulseScale = jointSoft.impulseScale;
    }
    float impulse = -x.mass * massScale * (speedAlong(a, b, d, x) + bias) - impulseScale * total;
    const float next = maxf(total + impulse, 0.0f);
    impulse = next - total;
    total = next;
    pushAxis(a, b, x, impulse);
}

TF_HD void solveMotor(JBody& a, JBody& b, const Axis& x, const Vec3& d, float speed, float maxImpulse, float& total) {
    const float old = total;
    total = minf(maxf(old - x.mass * (speedAlong(a, b, d, x) - speed), -maxImpulse), maxImpulse);
    pushAxis(a, b, x, total - old);
}

TF_HD Vec3 turnError(const DJoint& j, const JBody& a, const JBody& b) {
    Quat e = b.xf.q * conjugate(a.xf.q * j.restTurn);
    if (e.w < 0.0f) { e = -e; }
    return qvec(e) * 2.0f;
}

TF_HD float hingeAngle(const DJoint& j, const JBody& a, const JBody& b) {
    const Vec3 axis = rotate(a.xf.q, j.axisA);
    const Vec3 ra = rotate(a.xf.q, j.refA);
    const Vec3 rb = rotate(b.xf.q, j.refB);
    return atan2Rounded(dot(cross(ra, rb), axis), dot(ra, rb));
}

TF_HD Mat3 across(const Vec3& axis) { return mid() - outer(axis, axis); }

// src/joint.cpp:222-229.
TF_HD void solveTurnFriction(JBody& a, JBody& b, float maxImpulse, Vec3& total) {
    const Vec3 old = total;
    Vec3 next = old - pseudoInverse(a.invInertiaWorld + b.invInertiaWorld) * (b.w - a.w);
    const float len = length(next);
    if (len > maxImpulse) { next = next * (maxImpulse / len); }
    total = next;
    pushTurn(a, b, next - old);
}

// Body B's turn in body A's joint frame as a swing of the x axis and a twist about it (src/joint.cpp:232-252).
struct SwingTwist {
    Quat frame;
    Vec3 axisA, axisB;
    Quat swing;
    float twist;
};

TF_HD SwingTwist swingTwistOf(const DJoint& j, const JBody& a, const JBody& b) {
    SwingTwist st;
    st.frame = a.xf.q * j.frameA;
    const Quat frameB = b.xf.q * j.frameB;
    st.axisA = rotate(st.frame, Vec3{ 1, 0, 0 });
    st.axisB = rotate(frameB, Vec3{ 1, 0, 0 });
    Quat r = conjugate(st.frame) * frameB;
    if (r.w < 0.0f) { r = -r; }
    const float s = sqrtf(r.x * r.x + r.w * r.w);
    const Quat t = s > 0.0f ? Quat{ r.x / s, 0.0f, 0.0f, r.w / s } : qid();
    st.swing = r * conjugate(t);
    st.twist = 2.0f * atan2Rounded(t.x, t.w);
    return st;
}

TF_HD bool twistRate(const SwingTwist& st, Vec3& rate) {
    const float c = 1.0f + dot(st.axisA, st.axisB);
    if (c < 1e-3f) { return false; }
    rate = (st.axisA + st.axisB) / c;
    return true;
}

TF_HD bool swingFree(const DJoint& j) { return j.swingY >= 1.0f && j.swingZ >= 1.0f; }

// Room left before the swing meets its cone, and the relative spin that changes it (src/joint.cpp:266-287).
TF_HD bool swingRoom(const DJoint& j, const SwingTwist& st, float& error, Vec3& rate) {
    const float len = sqrtf(st.swing.y * st.swing.y + st.swing.z * st.swing.z);
    if (len < 1e-6f) { return false; }
    const float cy = st.swing.y / len, cz = st.swing.z / len;
    const float ey = cy / j.swingZ, ez = cz / j.swingY;
    const float reach = 1.0f / sqrtf(ey * ey + ez * ez);
    const Vec3 k = rotate(st.frame, Vec3{ 0.0f, cy, cz });
    rate = -k;
    float allowed = kJointPi;
    if (reach < 1.0f) {
        allowed = 2.0f * asinRounded(reach);
        const float slope = 2.0f * reach * reach * reach * (ey * cz / j.swingZ - ez * cy / j.swingY) /
                            sqrtf(1.0f - reach * reach);
        const Vec3 side = cross(st.axisB, k);
        const float det = dot(st.axisA, side);
        if (fabsf(det) > 1e-6f) { rate += side * (slope / det); }
    }
    error = allowed - 2.0f * atan2Rounded(len, st.swing.w);
    return true;
}

// src/joint.cpp:289-335.
TF_HD void warmStartJoint(JBody& a, JBody& b, const DJoint& j) {
    const Vec3 ra = jointArm(a, j.localA), rb = jointArm(b, j.localB);
    const Vec3 d = (b.com + rb) - (a.com + ra);
    float axial = j.axialImpulse + j.motorImpulse + j.lowerImpulse - j.upperImpulse;
    if (j.maxFriction > 0.0f) { axial += j.frictionImpulse; }
    switch (j.type) {
        case kJointPoint:
            pushPoint(a, b, ra, rb, j.linearImpulse);
            break;
        case kJointFixed:
            pushPoint(a, b, ra, rb, j.linearImpulse);
            pushTurn(a, b, j.angularImpulse);
            break;
        case kJointHinge: {
            const Vec3 axis = rotate(a.xf.q, j.axisA);
            Vec3 along;
            pushPoint(a, b, ra, rb, j.linearImpulse);
            pushTurn(a, b, across(axis) * j.angularImpulse);
            pushAxis(a, b, anchoredTurn(a, b, ra, rb, axis, along), axial);
            break;
        }
        case kJointSlider: {
            const Vec3 axis = rotate(a.xf.q, j.axisA);
            pushPoint(a, b, ra + d, rb, across(axis) * j.linearImpulse);
            pushTurn(a, b, j.angularImpulse);
            pushAxis(a, b, lockedSlide(a, b, ra + d, rb, axis), axial);
            break;
        }
        case kJointDistance: {
            const float len = length(d);
            if (len > 0.0f) { pushAxis(a, b, makeAxis(a, b, ra, rb, d / len), axial); }
            break;
        }
        default: {
            pushPoint(a, b, ra, rb, j.linearImpulse);
            pushTurn(a, b, j.frictionTurn);
            const SwingTwist st = swingTwistOf(j, a, b);
            Vec3 rate, along;
            if (axial != 0.0f && twistRate(st, rate)) { pushAxis(a, b, anchoredTurn(a, b, ra, rb, rate, along), axial); }
            float error = 0.0f;
            if (j.swingImpulse != 0.0f && swingRoom(j, st, error, rate)) {
                pushAxis(a, b, anchoredTurn(a, b, ra, rb, rate, along), j.swingImpulse);
            }
            break;
        }
    }
}

// src/joint.cpp:337-432.
TF_HD void solveJoint(JBody& a, JBody& b, DJoint& j, const StepParams& P, const Softness& jointSoft, bool useBias) {
    const Softness soft = useBias ? jointSoft : Softness{ 0.0f, 1.0f, 0.0f };
    const Vec3 ra = jointArm(a, j.localA), rb = jointArm(b, j.localB);
    const Vec3 d = (b.com + rb) - (a.com + ra);
    switch (j.type) {
        case kJointPoint:
            solvePoint(a, b, ra, rb, mid(), d, j.linearImpulse, soft);
            break;
        case kJointFixed:
            solveTurn(a, b, mid(), turnError(j, a, b), j.angularImpulse, soft);
            solvePoint(a, b, ra, rb, mid(), d, j.linearImpulse, soft);
            break;
        case kJointHinge: {
            const Vec3 axis = rotate(a.xf.q, j.axisA);
            Vec3 along;
            const Axis turn = anchoredTurn(a, b, ra, rb, axis, along);
            j.rowForce[0] = along;
            j.rowTorque[0] = axis;
            if (j.maxFriction > 0.0f) { solveMotor(a, b, turn, along, 0.0f, j.maxFriction * P.h, j.frictionImpulse); }
            if (j.maxMotor > 0.0f) { solveMotor(a, b, turn, along, j.motorSpeed, j.maxMotor * P.h, j.motorImpulse); }
            if (j.limited) {
                const float angle = hingeAngle(j, a, b);
                solveLimit(a, b, turn, along, angle - j.lower, j.lowerImpulse, P, jointSoft, useBias);
                solveLimit(a, b, flipped(turn), -along, j.upper - angle, j.upperImpulse, P, jointSoft, useBias);
            }
            solveTurn(a, b, across(axis), cross(axis, rotate(b.xf.q, j.axisB)), j.angularImpulse, soft);
            solvePoint(a, b, ra, rb, mid(), d, j.linearImpulse, soft);
            break;
        }
        case kJointSlider: {
            const Vec3 axis = rotate(a.xf.q, j.axisA);
            const Axis slide = lockedSlide(a, b, ra + d, rb, axis);
            j.rowForce[0] = axis;
            j.rowTorque[0] = slide.armB - cross(rb, axis);
            if (j.maxFriction > 0.0f) { solveMotor(a, b, slide, axis, 0.0f, j.maxFriction * P.h, j.frictionImpulse); }
            if (j.maxMotor > 0.0f) { solveMotor(a, b, slide, axis, j.motorSpeed, j.maxMotor * P.h, j.motorImpulse); }
            if (j.limited) {
                const float t = dot(d, axis);
                solveLimit(a, b, slide, axis, t - j.lower, j.lowerImpulse, P, jointSoft, useBias);
                solveLimit(a, b, flipped(slide), -axis, j.upper - t, j.upperImpulse, P, jointSoft, useBias);
            }
            solveTurn(a, b, mid(), turnError(j, a, b), j.angularImpulse, soft);
            const Mat3 side = across(axis);
            solvePoint(a, b, ra + d, rb, side, side * d, j.linearImpulse, soft);
            break;
        }
        case kJointDistance: {
            const float len = length(d);
            if (len <= 0.0f) { break; }
            const Vec3 u = d / len;
            const Axis x = makeAxis(a, b, ra, rb, u);
            const float reach = reachable(a, b, x);
            j.rowForce[0] = u;
            if (j.limited ? j.lower >= j.upper : j.hertz == 0.0f) {
                solveEqual(a, b, x, u, (len - (j.limited ? j.lower : j.length)) * reach, j.axialImpulse, soft);
                break;
            }
            if (j.hertz > 0.0f) {
                const Softness spring = makeSoft(j.hertz, j.dampingRatio, P.h);
                solveEqual(a, b, x, u, (len - j.length) * reach, j.axialImpulse, spring);
            }
            if (j.limited) {
                const float lower = len - j.lower, upper = j.upper - len;
                solveLimit(a, b, x, u, maxf(lower, lower * reach), j.lowerImpulse, P, jointSoft, useBias);
                solveLimit(a, b, flipped(x), -u, maxf(upper, upper * reach), j.upperImpulse, P, jointSoft, useBias);
            }
            break;
        }
        default: {
            if (j.maxFriction > 0.0f) { solveTurnFriction(a, b, j.maxFriction * P.h, j.frictionTurn); }
            const SwingTwist st = swingTwistOf(j, a, b);
            Vec3 rate, along;
            if (j.limited && twistRate(st, rate)) {
                const Axis turn = anchoredTurn(a, b, ra, rb, rate, along);
                j.rowForce[0] = along;
                j.rowTorque[0] = rate;
                solveLimit(a, b, turn, along, st.twist - j.lower, j.lowerImpulse, P, jointSoft, useBias);
                solveLimit(a, b, flipped(turn), -along, j.upper - st.twist, j.upperImpulse, P, jointSoft, useBias);
            } else {
                j.lowerImpulse = 0.0f;
                j.upperImpulse = 0.0f;
            }
            float error = 0.0f;
            if (!swingFree(j) && swingRoom(j, st, error, rate)) {
                const Axis turn = anchoredTurn(a, b, ra, rb, rate, along);
                j.rowForce[1] = along;
                j.rowTorque[1] = rate;
                solveLimit(a, b, turn, along, error, j.swingImpulse, P, jointSoft, useBias);
            } else {
                j.swingImpulse = 0.0f;
            }
            solvePoint(a, b, ra, rb, mid(), d, j.linearImpulse, soft);
            break;
        }
    }
}

// The force and torque on body B a relaxing solve adds up (src/joint.cpp:604-628).
TF_HD void addReaction(DJoint& j) {
    Vec3 force = j.linearImpulse, torque = zero3();
    const float axial = j.axialImpulse + j.motorImpulse + j.lowerImpulse - j.upperImpulse + j.frictionImpulse;
    switch (j.type) {
        case kJointPoint:
            break;
        case kJointFixed:
            torque = j.angularImpulse;
            break;
        case kJointHinge:
        case kJointSlider:
            force += j.rowForce[0] * axial;
            torque = j.angularImpulse + j.rowTorque[0] * axial;
            break;
        case kJointDistance:
            force = j.rowForce[0] * axial;
            break;
        default:
            force += j.rowForce[0] * axial + j.rowForce[1] * j.swingImpulse;
            torque = j.rowTorque[0] * axial + j.rowTorque[1] * j.swingImpulse + j.frictionTurn;
            break;
    }
    j.force += force;
    j.torque += torque;
}

// Position-level corrections after the step (src/joint.cpp:434-566): they move awake dynamic bodies only.
TF_HD void shiftBody(JBody& b, const Vec3& move, const Vec3& turn) {
    if (b.type != kDynamic || !b.awake) { return; }
    b.com += move;
    b.xf.q = integrate(b.xf.q, turn, 1.0f);
    b.xf.p = b.com - rotate(b.xf.q, b.localCenter);
}

TF_HD void movePoint(JBody& a, JBody& b, const Vec3& ra, const Vec3& rb, const Mat3& proj, const Vec3& error) {
    const Mat3 k = proj * (pointResponse(a, ra) + pointResponse(b, rb)) * proj;
    const Vec3 p = pseudoInverse(k) * (proj * error) * -1.0f;
    shiftBody(a, -(a.invMassWorld * p), -(a.invInertiaWorld * cross(ra, p)));
    shiftBody(b, b.invMassWorld * p, b.invInertiaWorld * cross(rb, p));
}

TF_HD void moveTurn(JBody& a, JBody& b, const Mat3& proj, const Vec3& error) {
    const Mat3 k = proj * (a.invInertiaWorld + b.invInertiaWorld) * proj;
    const Vec3 l = pseudoInverse(k) * (proj * error) * -1.0f;
    shiftBody(a, zero3(), -(a.invInertiaWorld * l));
    shiftBody(b, zero3(), b.invInertiaWorld * l);
}

TF_HD void moveAlong(JBody& a, JBody& b, const Axis& x, float error) {
    const float l = -x.mass * error;
    shiftBody(a, -(x.linearA * l), -(x.angularA * l));
    shiftBody(b, x.linearB * l, x.angularB * l);
}

TF_HD void settleJoint(JBody& a, JBody& b, const DJoint& j) {
    Vec3 ra = jointArm(a, j.localA), rb = jointArm(b, j.localB);
    Vec3 d = (b.com + rb) - (a.com + ra);
    auto measure = [&]() {
        ra = jointArm(a, j.localA);
        rb = jointArm(b, j.localB);
        d = (b.com + rb) - (a.com + ra);
    };
    switch (j.type) {
        case kJointPoint:
            movePoint(a, b, ra, rb, mid(), d);
            break;
        case kJointFixed:
            moveTurn(a, b, mid(), turnError(j, a, b));
            measure();
            movePoint(a, b, ra, rb, mid(), d);
            break;
        case kJointHinge: {
            const Vec3 axis = rotate(a.xf.q, j.axisA);
            if (j.limited) {
                const float angle = hingeAngle(j, a, b);
                const Axis turn = makeTurn(a, b, axis);
                if (angle < j.lower) { moveAlong(a, b, turn, angle - j.lower); }
                if (angle > j.upper) { moveAlong(a, b, turn, angle - j.upper); }
            }
            moveTurn(a, b, across(axis), cross(axis, rotate(b.xf.q, j.axisB)));
            measure();
            movePoint(a, b, ra, rb, mid(), d);
            break;
        }
        case kJointSlider: {
            moveTurn(a, b, mid(), turnError(j, a, b));
            measure();
            const Vec3 axis = rotate(a.xf.q, j.axisA);
            if (j.limited) {
                const float t = dot(d, axis);
                const Axis slide = lockedSlide(a, b, ra + d, rb, axis);
                if (t < j.lower) { moveAlong(a, b, slide, t - j.lower); }
                if (t > j.upper) { moveAlong(a, b, slide, t - j.upper); }
                measure();
            }
            const Mat3 side = across(axis);
            movePoint(a, b, ra + d, rb, side, d);
            break;
        }
        case kJointDistance: {
            const float len = length(d);
            if (len <= 0.0f) { break; }
            const Vec3 u = d / len;
            const Axis x = makeAxis(a, b, ra, rb, u);
            const float reach = reachable(a, b, x);
            if (j.limited ? j.lower >= j.upper : j.hertz == 0.0f) {
                moveAlong(a, b, x, (len - (j.limited ? j.lower : j.length)) * reach);
            } else if (j.limited && len < j.lower) {
                moveAlong(a, b, x, (len - j.lower) * reach);
            } else if (j.limited && len > j.upper) {
                moveAlong(a, b, x, (len - j.upper) * reach);
            }
            break;
        }
        default: {
            Vec3 rate;
            if (j.limited) {
                const SwingTwist st = swingTwistOf(j, a, b);
                if (twistRate(st, rate)) {
                    const Axis turn = makeTurn(a, b, rate);
                    if (st.twist < j.lower) { moveAlong(a, b, turn, st.twist - j.lower); }
                    if (st.twist > j.upper) { moveAlong(a, b, turn, st.twist - j.upper); }
                }
            }
            float error = 0.0f;
            if (!swingFree(j) && swingRoom(j, swingTwistOf(j, a, b), error, rate) && error < 0.0f) {
                moveAlong(a, b, makeTurn(a, b, rate), error);
            }
            measure();
            movePoint(a, b, ra, rb, mid(), d);
            break;
        }
    }
}

// The value a joint reports: hinge angle, slider translation, distance or twist (src/joint.cpp:592-602).
TF_HD float jointValue(const DJoint& j, const JBody& a, const JBody& b) {
    const Vec3 d = (b.com + jointArm(b, j.localB)) - (a.com + jointArm(a, j.localA));
    switch (j.type) {
        case kJointHinge: return hingeAngle(j, a, b);
        case kJointSlider: return dot(d, rotate(a.xf.q, j.axisA));
        case kJointDistance: return length(d);
        case kJointSwingTwist: return swingTwistOf(j, a, b).twist;
        default: return 0.0f;
    }
}

// A joint takes part in the step while it holds and one of its ends is an awake dynamic body
// (src/world.cpp:1623-1631).
TF_HD bool jointActive(const DJoint& j, const JBody& a, const JBody& b) {
    return j.alive && !j.broken && ((a.type == kDynamic && a.awake) || (b.type == kDynamic && b.awake));
}

}  // namespace tfb
