// Continuous collision after the substeps (src/world.cpp:1249-1419, src/distance.cpp:307-352): shapes that
// moved well past what their speculative contacts covered are swept against everything their swept bounds
// reach, and a dynamic body that hit something moves back along its sweep to the first hit, together with
// every dynamic body it hit.
//
// The reference turns sweeps with the C library's sinf, cosf and atan2f, and measures a body's turn with
// asinf. Here they are evaluated in double and rounded to float, which gives the correctly rounded value;
// where the host's float functions round the other way (their documented error reaches past half an ulp) a
// swept pose differs by one ulp.
#pragma once

#include "tf_mesh_collide.cuh"
#include "tf_planar.cuh"

namespace tfb {

TF_HD float sinRounded(float x) { return (float)sin((double)x); }
TF_HD float cosRounded(float x) { return (float)cos((double)x); }
TF_HD float atan2Rounded(float y, float x) { return (float)atan2((double)y, (double)x); }
TF_HD float asinRounded(float x) { return (float)asin((double)x); }

// A body's motion over the step: its center moves in a line, its rotation turns about one axis
// (src/internal.h:230-238).
struct Sweep {
    Vec3 localCenter;
    Vec3 c0, c1;
    Quat q0;
    Vec3 axis;
    float angle;
};

// src/distance.cpp:313-327.
TF_HD Sweep makeSweep(const Vec3& localCenter, const Vec3& c0, const Quat& q0, const Vec3& c1, const Quat& q1) {
    Sweep s;
    s.localCenter = localCenter;
    s.c0 = c0;
    s.c1 = c1;
    s.q0 = q0;
    s.axis = zero3();
    s.angle = 0.0f;
    Quat d = normalize(q1 * conjugate(q0));
    if (d.w < 0.0f) { d = -d; }
    const float sine = length(qvec(d));
    if (sine > 1.0e-7f) {
        s.axis = qvec(d) * (1.0f / sine);
        s.angle = 2.0f * atan2Rounded(sine, d.w);
    }
    return s;
}

TF_HD Sweep sweepOf(const DBody& b) { return makeSweep(b.localCenter, b.com0, b.q0, b.com, b.xf.q); }

// Quat::axisAngle (include/twofold/math.h:146-149).
TF_HD Quat axisAngle(const Vec3& axis, float angle) {
    const Vec3 a = normalize(axis) * sinRounded(0.5f * angle);
    return Quat{ a.x, a.y, a.z, cosRounded(0.5f * angle) };
}

// Sweep::at (src/distance.cpp:307-311).
TF_HD Transform sweepAt(const Sweep& s, float t) {
    const Quat q = s.angle > 0.0f ? axisAngle(s.axis, s.angle * t) * s.q0 : s.q0;
    const Vec3 c = s.c0 + (s.c1 - s.c0) * t;
    return Transform{ c - rotate(q, s.localCenter), q };
}

struct Gap {
    Vec3 normal;
    float distance;
};

// A half-space's distance to a convex shape along its normal (src/distance.cpp:175-186).
TF_HD Gap planeGap(const Transform& plane, const Convex& c, const Transform& xf) {
    const Vec3 n = rotate(plane.q, Vec3{ 0, 0, 1 });
    const Vec3 deepest = gjkSupport(c, xf, -n);
    const float height = dot(n, deepest - plane.p);
    return Gap{ n, height - c.radius };
}

// distance() from the shapes' first points (src/distance.cpp:269-305): the normal from a to b and the gap
// between the shapes, zero or less when they overlap.
TF_HD Gap gjkDistance(const Convex& a, const Transform& xa, const Convex& b, const Transform& xb) {
    if (a.halfSpace || b.halfSpace) {
        if (a.halfSpace && b.halfSpace) { return Gap{ Vec3{ 0, 0, 1 }, FLT_MAX }; }
        if (a.halfSpace) { return planeGap(xa, b, xb); }
        Gap r = planeGap(xb, a, xa);
        r.normal = -r.normal;
        return r;
    }
    Simplex s;
    Vec3 v;
    bool overlap;
    gjkSearch(a, xa, b, xb, -1.0f, s, v, overlap);
    const float gap = overlap ? 0.0f : length(v);
    Gap r;
    r.normal = gap > 0.0f ? v * (1.0f / gap) : Vec3{ 0, 0, 1 };
    r.distance = gap - a.radius - b.radius;
    return r;
}

enum ImpactKind : int { kMiss = 0, kHit = 1, kTouching = 2 };

// The first t in [0, 1] at which two swept shapes come within target of each other, by conservative
// advancement (src/distance.cpp:329-352). Reach bounds the distance from a body's center to its shape.
TF_HD int timeOfImpact(const Convex& a, const Transform& localA, const Sweep& sweepA, float reachA, const Convex& b,
                       const Transform& localB, const Sweep& sweepB, float reachB, float target, float& t) {
    const float tolerance = 0.25f * target;
    const Vec3 approach = (sweepA.c1 - sweepA.c0) - (sweepB.c1 - sweepB.c0);
    const float spin = sweepA.angle * reachA + sweepB.angle * reachB;
    t = 0.0f;
    for (int iter = 0; iter < 64; ++iter) {
        const Transform xa = sweepAt(sweepA, t) * localA, xb = sweepAt(sweepB, t) * localB;
        const Gap r = gjkDistance(a, xa, b, xb);
        if (r.distance <= target + tolerance) { return t > 0.0f ? kHit : kTouching; }
        // GJK can stop above the true distance; the gap along its normal never is.
        float gap = r.distance;
        if (!a.halfSpace && !b.halfSpace) {
            gap = minf(gap, dot(r.normal, gjkSupport(b, xb, -r.normal) - gjkSupport(a, xa, r.normal)) - a.radius - b.radius);
        }
        // No point of either shape closes the gap along the normal faster than this.
        const float closing = dot(approach, r.normal) + spin;
        if (closing <= 0.0f) { return kMiss; }
        if (gap <= target) { return t > 0.0f ? kHit : kTouching; }
        t += (gap - target) / closing;
        if (t >= 1.0f) { return kMiss; }
    }
    return kHit;
}

// src/world.cpp:1250.
TF_HD float shapeReach(const DShape& s, const DBody& b) { return length(s.local.p - b.localCenter) + s.extent; }

// Whether a shape of an awake dynamic body moved far enough over the step to be swept (src/world.cpp:1280-1292).
TF_HD bool sweepsShape(const PolyTables& pt, const DShape& s, const DBody& b, float moved, float angle) {
    if (s.kind == kMesh || s.sensor) { return false; }
    const float travel = moved + angle * shapeReach(s, b);
    return travel > b.expectedTravel && travel > b.expectedTravel + 0.5f * innerExtent(pt, s, b);
}

// Sweeps a fast shape f against shape o: first its core (a sphere of half its inner extent at its
// centroid), which decides whether it hit, then the whole shape, whose first touch is the time when it
// finds one (src/world.cpp:1341-1357). Returns whether f hit o, with the time in t.
TF_HD bool sweepAgainst(const CollideCtx& cx, const DShape& f, const DBody& bf, const Sweep& sf, const Convex& other,
                        const Transform& otherLocal, const Sweep& so, float otherReach, float target, float& t) {
    const Convex core{ &f.centroid, 1, 0.5f * innerExtent(cx.pt, f, bf), false };
    const float coreReach = length(apply(f.local, f.centroid) - bf.localCenter) + core.radius;
    float coreT = 1.0f;
    if (timeOfImpact(core, f.local, sf, coreReach, other, otherLocal, so, otherReach, target, coreT) != kHit) {
        return false;
    }
    if (timeOfImpact(convexOf(cx, f), f.local, sf, shapeReach(f, bf), other, otherLocal, so, otherReach, target, t) != kHit) {
        t = coreT;
    }
    return true;
}

// boundsInMesh (src/mesh.cpp:252-263): the box lo, hi of the world in the frame of a mesh at xm.
TF_HD void boundsInMesh(const Transform& xm, const Vec3& lo, const Vec3& hi, Vec3& meshLo, Vec3& meshHi) {
    const Vec3 c = applyInverse(xm, (lo + hi) * 0.5f);
    const Vec3 e = (hi - lo) * 0.5f;
    const Mat3 r = toMat3(conjugate(xm.q));
    Vec3 reach;
    for (int i = 0; i < 3; ++i) {
        setComp(reach, i, fabsf(r.r[i].x) * e.x + fabsf(r.r[i].y) * e.y + fabsf(r.r[i].z) * e.z);
    }
    meshLo = c - reach;
    meshHi = c + reach;
}

// Sweeps fast shape f against shape o (src/world.cpp:1341-1389): against a mesh, every triangle the tree
// finds within f's bounds over the step, from o's pose at both ends of the step, the earliest hit kept.
// Returns whether f hit o, with the time in t; false in `ok` for a tree deeper than the walk holds.
TF_HD bool sweepPair(const CollideCtx& cx, const DShape& f, const DBody& bf, const DShape& o, const DBody& bo,
                     const Vec3& sweptLo, const Vec3& sweptHi, float target, float& t, bool& ok) {
    const Sweep sf = sweepOf(bf), so = sweepOf(bo);
    ok = true;
    if (o.kind != kMesh) {
        const float otherReach = o.kind == kHalfSpace ? 0.0f : shapeReach(o, bo);
        return sweepAgainst(cx, f, bf, sf, convexOf(cx, o), o.local, so, otherReach, target, t);
    }
    if (o.mesh < 0) { return false; }
    const DMesh M = cx.mt.meshes[o.mesh];
    Vec3 lo0, hi0, lo1, hi1;
    boundsInMesh(sweepAt(so, 0.0f) * o.local, sweptLo, sweptHi, lo0, hi0);
    boundsInMesh(bo.xf * o.local, sweptLo, sweptHi, lo1, hi1);
    bool hit = false;
    t = 1.0f;
    ok = queryMesh(cx.mt, M, minVec(lo0, lo1), maxVec(hi0, hi1), [&](int tri) {
        Vec3 c[3];
        meshCorners(cx.mt, M, tri, c);
        float triReach = 0.0f;
        for (int k = 0; k < 3; ++k) { triReach = maxf(triReach, length(apply(o.local, c[k]) - bo.localCenter)); }
        float tt = 1.0f;
        const Convex triangle{ c, 3, 0.0f, false };
        if (sweepAgainst(cx, f, bf, sf, triangle, o.local, so, triReach, target, tt)) {
            t = minf(t, tt);
            hit = true;
        }
    });
    return hit;
}

}
