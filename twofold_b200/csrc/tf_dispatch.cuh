// Shape-kind dispatch of one pair (src/collide3d.cpp:1778-1811) with the half-space collisions
// (:1309-1345), over the pair classes the flat collision kernels are instantiated for. Cylinder pairs other
// than with a half-space go to the convex class.
#pragma once

#include "tf_round.cuh"

namespace tfb {

// Normal out of the half-space (src/collide3d.cpp:1309-1345).
TF_HD void collideHalfSpace(const CollideCtx& cx, const Transform& xh, const DShape& other, const Transform& xo,
                            float margin, float band, const Motion& motion, Manifold& m) {
    const Vec3 n = rotate(xh.q, Vec3{ 0, 0, 1 });
    const float offset = dot(n, xh.p);
    if (other.kind == kSphere) {
        const float d = dot(n, xo.p) - offset;
        const float sep = d - other.radius;
        if (sep > margin) { return; }
        m.normal = n;
        m.points[0] = { xo.p - n * (0.5f * (d + other.radius)), sep, 0.0f };
        m.count = 1;
        return;
    }
    if (other.kind == kCylinder) {
        Vec3 feature[kMaxFeature];
        Vec3 unused = zero3();
        const int nf = featureAlong(cx.cap, cylinderSolid(other, xo), -n, band, feature, unused);
        MPoint pts[kMaxFeature];
        int np = 0;
        for (int k = 0; k < nf; ++k) {
            const Vec3 w = feature[k];
            const float s = dot(n, w) - offset;
            if (s > margin) { continue; }
            pts[np++] = { w - n * (0.5f * s), s, motion.predict(w, n, s) };
        }
        reduceManifold(pts, np, n, band, m, 0.5f * band, motion.fast);
        return;
    }
    const Vec3 localN = unrotate(xo.q, n);
    const float localOffset = offset - dot(n, xo.p);
    const DPoly& P = cx.pt.polys[other.poly];
    MPoint pts[kMaxReduce];
    int np = 0;
    for (int k = 0; k < P.vCount && np < kMaxReduce; ++k) {
        const Vec3 v = cx.pt.verts[P.vFirst + k];
        const float s = dot(localN, v) - localOffset;
        if (s > margin) { continue; }
        const Vec3 w = apply(xo, v);
        pts[np++] = { w - n * (0.5f * s), s, motion.predict(w, n, s) };
    }
    reduceManifold(pts, np, n, band, m, 0.0f, motion.fast);
}

// Pair classes, by shape kinds. A kernel instantiated for one class compiles only that class's collision
// code; kClassAny compiles every path.
// kClassPlanar holds the pairs solved in a plane (decided by their bodies, not their shapes); its kernels
// fall back to every 3D path for profiles the plane does not cut.
// kClassMesh holds the pairs with a triangle mesh, which may make several contacts.
enum PairClass : int {
    kClassAny = -1, kClassSpheres = 0, kClassSpherePoly = 1, kClassPlane = 2, kClassConvex = 3, kClassPlanar = 4,
    kClassMesh = 5
};
constexpr int kPairClasses = 6;

TF_HD int pairClass(uint32_t ka, uint32_t kb) {
    if (ka == kHalfSpace || kb == kHalfSpace) { return kClassPlane; }
    if (ka == kCylinder || kb == kCylinder) { return kClassConvex; }
    if (ka == kSphere && kb == kSphere) { return kClassSpheres; }
    if (ka == kSphere || kb == kSphere) { return kClassSpherePoly; }
    return kClassConvex;
}

// Shape-kind dispatch (src/collide3d.cpp:1778-1811). Returns false for a mesh pair (collided by
// collideMesh), leaving m empty. For a class other than kClassAny the pair must be of that class.
template <int Cls = kClassAny>
TF_HD bool collideShapes(const CollideCtx& cx, const DShape& a, const Transform& xa, const DShape& b,
                         const Transform& xb, float margin, const Motion& motion, Manifold& m, int reuseKind,
                         int reuseA, int reuseB) {
    m.count = 0;
    m.featKind = kFeatNone;
    m.featA = m.featB = -1;
    m.normal = zero3();
    const uint32_t ka = a.kind, kb = b.kind;
    if (ka == kHalfSpace && kb == kHalfSpace) { return true; }
    if (ka == kMesh || kb == kMesh) { return false; }
    if constexpr (Cls == kClassAny || Cls == kClassPlane) {
        if (ka == kHalfSpace) {
            collideHalfSpace(cx, xa, b, xb, margin, cx.tol.linearSlop, motion, m);
            return true;
        }
        if (kb == kHalfSpace) {
            collideHalfSpace(cx, xb, a, xa, margin, cx.tol.linearSlop, motion.swapped(), m);
            m.normal = -m.normal;
            return true;
        }
    }
    if constexpr (Cls == kClassAny || Cls == kClassSpheres) {
        if (ka == kSphere && kb == kSphere) {
            collideSpheres(xa.p, a.radius, xb.p, b.radius, margin, m);
            return true;
        }
    }
    if constexpr (Cls == kClassAny || Cls == kClassSpherePoly) {
        if (ka == kSphere && kb != kCylinder) {
            collideSpherePoly(cx, b, xb, xa.p, a.radius, margin, m);
            m.normal = -m.normal;
            return true;
        }
        if (kb == kSphere && ka != kCylinder) {
            collideSpherePoly(cx, a, xa, xb.p, b.radius, margin, m);
            return true;
        }
    }
    if constexpr (Cls == kClassAny || Cls == kClassConvex) {
        if (ka == kSphere) {
            collideSphereCylinder(b, xb, xa.p, a.radius, margin, m);
            m.normal = -m.normal;
        } else if (kb == kSphere) {
            collideSphereCylinder(a, xa, xb.p, b.radius, margin, m);
        } else if (ka == kCylinder || kb == kCylinder) {
            collideRound(cx, a, xa, b, xb, margin, motion, m);
        } else {
            collideConvex(cx, a, xa, b, xb, margin, motion, m, reuseKind, reuseA, reuseB);
        }
    }
    return true;
}


}
