// Per-body and per-shape arithmetic shared by the host (scene setup) and the device (every step).
#pragma once

#include "tf_math.cuh"
#include "tf_types.cuh"

namespace tfb {

// The polyhedron tables of a batch, as device (or host) pointers.
struct PolyTables {
    const DPoly* polys;
    const Vec3* verts;
    const int32_t* indices;
    const DFace* faces;
    const Vec3* normals;
    const float* offsets;
    const DEdge* edges;
    const Vec3* arcs;
};

// The batch's triangle meshes (DMesh ranges into shared tables).
struct MeshTables {
    const DMesh* meshes;
    const Vec3* verts;
    const uint32_t* indices;
    const Vec3* normals;
    const uint8_t* edges;
    const MeshNode* nodes;
};

// Inverse of m restricted to the span of k orthonormal axes (src/world.cpp:44-60).
TF_HD Mat3 invertSubspace(const Mat3& m, const Vec3* axes, int k) {
    if (k == 0) { return mzero(); }
    if (k == 3) { return inverse(m); }
    if (k == 1) {
        const float d = dot(axes[0], m * axes[0]);
        return d > 0.0f ? outer(axes[0], axes[0]) * (1.0f / d) : mzero();
    }
    const float a = dot(axes[0], m * axes[0]);
    const float b = dot(axes[0], m * axes[1]);
    const float c = dot(axes[1], m * axes[0]);
    const float d = dot(axes[1], m * axes[1]);
    float det = a * d - b * c;
    if (det == 0.0f) { return mzero(); }
    det = 1.0f / det;
    return outer(axes[0], axes[0]) * (d * det) - outer(axes[0], axes[1]) * (b * det) -
           outer(axes[1], axes[0]) * (c * det) + outer(axes[1], axes[1]) * (a * det);
}

TF_HD bool isPlanar(const DBody& b) { return (b.locks & kLockPlanar) == kLockPlanar; }
TF_HD Vec3 planeNormal(const DBody& b) { return rotate(b.lockFrame, Vec3{ 0, 0, 1 }); }

// World-frame inverse mass and inertia on the free axes (src/world.cpp:62-92).
TF_HD void updateInverseMass(DBody& b) {
    const Mat3 lf = toMat3(b.lockFrame);
    Vec3 ang[3];
    int na = 0;
    b.linearProj = mzero();
    b.angularProj = mzero();
    for (int i = 0; i < 3; ++i) {
        const Vec3 axis = column(lf, i);
        if (!(b.locks & (kLockTX << i))) { b.linearProj = b.linearProj + outer(axis, axis); }
        if (!(b.locks & (kLockRX << i))) {
            ang[na++] = axis;
            b.angularProj = b.angularProj + outer(axis, axis);
        }
    }
    if (b.type != kDynamic || !b.awake) {
        b.invMassWorld = mzero();
        b.invInertiaWorld = mzero();
        b.planeInvMass = 0.0f;
        b.planeInvInertia = 0.0f;
        return;
    }
    b.invMassWorld = b.linearProj * b.invMass;
    const Mat3 r = toMat3(b.xf.q);
    const Mat3 iw = r * b.inertia * transpose(r);
    b.invInertiaWorld = invertSubspace(iw, ang, na);
    if (isPlanar(b)) {
        const Vec3 n = planeNormal(b);
        b.planeInvMass = b.invMass;
        b.planeInvInertia = dot(n, b.invInertiaWorld * n);
    }
}

// The part of updateInverseMass that a new pose changes: the world inverse inertia on the free rotation axes
// and, for a body locked to a plane, its inverse inertia about the plane normal; the projections and the world
// inverse mass depend only on the locks and come out as they were. The same operations as updateInverseMass,
// so the same bits. For awake dynamic bodies.
TF_HD void updateInverseInertia(DBody& b) {
    const Mat3 lf = toMat3(b.lockFrame);
    Vec3 ang[3];
    int na = 0;
    for (int i = 0; i < 3; ++i) {
        if (!(b.locks & (kLockRX << i))) { ang[na++] = column(lf, i); }
    }
    const Mat3 r = toMat3(b.xf.q);
    const Mat3 iw = r * b.inertia * transpose(r);
    b.invInertiaWorld = invertSubspace(iw, ang, na);
    if (isPlanar(b)) {
        const Vec3 n = planeNormal(b);
        b.planeInvInertia = dot(n, b.invInertiaWorld * n);
    }
}

// src/world.cpp:94-98.
TF_HD bool movingAwake(const DBody& b) {
    if (b.type == kDynamic) { return b.awake != 0; }
    if (b.type == kKinematic) { return lengthSquared(b.v) > 0.0f || lengthSquared(b.w) > 0.0f; }
    return false;
}

TF_HD bool movingBody(const DBody& b) { return b.type == kDynamic && b.awake; }

// Scales down the velocities of an awake dynamic body past the speed limits (src/solver.cpp:30-41).
template <class BodyT>
TF_HD void limitSpeed(BodyT& b, float maxSpeed, float maxSpin) {
    if (b.type != kDynamic || !b.awake) { return; }
    const float speed = length(b.v), spin = length(b.w);
    if (speed > maxSpeed) {
        b.v = b.v * (maxSpeed / speed);
        b.kept = minf(b.kept, maxSpeed / speed);
    }
    if (spin > maxSpin) {
        b.w = b.w * (maxSpin / spin);
        b.kept = minf(b.kept, maxSpin / spin);
    }
}

// How far two bodies can travel toward each other over dt (src/world.cpp:493-495).
TF_HD float relativeTravel(const DBody& a, const DBody& b, float dt) {
    return (length(b.v - a.v) + length(a.w) * a.extent + length(b.w) * b.extent) * dt;
}

// src/shape.cpp:134-140: the half extents of a cylinder turned so its axis is `axis`.
TF_HD Vec3 cylinderReach(const Vec3& axis, float radius, float halfHeight) {
    Vec3 r;
    for (int i = 0; i < 3; ++i) {
        const float a = comp(axis, i);
        setComp(r, i, halfHeight * fabsf(a) + radius * sqrtf(maxf(1.0f - a * a, 0.0f)));
    }
    return r;
}

// World bounds of a shape at transform xf (src/shape.cpp:227-295). Boxes and prisms take the reach of their
// outline and depth; hulls their vertices.
TF_HD void shapeBounds(const DShape& s, const PolyTables& pt, const Transform& xf, Vec3& lo, Vec3& hi) {
    if (s.kind == kHalfSpace) {
        const float big = 3.0e38f;
        lo = { -big, -big, -big };
        hi = { big, big, big };
        return;
    }
    if (s.kind == kSphere) {
        const Vec3 r{ s.radius, s.radius, s.radius };
        lo = xf.p - r;
        hi = xf.p + r;
        return;
    }
    if (s.kind == kCylinder) {
        const Vec3 r = cylinderReach(rotate(xf.q, Vec3{ 0, 0, 1 }), s.radius, s.halfHeight);
        lo = xf.p - r;
        hi = xf.p + r;
        return;
    }
    const Mat3 r = toMat3(xf.q);
    if (s.kind == kMesh) {
        // The mesh's root box turned into the world.
        if (s.mesh < 0) {
            lo = hi = xf.p;
            return;
        }
        const Vec3 c = apply(xf, s.centroid);
        const Vec3 e = s.halfExtents;
        Vec3 reach;
        for (int i = 0; i < 3; ++i) {
            setComp(reach, i, fabsf(r.r[i].x) * e.x + fabsf(r.r[i].y) * e.y + fabsf(r.r[i].z) * e.z);
        }
        lo = c - reach;
        hi = c + reach;
        return;
    }
    const DPoly& P = pt.polys[s.poly];
    const Vec3* v = pt.verts + P.vFirst;
    if (s.geometry == 1 /* box */ || s.geometry == 3 /* prism */) {
        // The first half of a prism's vertices is its outline at zMin, the second half at zMax.
        const int count = P.vCount / 2;
        const float zMin = v[0].z, zMax = v[count].z;
        for (int i = 0; i < 3; ++i) {
            const Vec3& row = r.r[i];
            float nearV = FLT_MAX, farV = -FLT_MAX;
            for (int k = 0; k < count; ++k) {
                const float x = row.x * v[k].x + row.y * v[k].y;
                nearV = nearV < x ? nearV : x;
                farV = farV > x ? farV : x;
            }
            const float z0 = row.z * zMin, z1 = row.z * zMax;
            setComp(lo, i, nearV + (z0 < z1 ? z0 : z1) + comp(xf.p, i));
            setComp(hi, i, farV + (z0 > z1 ? z0 : z1) + comp(xf.p, i));
        }
        return;
    }
    lo = hi = r * v[0] + xf.p;
    for (int k = 0; k < P.vCount; ++k) {
        const Vec3 w = r * v[k] + xf.p;
        lo = minVec(lo, w);
        hi = maxVec(hi, w);
    }
}

TF_HD bool boxesOverlap(const Vec3& loA, const Vec3& hiA, const Vec3& loB, const Vec3& hiB) {
    return loA.x <= hiB.x && loB.x <= hiA.x && loA.y <= hiB.y && loB.y <= hiA.y && loA.z <= hiB.z && loB.z <= hiA.z;
}

}
