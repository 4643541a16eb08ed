// Host-side shape building: the setup that runs once per shape, not per step.
//
// Restates the reference's buildShape/shapeMass (src/shape.cpp:149-225), makePolyhedron/makePrism/makeBox/
// polyhedronMass (src/polyhedron.cpp:8-112) and World::Impl::updateMass (src/world.cpp:439-479) with the same
// float operations in the same order, so the masses, inertias and polyhedra the device steps with are
// bit-identical to the reference's. Everything here is host code compiled without contraction.
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <utility>
#include <vector>

#include "tf_math.cuh"
#include "tf_types.cuh"

namespace tfb {

struct HostPoly {
    std::vector<Vec3> vertices;
    std::vector<int32_t> indices;
    std::vector<DFace> faces;
    std::vector<Vec3> normals;
    std::vector<float> offsets;
    std::vector<DEdge> edges;
    std::vector<Vec3> arcs;
    Vec3 centroid{ 0, 0, 0 };
    Vec3 lo{ 0, 0, 0 }, hi{ 0, 0, 0 };
};

struct MassProps {
    float mass = 0.0f;
    Vec3 center{ 0, 0, 0 };
    Mat3 inertia = mzero();
};

// Polyhedron from vertex loops, counter-clockwise seen from outside (src/polyhedron.cpp:8-61). Normals by
// Newell's method about the centroid; edges in ascending (v0, v1) order with v0 < v1, each twinned.
inline HostPoly makePolyhedron(std::vector<Vec3> vertices, const std::vector<std::vector<int>>& faces) {
    HostPoly p;
    p.vertices = std::move(vertices);
    Vec3 c{ 0, 0, 0 };
    for (const Vec3& v : p.vertices) { c += v; }
    p.centroid = c;
    if (!p.vertices.empty()) {
        p.centroid = p.centroid / (float)p.vertices.size();
        p.lo = p.hi = p.vertices[0];
    }
    for (const Vec3& v : p.vertices) {
        p.lo = minVec(p.lo, v);
        p.hi = maxVec(p.hi, v);
    }
    // (from, to) -> face of each directed edge; sorted like an ordered map keyed by (from, to).
    std::vector<std::pair<std::pair<int, int>, int>> directed;
    for (const std::vector<int>& loop : faces) {
        if (loop.size() < 3) { continue; }
        DFace f;
        f.first = (int)p.indices.size();
        f.count = (int)loop.size();
        Vec3 n{ 0, 0, 0 };
        for (int i = 0; i < f.count; ++i) {
            const Vec3 a = p.vertices[loop[i]] - p.centroid;
            const Vec3 b = p.vertices[loop[(i + 1) % f.count]] - p.centroid;
            n.x += (a.y - b.y) * (a.z + b.z);
            n.y += (a.z - b.z) * (a.x + b.x);
            n.z += (a.x - b.x) * (a.y + b.y);
        }
        p.normals.push_back(normalize(n));
        p.offsets.push_back(dot(p.normals.back(), p.vertices[loop[0]]));
        const int fi = (int)p.faces.size();
        for (int i = 0; i < f.count; ++i) {
            p.indices.push_back(loop[i]);
            const std::pair<int, int> key{ loop[i], loop[(i + 1) % f.count] };
            auto it = std::find_if(directed.begin(), directed.end(), [&](const auto& e) { return e.first == key; });
            if (it != directed.end()) {
                it->second = fi;  // a repeated directed edge keeps the last face, as map assignment does
            } else {
                directed.push_back({ key, fi });
            }
        }
        p.faces.push_back(f);
    }
    std::sort(directed.begin(), directed.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    for (const auto& e : directed) {
        const int a = e.first.first, b = e.first.second;
        if (a > b) { continue; }
        auto twin = std::lower_bound(directed.begin(), directed.end(), std::make_pair(std::make_pair(b, a), INT32_MIN),
                                     [](const auto& x, const auto& y) { return x.first < y.first; });
        if (twin == directed.end() || twin->first != std::make_pair(b, a)) { continue; }
        DEdge edge;
        edge.v0 = a;
        edge.v1 = b;
        edge.f0 = e.second;
        edge.f1 = twin->second;
        edge.length = length(p.vertices[b] - p.vertices[a]);
        p.edges.push_back(edge);
        p.arcs.push_back(cross(p.normals[edge.f1], p.normals[edge.f0]));
    }
    return p;
}

// Prism over a counter-clockwise polygon (src/polyhedron.cpp:63-82).
inline HostPoly makePrism(const std::vector<Vec2>& polygon, float zMin, float zMax) {
    const int n = (int)polygon.size();
    std::vector<Vec3> verts;
    verts.reserve(2 * n);
    for (const Vec2& v : polygon) { verts.push_back({ v.x, v.y, zMin }); }
    for (const Vec2& v : polygon) { verts.push_back({ v.x, v.y, zMax }); }
    std::vector<std::vector<int>> faces;
    std::vector<int> top, bottom;
    for (int i = 0; i < n; ++i) {
        top.push_back(n + i);
        bottom.push_back(n - 1 - i);
        const int j = (i + 1) % n;
        faces.push_back({ i, j, n + j, n + i });
    }
    faces.push_back(top);
    faces.push_back(bottom);
    return makePolyhedron(std::move(verts), faces);
}

inline HostPoly makeBox(const Vec3& h) {
    return makePrism({ { -h.x, -h.y }, { h.x, -h.y }, { h.x, h.y }, { -h.x, h.y } }, -h.z, h.z);
}

// Mass, center and inertia about the center by the divergence theorem over fan triangles
// (src/polyhedron.cpp:84-112).
inline MassProps polyhedronMass(const HostPoly& poly, float density) {
    MassProps mp;
    const Vec3 ref = poly.centroid;
    float volume = 0.0f;
    Vec3 center{ 0, 0, 0 };
    Mat3 cov = mzero();
    for (const DFace& f : poly.faces) {
        const Vec3 a = poly.vertices[poly.indices[f.first]] - ref;
        for (int i = 1; i + 1 < f.count; ++i) {
            const Vec3 b = poly.vertices[poly.indices[f.first + i]] - ref;
            const Vec3 c = poly.vertices[poly.indices[f.first + i + 1]] - ref;
            const float det = dot(a, cross(b, c));
            volume += det / 6.0f;
            center += (a + b + c) * (det / 24.0f);
            const Vec3 s = a + b + c;
            cov = cov + (outer(a, a) + outer(b, b) + outer(c, c) + outer(s, s)) * (det / 120.0f);
        }
    }
    if (volume <= 0.0f) { return mp; }
    center = center / volume;
    mp.mass = density * volume;
    const Mat3 cc = cov * density - outer(center, center) * mp.mass;
    const float tr = cc.r[0].x + cc.r[1].y + cc.r[2].z;
    mp.inertia = mdiag({ tr, tr, tr }) - cc;
    mp.center = center + ref;
    return mp;
}

// Below this a box side is treated as having no length (src/shape.cpp:22).
inline float thinLimit(float size, float reach) { return std::max({ 1e-6f * size, 3.0f * FLT_EPSILON * reach, 1e-8f }); }
inline float slabFor(float size, float limit) { return std::max({ 0.005f * size, 1e-4f, 10.0f * limit }); }
inline float solidSize(float s) { return std::isfinite(s) ? std::fabs(s) : 0.0f; }

// src/shape.cpp:80-90.
inline Vec3 solidBox(Vec3 h) {
    for (int k = 0; k < 3; ++k) { setComp(h, k, std::isfinite(comp(h, k)) ? std::fabs(comp(h, k)) : 0.0f); }
    const float size = 2.0f * length(h);
    const float limit = thinLimit(size, h.x + h.y + h.z);
    for (int k = 0; k < 3; ++k) {
        if (2.0f * comp(h, k) <= limit) { setComp(h, k, slabFor(size, limit)); }
    }
    return h;
}

// src/shape.cpp:93-97.
inline float solidRadius(float r) {
    r = solidSize(r);
    const float limit = thinLimit(2.0f * r, r);
    return 2.0f * r <= limit ? slabFor(2.0f * r, limit) : r;
}

constexpr float kPiF = 3.14159265358979f;

// The built form of one shape: the device record plus its polyhedron (empty for spheres and half-spaces).
struct HostShape {
    DShape d{};
    HostPoly poly;
    float density = 1.0f;
    bool hasPoly = false;
    uint32_t generation = 0;
};

// Shape kind, cleaned size, polyhedron, extent, centroid and minExtent (src/shape.cpp:149-202). Returns
// false for geometry this build does not make.
inline bool buildShapeGeometry(HostShape& s, int geometry, float radius, const Vec3& halfExtents) {
    DShape& d = s.d;
    d.radius = 0.0f;
    d.halfHeight = 0.0f;
    d.centroid = { 0, 0, 0 };
    s.poly = HostPoly{};
    s.hasPoly = false;
    d.geometry = (uint32_t)geometry;
    if (geometry == 0 /* TF_SPHERE */) {
        d.kind = kSphere;
        d.radius = solidRadius(radius);
        d.extent = d.radius;
    } else if (geometry == 1 /* TF_BOX */) {
        d.kind = kConvex;
        d.halfExtents = solidBox(halfExtents);
        s.poly = makeBox(d.halfExtents);
        s.hasPoly = true;
    } else if (geometry == 5 /* TF_HALFSPACE */) {
        d.kind = kHalfSpace;
        d.extent = 0.0f;
    } else {
        return false;
    }
    d.minExtent = d.kind == kCylinder ? std::min(d.radius, d.halfHeight) : d.radius;
    if (d.kind == kConvex) {
        float e = 0.0f;
        for (const Vec3& v : s.poly.vertices) { e = std::max(e, length(v)); }
        d.extent = e;
        d.centroid = s.poly.centroid;
        d.minExtent = e;
        for (size_t i = 0; i < s.poly.faces.size(); ++i) {
            d.minExtent = std::min(d.minExtent, s.poly.offsets[i] - dot(s.poly.normals[i], d.centroid));
        }
    }
    return true;
}

// src/shape.cpp:204-225.
inline MassProps shapeMass(const HostShape& s) {
    MassProps mp;
    const DShape& d = s.d;
    if (d.geometry == 0 /* sphere */) {
        const float r = d.radius;
        mp.mass = s.density * (4.0f / 3.0f) * kPiF * r * r * r;
        const float i = 0.4f * mp.mass * r * r;
        mp.inertia = mdiag({ i, i, i });
    } else if (d.kind == kConvex) {
        mp = polyhedronMass(s.poly, s.density);
    } else {
        return mp;
    }
    const Mat3 r = toMat3(d.local.q);
    mp.inertia = r * mp.inertia * transpose(r);
    mp.center = apply(d.local, mp.center);
    return mp;
}

}
