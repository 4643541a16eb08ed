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

#include "tf_hull.h"
#include "tf_mesh.h"
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

// ---- Prism outlines (src/shape.cpp:13-130) ----

// The polygon in counter-clockwise order (src/shape.cpp:13-18).
inline std::vector<Vec2> counterClockwise(std::vector<Vec2> poly) {
    float area = 0.0f;
    for (size_t i = 0; i < poly.size(); ++i) { area += cross(poly[i], poly[(i + 1) % poly.size()]); }
    if (area < 0.0f) { std::reverse(poly.begin(), poly.end()); }
    return poly;
}

inline bool turnsLeft(const Vec2& a, const Vec2& b, const Vec2& c, float limit) {
    return cross(b - a, c - b) > limit * length(c - a);
}

// Whether the outline winds once counter-clockwise with every corner clear of its neighbours' line
// (src/shape.cpp:30-43). The winding sums the host C library's atan2, as the reference does.
inline bool cleanOutline(const std::vector<Vec2>& poly, float limit) {
    const size_t n = poly.size();
    if (n < 3) { return false; }
    float turning = 0.0f;
    for (size_t i = 0; i < n; ++i) {
        const Vec2& a = poly[i];
        const Vec2& b = poly[(i + 1) % n];
        const Vec2& c = poly[(i + 2) % n];
        if (!turnsLeft(a, b, c, limit)) { return false; }
        turning += std::atan2(cross(b - a, c - b), dot(b - a, c - b));
    }
    return turning < 3.0f * kPiF;
}

// The convex outline of the points by a monotone chain over (x, y) order, dropping repeated and nearly
// collinear points; two points far enough apart become a thin rectangle, fewer a square around c
// (src/shape.cpp:47-69).
inline std::vector<Vec2> solidOutline(std::vector<Vec2> pts, float limit, float slab, const Vec2& c) {
    std::sort(pts.begin(), pts.end(), [](const Vec2& a, const Vec2& b) { return a.x < b.x || (a.x == b.x && a.y < b.y); });
    std::vector<Vec2> out;
    for (int pass = 0; pass < 2 && !pts.empty(); ++pass) {
        const size_t base = out.size();
        for (const Vec2& p : pts) {
            while (out.size() >= base + 2 && !turnsLeft(out[out.size() - 2], out.back(), p, limit)) { out.pop_back(); }
            out.push_back(p);
        }
        out.pop_back();
        std::reverse(pts.begin(), pts.end());
    }
    if (out.size() >= 3) { return out; }
    if (out.size() == 2 && length(out[1] - out[0]) > limit) {
        const Vec2 d = normalize(out[1] - out[0]);
        const Vec2 side = Vec2{ -d.y, d.x } * slab;
        return { out[0] - side, out[1] - side, out[1] + side, out[0] + side };
    }
    return { c + Vec2{ -slab, -slab }, c + Vec2{ slab, -slab }, c + Vec2{ slab, slab }, c + Vec2{ -slab, slab } };
}

// A prism cleaned as buildShape cleans it (src/shape.cpp:102-130): non-finite points dropped, the outline made
// counter-clockwise and replaced by its convex outline when it is not clean, no height thickened to a slab.
inline void solidPrism(std::vector<Vec2>& polygon, float& zMin, float& zMax) {
    std::vector<Vec2> pts;
    for (const Vec2& p : polygon) {
        if (std::isfinite(p.x) && std::isfinite(p.y)) { pts.push_back(p); }
    }
    if (!std::isfinite(zMin)) { zMin = 0.0f; }
    if (!std::isfinite(zMax)) { zMax = 0.0f; }
    if (zMax < zMin) { std::swap(zMin, zMax); }
    pts = counterClockwise(std::move(pts));
    Vec2 lo{ 0, 0 }, hi{ 0, 0 };
    if (!pts.empty()) { lo = hi = pts[0]; }
    for (const Vec2& p : pts) {
        lo = { std::min(lo.x, p.x), std::min(lo.y, p.y) };
        hi = { std::max(hi.x, p.x), std::max(hi.y, p.y) };
    }
    const float width = length(hi - lo);
    const float wide = std::max(std::fabs(lo.x), std::fabs(hi.x)) + std::max(std::fabs(lo.y), std::fabs(hi.y));
    const float height = zMax - zMin;
    const float size = std::sqrt(width * width + height * height);
    const float limit = thinLimit(size, wide + std::max(std::fabs(zMin), std::fabs(zMax)));
    const float slab = slabFor(size, limit);
    const float flat = thinLimit(width, wide);
    if (!cleanOutline(pts, flat)) { pts = solidOutline(std::move(pts), flat, slab, (lo + hi) * 0.5f); }
    polygon = std::move(pts);
    if (height <= limit) {
        const float mid = 0.5f * (zMin + zMax);
        zMin = mid - slab;
        zMax = mid + slab;
    }
}

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
inline bool buildShapeGeometry(HostShape& s, int geometry, float radius, const Vec3& halfExtents,
                               const float* points = nullptr, int pointCount = 0, float zMin = -0.5f, float zMax = 0.5f,
                               int maxVertices = 64, const HostMesh* mesh = nullptr, int meshId = -1,
                               float halfHeight = 0.5f) {
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
    } else if (geometry == 2 /* TF_CYLINDER */) {
        // solidCylinder (src/shape.cpp:88-95).
        d.kind = kCylinder;
        float r = solidSize(radius), h = solidSize(halfHeight);
        const float size = 2.0f * std::sqrt(r * r + h * h);
        const float limit = thinLimit(size, r + h);
        if (2.0f * r <= limit) { r = slabFor(size, limit); }
        if (2.0f * h <= limit) { h = slabFor(size, limit); }
        d.radius = r;
        d.halfHeight = h;
        d.extent = std::sqrt(r * r + h * h);
    } else if (geometry == 3 /* TF_PRISM */) {
        d.kind = kConvex;
        std::vector<Vec2> polygon;
        for (int i = 0; i < pointCount && points; ++i) { polygon.push_back({ points[2 * i], points[2 * i + 1] }); }
        solidPrism(polygon, zMin, zMax);
        s.poly = makePrism(polygon, zMin, zMax);
        s.hasPoly = true;
    } else if (geometry == 4 /* TF_HULL */) {
        d.kind = kConvex;
        std::vector<Vec3> cloud;
        for (int i = 0; i < pointCount && points; ++i) { cloud.push_back({ points[3 * i], points[3 * i + 1], points[3 * i + 2] }); }
        HullResult mesh = computeHull(cloud, maxVertices);
        if (mesh.vertices.empty()) { mesh = computeHull({ Vec3{ 0, 0, 0 } }, maxVertices); }
        s.poly = makePolyhedron(std::move(mesh.vertices), mesh.faces);
        s.hasPoly = true;
    } else if (geometry == 5 /* TF_HALFSPACE */) {
        d.kind = kHalfSpace;
        d.extent = 0.0f;
    } else if (geometry == 6 /* TF_MESH */) {
        d.kind = kMesh;
        d.extent = 0.0f;
        d.mesh = -1;
        if (mesh && !mesh->nodes.empty()) {
            for (const Vec3& v : mesh->vertices) { d.extent = std::max(d.extent, length(v)); }
            const MeshNode& root = mesh->nodes[0];
            d.centroid = (root.lo + root.hi) * 0.5f;
            d.halfExtents = (root.hi - root.lo) * 0.5f;
            d.mesh = meshId;
        }
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
    } else if (d.kind == kCylinder) {
        const float r = d.radius, h = 2.0f * d.halfHeight;
        mp.mass = s.density * kPiF * r * r * h;
        const float side = mp.mass * (3.0f * r * r + h * h) / 12.0f;
        mp.inertia = mdiag({ side, side, 0.5f * mp.mass * r * r });
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
