// A sphere or polyhedron against a triangle mesh (src/collide3d.cpp:1386-1488, 1577-1776): every triangle
// the tree finds near the other shape is collided as a two-faced polyhedron (or by its closest point, for a
// sphere), a contact on an edge or corner without a normal of its own is pushed along the face instead, and
// triangle manifolds whose normals agree within kSameNormal merge into one manifold per group.
#pragma once

#include "tf_round.cuh"

namespace tfb {

constexpr float kSameNormal = 0.996f;  // src/collide3d.cpp:1348
constexpr int kMaxMeshFound = 64;      // triangle manifolds of one pair
constexpr int kMaxMeshParts = 16;      // grouped manifolds of one pair
constexpr int kMaxMeshBounds = 128;    // triangles one fast pair rules out by distance
constexpr int kMeshStack = 64;         // tree walk, as src/internal.h:70

// Why a mesh pair could not be collided as the reference collides it.
constexpr int kMeshOk = 0, kMeshTooMany = 1, kMeshUnsupported = 2;

// A mesh triangle found no nearer to the other shape than distance (src/internal.h:386-389).
struct TriangleBound {
    int32_t triangle;
    float distance;
};

// Triangles ruled out by distance go to found (when recording); those in known, sorted by triangle, are
// skipped while their distance less moved stays past the margin (src/internal.h:391-398).
struct MeshBounds {
    TriangleBound* found;
    int foundCount;
    const TriangleBound* known;
    int knownCount;
    float moved;
};

// The edge or corner of the triangle farthest along d, numbered as above: the edge when its far corner is
// within tolerance (src/collide3d.cpp:1437-1443).
TF_HD int triangleFeature(const Vec3 c[3], const Vec3& d, float tolerance) {
    const float h[3] = { dot(c[0], d), dot(c[1], d), dot(c[2], d) };
    const int top = h[1] > h[0] ? (h[2] > h[1] ? 2 : 1) : (h[2] > h[0] ? 2 : 0);
    const int next = (top + 1) % 3, prev = (top + 2) % 3;
    if (h[next] >= h[prev]) { return h[next] >= h[top] - tolerance ? 3 + top : top; }
    return h[prev] >= h[top] - tolerance ? 3 + prev : top;
}

// Whether p lies over the triangle along its normal n, within tolerance of its edges (src/collide3d.cpp:1446-1452).
TF_HD bool overTriangle(const Vec3 c[3], const Vec3& n, const Vec3& p, float tolerance) {
    for (int k = 0; k < 3; ++k) {
        const Vec3 e = c[(k + 1) % 3] - c[k];
        if (dot(cross(e, n), p - c[k]) > tolerance * length(e)) { return false; }
    }
    return true;
}

// Whether a contact on the feature may keep a normal other than the face's, seen from side 0 (front) or 1
// (src/collide3d.cpp:1455-1460).
TF_HD bool ownNormal(uint8_t edges, int feature, int side) {
    const int shift = 3 * side;
    if (feature >= 3 && feature < 6) { return (edges >> (shift + feature - 3)) & 1; }
    if (feature < 3) { return ((edges >> (shift + feature)) & 1) || ((edges >> (shift + (feature + 2) % 3)) & 1); }
    return true;
}

// src/collide3d.cpp:1464-1466.
TF_HD bool keepsNormal(uint8_t edges, int feature, int side, const Vec3& normal, const Vec3& n) {
    return ownNormal(edges, feature, side) || ownNormal(edges, feature, dot(normal, n) >= 0.0f ? 0 : 1);
}

// src/collide3d.cpp:1468-1474.
TF_HD bool outOfReach(const MeshBounds* bounds, int t, float margin) {
    if (!bounds || bounds->knownCount == 0) { return false; }
    int lo = 0, hi = bounds->knownCount;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (bounds->known[mid].triangle < t) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo < bounds->knownCount && bounds->known[lo].triangle == t && bounds->known[lo].distance - bounds->moved > margin;
}

// src/collide3d.cpp:1476-1478.
TF_HD void ruleOut(MeshBounds* bounds, int t, float distance, int& status) {
    if (!bounds || !bounds->found) { return; }
    if (bounds->foundCount >= kMaxMeshBounds) {
        status = kMeshTooMany;
        return;
    }
    bounds->found[bounds->foundCount++] = TriangleBound{ t, distance };
}

// A triangle as a polyhedron with a front and a back face, so the face queries and clipping of polyhedra
// apply (src/collide3d.cpp:1350-1381). Its tables point into the struct: build it in place, never copy it.
struct TriangleFrame {
    DPoly poly;
    Vec3 verts[3];
    Vec3 normals[2];
    float offsets[2];
    DFace faces[2];
    int32_t indices[6];
    DEdge edges[3];
    PolyTables t;

    TF_HD void set(const Vec3 c[3], const Vec3& n) {
        for (int k = 0; k < 3; ++k) {
            verts[k] = c[k];
            edges[k] = DEdge{ k, (k + 1) % 3, 0, 1, length(c[(k + 1) % 3] - c[k]) };
        }
        normals[0] = n;
        normals[1] = -n;
        offsets[0] = dot(n, c[0]);
        offsets[1] = -offsets[0];
        faces[0] = DFace{ 0, 3 };
        faces[1] = DFace{ 3, 3 };
        const int32_t loop[6] = { 0, 1, 2, 0, 2, 1 };
        for (int k = 0; k < 6; ++k) { indices[k] = loop[k]; }
        poly = DPoly{ 0, 3, 0, 2, 0, 3, 0, 6, (c[0] + c[1] + c[2]) * (1.0f / 3.0f), minVec(minVec(c[0], c[1]), c[2]),
                      maxVec(maxVec(c[0], c[1]), c[2]) };
        t = PolyTables{ &poly, verts, indices, faces, normals, offsets, edges, nullptr };
    }
};

// Edge queries against a triangle a: a triangle edge's arc on the Gauss map is the half circle from the
// front normal through the edge's outward direction to the back normal (src/collide3d.cpp:1386-1433).
TF_HD EdgeQuery queryTriangleEdges(const FramePoly& a, const FramePoly& b, float reach) {
    EdgeQuery q = noEdge();
    const Vec3 grow{ reach, reach, reach };
    uint8_t past[kMaxVerts];
    int16_t nearB[kMaxEdges];
    const int nb = edgesInBox(b, maxVec(a.lo, b.lo) - grow, minVec(a.hi, b.hi) + grow, past, nearB);
    q.pruned = nb < b.edgeCount();
    const Vec3 n = a.n(0);
    for (int k = 0; k < 3; ++k) {
        const Vec3 pa = a.v(k);
        const Vec3 e = a.v((k + 1) % 3) - pa;
        const Vec3 out = cross(e, n);
        const float lengthA = a.edge(k).length;
        for (int y = 0; y < nb; ++y) {
            const int j = nearB[y];
            const DEdge eb = b.edge(j);
            const Vec3 u = b.n(eb.f0), v = b.n(eb.f1);
            const float du = dot(u, e), dv = dot(v, e);
            const float facing = dot(u * dv - v * du, out);
            if (!((0.0f > du * dv) && (0.0f > (dv > 0.0f ? facing : -facing)))) { continue; }
            // Where b's arc crosses the plane of a's arc; the pair forms a face when a's normal there points
            // the opposite way.
            const Vec3 p = (u * dv - v * du) * (dv > 0.0f ? 1.0f : -1.0f);
            const Vec3 pb = b.v(eb.v0);
            Vec3 axis = cross(e, b.v(eb.v1) - pb);
            const float len = length(axis);
            if (len < kParallelEdges * lengthA * eb.length) { continue; }
            axis = axis / len;
            if (dot(axis, p) > 0.0f) { axis = -axis; }
            const float s = dot(axis, pb - pa);
            if (s > q.separation) {
                q.separation = s;
                q.a = k;
                q.b = j;
                q.axis = axis;
            }
        }
    }
    return q;
}

// Visits the triangles of mesh M whose tree boxes meet lo, hi, in the tree's order (src/internal.h:67-86).
template <class Visit>
TF_HD bool queryMesh(const MeshTables& mt, const DMesh& M, const Vec3& lo, const Vec3& hi, Visit&& visit) {
    if (M.nCount == 0) { return true; }
    int stack[kMeshStack];
    int top = 0;
    stack[top++] = 0;
    while (top > 0) {
        const MeshNode n = mt.nodes[M.nFirst + stack[--top]];
        if (n.lo.x > hi.x || n.hi.x < lo.x || n.lo.y > hi.y || n.hi.y < lo.y || n.lo.z > hi.z || n.hi.z < lo.z) {
            continue;
        }
        if (n.count > 0) {
            for (int t = n.first; t < n.first + n.count; ++t) { visit(t); }
        } else {
            if (top + 2 > kMeshStack) { return false; }
            stack[top++] = n.first + 1;
            stack[top++] = n.first;
        }
    }
    return true;
}

TF_HD void meshCorners(const MeshTables& mt, const DMesh& M, int t, Vec3 c[3]) {
    const uint32_t* idx = mt.indices + 3 * (size_t)(M.tFirst + t);
    for (int k = 0; k < 3; ++k) { c[k] = mt.verts[M.vFirst + (int)idx[k]]; }
}

// What one triangle of a mesh pair gives: nothing, a manifold, or a distance that rules it out.
constexpr int kTriNone = 0, kTriKept = 1, kTriRuledOut = 2;

// Collects a pair's triangle results on one thread, in the tree's visiting order: kept manifolds into found (at
// most kMaxMeshFound; one more makes the pair kMeshTooMany), ruled-out distances into bounds when it records.
struct SerialCollect {
    Manifold* found;
    int nFound;
    MeshBounds* bounds;
    int status;

    template <class Tri>
    TF_HD bool operator()(const MeshTables& mt, const DMesh& M, const Vec3& lo, const Vec3& hi, Tri&& tri) {
        return queryMesh(mt, M, lo, hi, [&](int t) {
            Manifold m;
            float d = 0.0f;
            const int r = tri(t, m, d);
            if (r == kTriKept) {
                if (nFound >= kMaxMeshFound) {
                    status = kMeshTooMany;
                } else {
                    found[nFound++] = m;
                }
            } else if (r == kTriRuledOut) {
                ruleOut(bounds, t, d, status);
            }
        });
    }
};

#if defined(__CUDACC__)
// The same results with a warp's lanes over the triangles: every lane walks the tree alike (the same nodes, so
// the loads are broadcast), the triangles it finds are dealt to the lanes in visiting order, and each full hand
// of 32 is collided at once; ballots place the kept manifolds (in found, shared by the warp) and the ruled-out
// triangles (in bounds->found) in visiting order, as the serial walk stores them. Every lane's nFound, status
// and bounds count come out equal.
struct WarpCollect {
    Manifold* found;
    int nFound;
    MeshBounds* bounds;
    int status;
    uint32_t lane;

    template <class Tri>
    __device__ bool operator()(const MeshTables& mt, const DMesh& M, const Vec3& lo, const Vec3& hi, Tri&& tri) {
        int mine = -1, dealt = 0;
        const uint32_t below = (1u << lane) - 1u;
        auto collide = [&]() {
            Manifold m;
            float d = 0.0f;
            const int r = mine >= 0 ? tri(mine, m, d) : kTriNone;
            const uint32_t kept = __ballot_sync(0xffffffffu, r == kTriKept);
            if (r == kTriKept) {
                const int pos = nFound + __popc(kept & below);
                if (pos < kMaxMeshFound) { found[pos] = m; }
            }
            nFound += __popc(kept);
            if (bounds && bounds->found) {
                const uint32_t ruled = __ballot_sync(0xffffffffu, r == kTriRuledOut);
                if (r == kTriRuledOut) {
                    const int pos = bounds->foundCount + __popc(ruled & below);
                    if (pos < kMaxMeshBounds) { bounds->found[pos] = TriangleBound{ mine, d }; }
                }
                bounds->foundCount += __popc(ruled);
            }
            __syncwarp();
            mine = -1;
            dealt = 0;
        };
        const bool walked = queryMesh(mt, M, lo, hi, [&](int t) {
            if ((int)lane == dealt) { mine = t; }
            if (++dealt == 32) { collide(); }
        });
        if (dealt > 0) { collide(); }
        if (nFound > kMaxMeshFound) {
            status = kMeshTooMany;
            nFound = kMaxMeshFound;
        }
        if (bounds && bounds->found && bounds->foundCount > kMaxMeshBounds) {
            status = kMeshTooMany;
            bounds->foundCount = kMaxMeshBounds;
        }
        return walked;
    }
};
#endif

// collideMesh (src/collide3d.cpp:1577-1776) for a sphere or polyhedron, up to grouping: every triangle the tree
// finds near the other shape collided, its result handed to collect in visiting order. Returns kMeshOk, or
// why the pair could not be collided exactly.
template <class Collect>
TF_HD int collideMeshTriangles(const CollideCtx& cx, const DShape& mesh, const Transform& xm, const DShape& other,
                               const Transform& xo, float margin, const Motion& motion, const MeshBounds* bounds,
                               Collect& collect) {
    if (mesh.mesh < 0 || other.kind == kHalfSpace || other.kind == kMesh) { return kMeshOk; }
    const MeshTables& mt = cx.mt;
    const DMesh M = mt.meshes[mesh.mesh];
    const Tolerances tol = cx.tol;
    const Transform rel{ unrotate(xm.q, xo.p - xm.p), conjugate(xm.q) * xo.q };
    const float absTol = 0.5f * tol.linearSlop;
    bool walked;
    if (other.kind == kSphere) {
        const Vec3 center = rel.p;
        const float r = other.radius;
        const Vec3 reach{ r + margin, r + margin, r + margin };
        walked = collect(mt, M, center - reach, center + reach, [&](int t, Manifold& m, float& ruledAt) {
            if (outOfReach(bounds, t, margin)) { return kTriNone; }
            Vec3 c[3];
            meshCorners(mt, M, t, c);
            const Vec3 n = mt.normals[M.tFirst + t];
            int feature;
            const Vec3 q = closestOnTriangle(c, center, feature);
            const float h = dot(n, center - c[0]);
            const int side = h >= 0.0f ? 0 : 1;
            const float dist = length(center - q);
            Vec3 normal, surface;
            float sep;
            const bool own = feature != 6 && dist > 0.0f && ownNormal(mt.edges[M.tFirst + t], feature, side);
            if (!own && dist - fabsf(h) > tol.linearSlop) { return kTriNone; }
            if (!own) {
                normal = side == 0 ? n : -n;
                sep = fabsf(h) - r;
                surface = center - normal * fabsf(h);
            } else {
                normal = (center - q) / dist;
                sep = dist - r;
                surface = q;
            }
            if (sep > margin) {
                ruledAt = sep;
                return kTriRuledOut;
            }
            m.featKind = kFeatNone;
            m.featA = m.featB = -1;
            m.normal = rotate(xm.q, normal);
            const Vec3 w = apply(xm, (surface + center - normal * r) * 0.5f);
            m.points[0] = MPoint{ w, sep, motion.predict(w, m.normal, sep) };
            m.count = 1;
            return kTriKept;
        });
    } else if (other.kind == kCylinder) {
        const Solid b = cylinderSolid(other, rel);
        const Vec3 reach = cylinderReach(b.axis, b.radius, b.halfHeight) + Vec3{ margin, margin, margin };
        const Convex convexB = convexOf(cx, other);
        walked = collect(mt, M, b.center - reach, b.center + reach, [&](int t, Manifold& m, float& ruledAt) {
            if (outOfReach(bounds, t, margin)) { return kTriNone; }
            Vec3 c[3];
            meshCorners(mt, M, t, c);
            const Vec3 n = mt.normals[M.tFirst + t];
            TriangleFrame tri;
            tri.set(c, n);
            const Solid a = polySolid(ownFrame(tri.t, 0));
            const Convex triangle{ tri.verts, 3, 0.0f, false };
            Separation best;
            if (!separate(a, b, triangle, xm, convexB, xo, xm.q, margin, tol, best)) {
                ruledAt = best.gap;
                return kTriRuledOut;
            }
            m.count = 0;
            m.featKind = kFeatNone;
            m.featA = m.featB = -1;
            solidContact(cx.cap, a, b, best.normal, best.gap, xm, margin, tol.linearSlop, motion, m);
            if (m.count == 0) { return kTriNone; }
            // An edge or corner without a normal of its own leaves the push to the face.
            if (fabsf(dot(best.normal, n)) < 0.9999f) {
                Separation front = noSeparation(), back = noSeparation();
                tryAxis(a, b, n, front);
                tryAxis(a, b, -n, back);
                const int side = front.gap >= back.gap ? 0 : 1;
                if (!keepsNormal(mt.edges[M.tFirst + t], triangleFeature(c, best.normal, tol.linearSlop), side, best.normal, n)) {
                    const Separation& face = side == 0 ? front : back;
                    m.count = 0;
                    solidContact(cx.cap, a, b, face.normal, face.gap, xm, margin, tol.linearSlop, motion, m);
                    for (int k = 0; k < m.count; ++k) {
                        const Vec3 p = applyInverse(xm, m.points[k].position);
                        if (m.points[k].separation < best.gap - tol.linearSlop && !overTriangle(c, n, p, tol.linearSlop)) {
                            return kTriNone;
                        }
                    }
                    if (m.count == 0) { return kTriNone; }
                }
            }
            return kTriKept;
        });
    } else {
        const FramePoly b = otherFrame(cx.pt, other.poly, rel);
        const Convex convexB = convexOf(cx, other);
        const Vec3 grow{ margin, margin, margin };
        walked = collect(mt, M, b.lo - grow, b.hi + grow, [&](int t, Manifold& m, float& ruledAt) {
            if (outOfReach(bounds, t, margin)) { return kTriNone; }
            Vec3 c[3];
            meshCorners(mt, M, t, c);
            const Vec3 n = mt.normals[M.tFirst + t];
            TriangleFrame tri;
            tri.set(c, n);
            const FramePoly a = ownFrame(tri.t, 0);
            const FaceQuery fa = queryFaces(a, b, margin);
            if (fa.separation > margin) {
                ruledAt = fa.separation;
                return kTriRuledOut;
            }
            const FaceQuery fb = queryFaces(b, a, margin);
            if (fb.separation > margin) {
                ruledAt = fb.separation;
                return kTriRuledOut;
            }
            const float reach = maxf(margin, -maxf(fa.separation, fb.separation));
            const EdgeQuery eq = queryTriangleEdges(a, b, reach);
            if (eq.separation > margin) {
                ruledAt = eq.separation;
                return kTriRuledOut;
            }
            // Edges out of reach were skipped, so GJK confirms the shapes come within margin, unless the
            // vertex of b deepest toward the triangle already does.
            if (eq.pruned) {
                const Vec3 toward = a.n(fa.index);
                int deep = 0;
                for (int k = 1; k < b.vertexCount(); ++k) {
                    if (dot(b.v(k), toward) < dot(b.v(deep), toward)) { deep = k; }
                }
                int feature;
                const Vec3 q = closestOnTriangle(c, b.v(deep), feature);
                if (lengthSquared(b.v(deep) - q) > margin * margin) {
                    const Convex triangle{ tri.verts, 3, 0.0f, false };
                    if (apart(triangle, xm, convexB, xo, margin)) { return kTriNone; }
                }
            }
            m.count = 0;
            m.featKind = kFeatNone;
            m.featA = m.featB = -1;
            if (eq.a >= 0 && eq.separation > 0.9f * maxf(fa.separation, fb.separation) + absTol) {
                edgeContact(a, b, eq, xm, margin, tol.linearSlop, motion, m);
            } else if (fb.separation > 0.98f * fa.separation + absTol) {
                faceContact(b, fb.index, a, true, xm, margin, tol.linearSlop, motion.swapped(), m);
            } else {
                faceContact(a, fa.index, b, false, xm, margin, tol.linearSlop, motion, m);
            }
            if (m.count == 0) { return kTriNone; }
            // Off the face normal on an edge or corner with no normal of its own, the neighbour takes that
            // direction and this triangle pushes only along its face; where the face is deeper than the
            // shapes overlap, the contact belongs to the neighbour.
            const Vec3 normal = unrotate(xm.q, m.normal);
            if (fabsf(dot(normal, n)) < 0.9999f) {
                if (!keepsNormal(mt.edges[M.tFirst + t], triangleFeature(c, normal, tol.linearSlop), fa.index, normal, n)) {
                    const float floor = maxf(maxf(fa.separation, fb.separation), eq.separation) - tol.linearSlop;
                    m.count = 0;
                    faceContact(a, fa.index, b, false, xm, margin, tol.linearSlop, motion, m);
                    for (int k = 0; k < m.count; ++k) {
                        const Vec3 p = applyInverse(xm, m.points[k].position);
                        if (m.points[k].separation < floor && !overTriangle(c, n, p, tol.linearSlop)) { return kTriNone; }
                    }
                    if (m.count == 0) { return kTriNone; }
                }
            }
            for (int k = 0; k < m.count; ++k) {
                MPoint& p = m.points[k];
                p.predicted = motion.predict(p.position, m.normal, p.separation);
            }
            return kTriKept;
        });
    }
    return walked ? kMeshOk : kMeshTooMany;
}

// Triangles facing the same way share one manifold, under the normal of the deepest of them
// (src/collide3d.cpp:1746-1776): found in visiting order into at most kMaxMeshParts manifolds.
TF_HD int groupMeshManifolds(const Manifold* found, int nFound, const Tolerances& tol, Manifold* out, int& outCount) {
    outCount = 0;
    int8_t owner[kMaxMeshFound];
    for (int i = 0; i < nFound; ++i) { owner[i] = -1; }
    MPoint pts[4 * kMaxMeshFound];
    for (int i = 0; i < nFound; ++i) {
        if (owner[i] >= 0) { continue; }
        if (outCount >= kMaxMeshParts) { return kMeshTooMany; }
        int np = 0;
        int lead = i;
        float deepest = FLT_MAX;
        for (int j = i; j < nFound; ++j) {
            if (owner[j] >= 0 || dot(found[j].normal, found[i].normal) < kSameNormal) { continue; }
            owner[j] = (int8_t)outCount;
            for (int k = 0; k < found[j].count; ++k) {
                pts[np++] = found[j].points[k];
                if (found[j].points[k].separation < deepest) {
                    deepest = found[j].points[k].separation;
                    lead = j;
                }
            }
        }
        // A curved patch is deepest at one end, so spread is chosen among all penetrating points.
        float deep = FLT_MAX;
        for (int k = 0; k < np; ++k) { deep = minf(deep, pts[k].predicted); }
        Manifold& m = out[outCount++];
        m.featKind = kFeatNone;
        m.featA = m.featB = -1;
        reduceManifold(pts, np, found[lead].normal, maxf(tol.linearSlop, -deep), m, 0.0f, false);
    }
    return kMeshOk;
}

// collideMesh (src/collide3d.cpp:1577-1776) for a sphere or polyhedron on one thread: up to kMaxMeshParts
// manifolds with normals from the mesh, into out. Returns kMeshOk, or why the pair could not be collided
// exactly.
TF_HD int collideMesh(const CollideCtx& cx, const DShape& mesh, const Transform& xm, const DShape& other,
                      const Transform& xo, float margin, const Motion& motion, Manifold* out, int& outCount,
                      MeshBounds* bounds) {
    outCount = 0;
    Manifold found[kMaxMeshFound];
    SerialCollect collect{ found, 0, bounds, kMeshOk };
    const int walk = collideMeshTriangles(cx, mesh, xm, other, xo, margin, motion, bounds, collect);
    if (walk != kMeshOk) { return walk; }
    if (collect.status != kMeshOk) { return collect.status; }
    return groupMeshManifolds(found, collect.nFound, cx.tol, out, outCount);
}

#if defined(__CUDACC__)
// The same with the warp's lanes over the triangles; found is the warp's shared room for kMaxMeshFound
// manifolds, and each lane passes its own copy of bounds (whose found, if any, the warp shares). The grouping
// runs on lane 0, whose out and outCount and return value are the pair's; the other lanes return kMeshOk with
// nothing in out unless the triangles already failed.
static __device__ int collideMeshWarp(const CollideCtx& cx, const DShape& mesh, const Transform& xm, const DShape& other,
                               const Transform& xo, float margin, const Motion& motion, Manifold* out, int& outCount,
                               MeshBounds* bounds, Manifold* found, uint32_t lane) {
    outCount = 0;
    WarpCollect collect{ found, 0, bounds, kMeshOk, lane };
    const int walk = collideMeshTriangles(cx, mesh, xm, other, xo, margin, motion, bounds, collect);
    if (walk != kMeshOk) { return walk; }
    if (collect.status != kMeshOk) { return collect.status; }
    if (lane != 0) { return kMeshOk; }
    return groupMeshManifolds(found, collect.nFound, cx.tol, out, outCount);
}
#endif

}
