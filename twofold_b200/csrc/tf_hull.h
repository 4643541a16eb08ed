// Convex hulls of point clouds, for hull shapes (twofold::computeHull, include/twofold/hull.h:17).
//
// The hull's vertex order and face loops decide a shape's mass sums and every feature id the narrowphase
// reports, so they must come out exactly as the reference builds them (src/hull.cpp). What has to agree is
// the arithmetic of every plane test and the order in which ties are broken; both are kept below, and each
// one names the rule it keeps. The surface itself is held differently: faces are columns of arrays with an
// explicit neighbour across each edge, the points waiting above a face are a list threaded through one array,
// and the live vertex count is kept as faces come and go.
//
// The method is quickhull (Barber, Dobkin and Huhdanpaa, 1996) with a vertex budget: a tetrahedron of extreme
// points, then repeatedly the point farthest above any face is joined to the horizon of the faces it sees.
// Faces merge afterwards into coplanar convex polygons. Clouds that span no volume are thickened into a slab.
#pragma once

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <utility>
#include <vector>

#include "tf_math.cuh"

namespace tfb {

struct HullResult {
    std::vector<Vec3> vertices;
    std::vector<std::vector<int>> faces;  // counter-clockwise seen from outside
};

namespace hull {

// Neighbouring faces whose normals agree closer than this cosine merge into one polygon.
constexpr float kMergeCos = 0.9998f;
constexpr int kNone = -1;

// The triangulated surface as it grows. Face f has corners tri[f], counter-clockwise seen from outside; its
// edge e runs tri[f][e] -> tri[f][(e + 1) % 3], and across[f][e] is the face on the other side of that edge.
// The points above face f that it is the best face for wait in a list in the order they came, from first[f]
// through follow[] to last[f].
struct Surface {
    const std::vector<Vec3>& pts;
    float tol = 0.0f;
    float foldSine = 0.0f;  // the steepest fold-back that keeps every corner within the tolerance

    std::vector<std::array<int, 3>> tri, across;
    std::vector<Vec3> normal;
    std::vector<float> offset;
    std::vector<uint8_t> live;
    std::vector<int> first, last, follow;
    std::vector<int> useCount;  // live faces at each point
    int liveVertices = 0;
    std::vector<int> nearly;     // points within the tolerance above some face, kept for one more try
    std::vector<uint8_t> tried;  // points already given that try

    Surface(const std::vector<Vec3>& p, float tolerance, float size)
        : pts(p), tol(tolerance), foldSine(tolerance / size), follow(p.size(), kNone), useCount(p.size(), 0),
          tried(p.size(), 0) {}

    int faceCount() const { return (int)tri.size(); }

    // The plane test every decision below rests on (src/hull.cpp: Builder::distance).
    float height(int f, int p) const { return dot(normal[f], pts[p]) - offset[f]; }

    int addFace(int a, int b, int c) {
        const int f = faceCount();
        tri.push_back({ a, b, c });
        across.push_back({ kNone, kNone, kNone });
        const Vec3 n = normalize(cross(pts[b] - pts[a], pts[c] - pts[a]));
        normal.push_back(n);
        offset.push_back(dot(n, pts[a]));
        live.push_back(1);
        first.push_back(kNone);
        last.push_back(kNone);
        for (int v : { a, b, c }) {
            if (useCount[v]++ == 0) { ++liveVertices; }
        }
        return f;
    }

    void removeFace(int f) {
        live[f] = 0;
        for (int v : tri[f]) {
            if (--useCount[v] == 0) { --liveVertices; }
        }
        first[f] = last[f] = kNone;
    }

    void enqueue(int f, int p) {
        follow[p] = kNone;
        if (last[f] == kNone) {
            first[f] = p;
        } else {
            follow[last[f]] = p;
        }
        last[f] = p;
    }

    void dequeue(int f, int p) {
        int prev = kNone;
        for (int q = first[f]; q != kNone; prev = q, q = follow[q]) {
            if (q != p) { continue; }
            if (prev == kNone) {
                first[f] = follow[q];
            } else {
                follow[prev] = follow[q];
            }
            if (last[f] == q) { last[f] = prev; }
            return;
        }
    }

    // The edge of face g that runs b -> a, where a -> b is an edge of its neighbour.
    int edgeBack(int g, int a, int b) const {
        for (int e = 0; e < 3; ++e) {
            if (tri[g][e] == b && tri[g][(e + 1) % 3] == a) { return e; }
        }
        return kNone;
    }

    // Each point joins the face it is farthest above, by more than the tolerance, the first such face in the
    // order given winning ties; a point above some face by no more than the tolerance is kept for one more
    // try, once (src/hull.cpp: Builder::assign).
    void place(const std::vector<int>& points, const std::vector<int>& faces) {
        for (int p : points) {
            int best = kNone;
            float bestHeight = tol, highest = -FLT_MAX;
            for (int f : faces) {
                const float h = height(f, p);
                highest = std::max(highest, h);
                if (h > bestHeight) {
                    bestHeight = h;
                    best = f;
                }
            }
            if (best != kNone) {
                enqueue(best, p);
            } else if (highest > 0.0f && !tried[p]) {
                nearly.push_back(p);
            }
        }
    }

    // Whether face g, across edge a -> b of the face `from` that the eye sees, has to go too: the eye is
    // clearly above it, or the new face over a -> b would be a sliver, face inward, or fold back over it by
    // more than the tolerance allows (src/hull.cpp: Builder::sees).
    bool goesToo(int from, int g, int a, int b, int eye) const {
        const float h = height(g, eye);
        if (h > tol) { return true; }
        const Vec3 edge = normalize(pts[b] - pts[a]);
        const Vec3 r = pts[eye] - pts[a];
        const float reach = length(r - edge * dot(r, edge));
        if (reach <= tol) { return true; }
        if (height(from, eye) <= tol && dot(r, cross(normal[from], edge)) <= 0.0f) { return true; }
        if (h <= 0.0f) { return false; }
        return dot(r, cross(normal[g], edge)) <= 0.0f || h > foldSine * reach;
    }

    struct RimEdge {
        int a, b;    // the edge, as the removed face ran it
        int outer;   // the face kept on its far side
    };

    // Whether the rim edges, each start used once, chain into one loop through all of them that begins and
    // ends at the first edge (src/hull.cpp: Builder::singleLoop).
    static bool oneLoop(const std::vector<RimEdge>& rim) {
        const size_t n = rim.size();
        if (n == 0) { return false; }
        std::vector<std::pair<int, int>> byStart(n);  // (start vertex, edge)
        for (size_t i = 0; i < n; ++i) { byStart[i] = { rim[i].a, (int)i }; }
        std::sort(byStart.begin(), byStart.end());
        for (size_t i = 1; i < n; ++i) {
            if (byStart[i].first == byStart[i - 1].first) { return false; }
        }
        size_t at = 0;
        for (size_t step = 1; step < n; ++step) {
            const int v = rim[at].b;
            const auto it = std::lower_bound(byStart.begin(), byStart.end(), std::make_pair(v, -1));
            if (it == byStart.end() || it->first != v || it->second == 0) { return false; }
            at = (size_t)it->second;
        }
        return rim[at].b == rim[0].a;
    }

    // Joins `eye` to the horizon of the faces it sees, starting from face `start`; changes nothing and returns
    // false unless that horizon is one loop (src/hull.cpp: Builder::addPoint). The faces seen are found in
    // breadth-first order over the edges in corner order, which fixes the order of the rim and so of the new
    // faces.
    bool raise(int start, int eye) {
        std::vector<int> cone{ start };
        std::vector<uint8_t> inCone(faceCount(), 0);
        inCone[start] = 1;
        std::vector<RimEdge> rim;
        for (size_t k = 0; k < cone.size(); ++k) {
            const int f = cone[k];
            for (int e = 0; e < 3; ++e) {
                const int g = across[f][e];
                if (inCone[g]) { continue; }
                const int a = tri[f][e], b = tri[f][(e + 1) % 3];
                if (goesToo(f, g, a, b, eye)) {
                    inCone[g] = 1;
                    cone.push_back(g);
                } else {
                    rim.push_back({ a, b, g });
                }
            }
        }
        // A face first met from one side and later taken from another leaves an edge that is not rim.
        rim.erase(std::remove_if(rim.begin(), rim.end(), [&](const RimEdge& r) { return inCone[r.outer] != 0; }),
                  rim.end());
        if (!oneLoop(rim)) { return false; }

        std::vector<int> homeless;
        for (int f : cone) {
            for (int p = first[f]; p != kNone; p = follow[p]) {
                if (p != eye) { homeless.push_back(p); }
            }
            removeFace(f);
        }
        // The fan: one face per rim edge, in rim order. Face j sits on rim edge a_j -> b_j; across its edge 0 is
        // the kept face, across edge 1 (b_j -> eye) the fan face starting at b_j, across edge 2 (eye -> a_j) the
        // fan face ending at a_j.
        const int fan0 = faceCount();
        const int n = (int)rim.size();
        std::vector<std::pair<int, int>> startOf(n), endOf(n);
        for (int j = 0; j < n; ++j) {
            addFace(rim[j].a, rim[j].b, eye);
            startOf[j] = { rim[j].a, fan0 + j };
            endOf[j] = { rim[j].b, fan0 + j };
        }
        std::sort(startOf.begin(), startOf.end());
        std::sort(endOf.begin(), endOf.end());
        auto find = [](const std::vector<std::pair<int, int>>& v, int key) {
            return std::lower_bound(v.begin(), v.end(), std::make_pair(key, -1))->second;
        };
        std::vector<int> fan(n);
        for (int j = 0; j < n; ++j) {
            const int f = fan0 + j;
            fan[j] = f;
            const int outer = rim[j].outer;
            across[f][0] = outer;
            across[outer][edgeBack(outer, rim[j].a, rim[j].b)] = f;
            across[f][1] = find(startOf, rim[j].b);
            across[f][2] = find(endOf, rim[j].a);
        }
        place(homeless, fan);
        return true;
    }

    // The tetrahedron (faces in the order and orientation src/hull.cpp: Builder::build gives them), then
    // points until the budget is spent or none is left above a face.
    void build(const int simplex[4], int maxVertices) {
        Vec3 center{ 0, 0, 0 };
        for (int i = 0; i < 4; ++i) { center += pts[simplex[i]] * 0.25f; }
        static const int kTetra[4][3] = { { 0, 1, 2 }, { 0, 1, 3 }, { 0, 2, 3 }, { 1, 2, 3 } };
        for (const auto& t : kTetra) {
            int a = simplex[t[0]], b = simplex[t[1]], c = simplex[t[2]];
            if (dot(cross(pts[b] - pts[a], pts[c] - pts[a]), pts[a] - center) < 0.0f) { std::swap(b, c); }
            addFace(a, b, c);
        }
        for (int f = 0; f < 4; ++f) {
            for (int e = 0; e < 3; ++e) {
                for (int g = 0; g < 4; ++g) {
                    if (g != f && edgeBack(g, tri[f][e], tri[f][(e + 1) % 3]) != kNone) { across[f][e] = g; }
                }
            }
        }
        std::vector<int> others;
        for (int i = 0; i < (int)pts.size(); ++i) {
            if (i != simplex[0] && i != simplex[1] && i != simplex[2] && i != simplex[3]) { others.push_back(i); }
        }
        place(others, { 0, 1, 2, 3 });
        while (liveVertices < maxVertices) {
            // The farthest point above any face: faces in order, each face's points in the order they came.
            int face = kNone, eye = kNone;
            float far = 0.0f;
            for (int f = 0; f < faceCount(); ++f) {
                if (!live[f]) { continue; }
                for (int p = first[f]; p != kNone; p = follow[p]) {
                    const float h = height(f, p);
                    if (h > far) {
                        far = h;
                        face = f;
                        eye = p;
                    }
                }
            }
            if (face == kNone) {
                if (retryNearly()) { continue; }
                break;
            }
            if (!raise(face, eye)) { dequeue(face, eye); }
        }
    }

    // The points kept within the tolerance, tried once more against the faces as they are now.
    bool retryNearly() {
        std::vector<int> points;
        points.swap(nearly);
        for (int p : points) { tried[p] = 1; }
        std::vector<int> faces;
        for (int f = 0; f < faceCount(); ++f) {
            if (live[f]) { faces.push_back(f); }
        }
        place(points, faces);
        for (int f : faces) {
            if (first[f] != kNone) { return true; }
        }
        return false;
    }

    // Whether face g lies in the plane of the region's seed, within the tolerance at each corner.
    bool inPlane(int seed, int g) const {
        if (dot(normal[seed], normal[g]) < kMergeCos) { return false; }
        for (int v : tri[g]) {
            if (std::fabs(height(seed, v)) > tol) { return false; }
        }
        return true;
    }

    // The outline of the faces marked `id` in `owner`, as one loop from its lowest vertex; false unless the
    // outline is one simple loop (src/hull.cpp: Builder::boundary).
    bool outline(const std::vector<int>& faces, const std::vector<int>& owner, int id, std::vector<int>& loop) const {
        std::vector<std::pair<int, int>> step;  // (from, to) of every outline edge
        for (int f : faces) {
            for (int e = 0; e < 3; ++e) {
                if (owner[across[f][e]] == id) { continue; }
                step.push_back({ tri[f][e], tri[f][(e + 1) % 3] });
            }
        }
        if (step.empty()) { return false; }
        std::sort(step.begin(), step.end());
        for (size_t i = 1; i < step.size(); ++i) {
            if (step[i].first == step[i - 1].first) { return false; }
        }
        const int from = step[0].first;
        int v = from;
        do {
            loop.push_back(v);
            const auto it = std::lower_bound(step.begin(), step.end(), std::make_pair(v, INT32_MIN));
            if (it == step.end() || it->first != v || loop.size() > step.size()) { return false; }
            v = it->second;
        } while (v != from);
        return loop.size() == step.size();
    }

    // No corner of the loop bends back by more than the tolerance (src/hull.cpp: Builder::convex).
    bool convexLoop(const std::vector<int>& loop, const Vec3& n) const {
        const size_t k = loop.size();
        for (size_t i = 0; i < k; ++i) {
            const Vec3& a = pts[loop[i]];
            const Vec3& b = pts[loop[(i + 1) % k]];
            const Vec3& c = pts[loop[(i + 2) % k]];
            if (dot(cross(b - a, c - b), n) < -tol * length(c - a)) { return false; }
        }
        return true;
    }

    // The coplanar neighbours of `seed`, breadth first over the edges in corner order, marked in `owner`.
    std::vector<int> flood(int seed, std::vector<int>& owner, int id) const {
        std::vector<int> faces{ seed };
        owner[seed] = id;
        for (size_t k = 0; k < faces.size(); ++k) {
            for (int e = 0; e < 3; ++e) {
                const int g = across[faces[k]][e];
                if (owner[g] < 0 && inPlane(seed, g)) {
                    owner[g] = id;
                    faces.push_back(g);
                }
            }
        }
        return faces;
    }

    // A region grown from the seed one neighbour at a time, each kept only if the outline stays one convex
    // loop (src/hull.cpp: Builder::grow).
    std::vector<int> growConvex(int seed, std::vector<int>& owner, int id) const {
        std::vector<int> faces{ seed }, loop;
        outline(faces, owner, id, loop);
        for (size_t k = 0; k < faces.size(); ++k) {
            for (int e = 0; e < 3; ++e) {
                const int g = across[faces[k]][e];
                if (owner[g] >= 0 || !inPlane(seed, g)) { continue; }
                owner[g] = id;
                faces.push_back(g);
                std::vector<int> grown;
                if (outline(faces, owner, id, grown) && convexLoop(grown, normal[seed])) {
                    loop.swap(grown);
                } else {
                    owner[g] = kNone;
                    faces.pop_back();
                }
            }
        }
        return loop;
    }

    // The faces merged into polygons, regions seeded in face order; vertices numbered in order of first use.
    HullResult polygons(const std::vector<Vec3>& original) const {
        std::vector<int> owner(faceCount(), kNone);
        std::vector<std::vector<int>> loops;
        for (int seed = 0; seed < faceCount(); ++seed) {
            if (!live[seed] || owner[seed] >= 0) { continue; }
            const int id = (int)loops.size();
            const std::vector<int> region = flood(seed, owner, id);
            std::vector<int> loop;
            if (!outline(region, owner, id, loop) || !convexLoop(loop, normal[seed])) {
                for (size_t k = 1; k < region.size(); ++k) { owner[region[k]] = kNone; }
                loop = growConvex(seed, owner, id);
            }
            loops.push_back(std::move(loop));
        }
        HullResult out;
        std::vector<int> number(pts.size(), kNone);
        for (std::vector<int>& loop : loops) {
            for (int& v : loop) {
                if (number[v] == kNone) {
                    number[v] = (int)out.vertices.size();
                    out.vertices.push_back(original[v]);
                }
                v = number[v];
            }
            out.faces.push_back(std::move(loop));
        }
        return out;
    }
};

// Every point moved to each corner of a box of half size t along `count` axes, corners in binary order and the
// axes added one after another (src/hull.cpp: thicken).
inline std::vector<Vec3> slab(const std::vector<Vec3>& points, const Vec3* axes, int count, float t) {
    std::vector<Vec3> out;
    out.reserve(points.size() << count);
    for (const Vec3& p : points) {
        for (int corner = 0; corner < (1 << count); ++corner) {
            Vec3 q = p;
            for (int i = 0; i < count; ++i) { q += axes[i] * (((corner >> i) & 1) ? t : -t); }
            out.push_back(q);
        }
    }
    return out;
}

// The first point farthest by `measure` (strictly greater wins, so the first of equals stays), with its value.
template <class Measure>
inline std::pair<int, float> farthest(const std::vector<Vec3>& points, Measure measure) {
    int at = 0;
    float best = 0.0f;
    for (int i = 0; i < (int)points.size(); ++i) {
        const float d = measure(points[i]);
        if (d > best) {
            best = d;
            at = i;
        }
    }
    return { at, best };
}

// src/hull.cpp: hullOf. Tolerances from the cloud's extent; the tetrahedron from the farthest pair of axis
// extremes, the point farthest from their line and the point farthest from that plane; a cloud without volume
// is thickened once (the slab is far wider than the tolerance, so the thickened cloud has volume).
inline HullResult hullOf(const std::vector<Vec3>& points, int maxVertices, bool mayThicken) {
    if (points.empty()) { return {}; }
    Vec3 lo = points[0], hi = points[0];
    int ext[6] = { 0, 0, 0, 0, 0, 0 };  // lowest and highest point along x, y, z (first of equals)
    for (int i = 0; i < (int)points.size(); ++i) {
        for (int k = 0; k < 3; ++k) {
            if (comp(points[i], k) < comp(points[ext[2 * k]], k)) { ext[2 * k] = i; }
            if (comp(points[i], k) > comp(points[ext[2 * k + 1]], k)) { ext[2 * k + 1] = i; }
        }
        lo = minVec(lo, points[i]);
        hi = maxVec(hi, points[i]);
    }
    const float size = length(hi - lo);
    float reach = 0.0f;
    for (int k = 0; k < 3; ++k) { reach += std::max(std::fabs(comp(lo, k)), std::fabs(comp(hi, k))); }
    if (!std::isfinite(size) || !std::isfinite(reach)) { return {}; }
    const float tol = std::max({ 1e-4f * size, 3.0f * FLT_EPSILON * reach, 1e-8f });
    const float half = std::max({ 0.005f * size, 1e-4f, 10.0f * tol });

    int corner[4] = { ext[0], ext[0], 0, 0 };
    float spread = 0.0f;
    for (int i = 0; i < 6; ++i) {
        for (int j = i + 1; j < 6; ++j) {
            const float d = lengthSquared(points[ext[i]] - points[ext[j]]);
            if (d > spread) {
                spread = d;
                corner[0] = ext[i];
                corner[1] = ext[j];
            }
        }
    }
    if (spread <= tol * tol) {
        if (!mayThicken) { return {}; }
        const Vec3 axes[3] = { { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } };
        return hullOf(slab(points, axes, 3, half), maxVertices, false);
    }
    const Vec3 o = points[corner[0]];
    const Vec3 dir = normalize(points[corner[1]] - o);
    const auto offLine = farthest(points, [&](const Vec3& p) { return length(cross(p - o, dir)); });
    corner[2] = offLine.first;
    if (offLine.second <= tol) {
        if (!mayThicken) { return {}; }
        const Vec3 u = perpendicular(dir);
        const Vec3 axes[2] = { u, cross(dir, u) };
        return hullOf(slab(points, axes, 2, half), maxVertices, false);
    }
    const Vec3 n = normalize(cross(points[corner[1]] - o, points[corner[2]] - o));
    const auto offPlane = farthest(points, [&](const Vec3& p) { return std::fabs(dot(p - o, n)); });
    corner[3] = offPlane.first;
    if (offPlane.second <= tol) {
        if (!mayThicken) { return {}; }
        return hullOf(slab(points, &n, 1, half), maxVertices, false);
    }
    // Built about the box's centre, so the tolerance needs no allowance for distance from the origin.
    const Vec3 mid = (lo + hi) * 0.5f;
    std::vector<Vec3> local;
    local.reserve(points.size());
    for (const Vec3& p : points) { local.push_back(p - mid); }
    Surface s(local, std::max(1e-4f * size, 1e-8f), size);
    s.build(corner, maxVertices);
    return s.polygons(points);
}

}  // namespace hull

// At least 4 vertices; non-finite points are skipped (src/hull.cpp: computeHull).
inline HullResult computeHull(const std::vector<Vec3>& points, int maxVertices) {
    maxVertices = std::max(maxVertices, 4);
    std::vector<Vec3> kept;
    kept.reserve(points.size());
    for (const Vec3& p : points) {
        if (std::isfinite(p.x) && std::isfinite(p.y) && std::isfinite(p.z)) { kept.push_back(p); }
    }
    return hull::hullOf(kept, maxVertices, true);
}

}  // namespace tfb
