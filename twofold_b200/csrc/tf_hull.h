// Convex hulls of point clouds for hull shapes: the reference's computeHull (src/hull.cpp:1-412), restated as
// host code with the same float operations in the same order, so that the vertex and face order, and with
// them every feature id the narrowphase reports, come out as the reference's.
//
// The method: incremental quickhull over triangles with a vertex budget. Start from a tetrahedron of extreme
// points; repeatedly take the point farthest outside any face (the eye), remove the faces it sees (with
// tolerance rules against slivers and fold-backs), and fan new faces from the horizon to the eye; points the
// tolerance dropped get one more try at the end. The triangles are then merged into coplanar convex polygons.
// Degenerate clouds (a point, a segment, a plane) are thickened into a thin slab first.
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <map>
#include <unordered_map>
#include <utility>
#include <vector>

#include "tf_math.cuh"

namespace tfb {

struct HullResult {
    std::vector<Vec3> vertices;
    std::vector<std::vector<int>> faces;  // counter-clockwise seen from outside
};

namespace hull {

constexpr float kCoplanarCos = 0.9998f;  // neighbouring faces closer than this merge into one polygon

inline uint64_t directedEdge(int a, int b) { return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b; }

struct Tri {
    int v[3];
    Vec3 normal;
    float offset = 0.0f;
    std::vector<int> outside;  // points this face is the best choice for
    bool alive = true;
};

// The hull of points already moved near the origin (`p`); `original` are the caller's points, returned in the
// result.
class Quickhull {
public:
    Quickhull(const std::vector<Vec3>& p, const std::vector<Vec3>& original, float tol, float size)
        : p_(p), original_(original), tol_(tol), fold_(tol / size), reclaimed_(p.size(), false) {}

    void run(const int simplex[4], int maxVertices) {
        Vec3 center{ 0, 0, 0 };
        for (int i = 0; i < 4; ++i) { center += p_[simplex[i]] * 0.25f; }
        static const int tet[4][3] = { { 0, 1, 2 }, { 0, 1, 3 }, { 0, 2, 3 }, { 1, 2, 3 } };
        for (const auto& t : tet) {
            int a = simplex[t[0]], b = simplex[t[1]], c = simplex[t[2]];
            if (dot(cross(p_[b] - p_[a], p_[c] - p_[a]), p_[a] - center) < 0.0f) { std::swap(b, c); }
            addTri(a, b, c);
        }
        std::vector<int> others;
        for (int i = 0; i < (int)p_.size(); ++i) {
            if (i != simplex[0] && i != simplex[1] && i != simplex[2] && i != simplex[3]) { others.push_back(i); }
        }
        distribute(others, { 0, 1, 2, 3 });
        while (usedVertices() < maxVertices) {
            int face = -1, eye = -1;
            float far = 0.0f;
            for (int fi = 0; fi < (int)tris_.size(); ++fi) {
                if (!tris_[fi].alive) { continue; }
                for (int pi : tris_[fi].outside) {
                    const float d = above(tris_[fi], pi);
                    if (d > far) {
                        far = d;
                        face = fi;
                        eye = pi;
                    }
                }
            }
            if (face < 0) {
                if (retryDropped()) { continue; }
                break;
            }
            if (!addEye(face, eye)) {
                std::vector<int>& out = tris_[face].outside;
                out.erase(std::find(out.begin(), out.end(), eye));
            }
        }
    }

    // Coplanar neighbours merged into convex polygons; vertices numbered in order of first use.
    HullResult result() const {
        std::vector<int> region(tris_.size(), -1);
        std::vector<std::vector<int>> polygons;
        for (int seed = 0; seed < (int)tris_.size(); ++seed) {
            if (!tris_[seed].alive || region[seed] >= 0) { continue; }
            const int id = (int)polygons.size();
            std::vector<int> members{ seed };
            region[seed] = id;
            for (size_t k = 0; k < members.size(); ++k) {
                const Tri& f = tris_[members[k]];
                for (int i = 0; i < 3; ++i) {
                    const int twin = edgeOwner_.at(directedEdge(f.v[(i + 1) % 3], f.v[i]));
                    if (region[twin] >= 0 || !coplanar(tris_[seed], tris_[twin])) { continue; }
                    region[twin] = id;
                    members.push_back(twin);
                }
            }
            std::vector<int> loop;
            if (!outline(members, region, id, loop) || !convexLoop(loop, tris_[seed].normal)) {
                for (size_t k = 1; k < members.size(); ++k) { region[members[k]] = -1; }
                loop = growConvex(seed, region, id);
            }
            polygons.push_back(loop);
        }
        HullResult out;
        std::vector<int> number(p_.size(), -1);
        for (std::vector<int>& loop : polygons) {
            for (int& v : loop) {
                if (number[v] < 0) {
                    number[v] = (int)out.vertices.size();
                    out.vertices.push_back(original_[v]);
                }
                v = number[v];
            }
            out.faces.push_back(std::move(loop));
        }
        return out;
    }

private:
    void addTri(int a, int b, int c) {
        Tri f;
        f.v[0] = a;
        f.v[1] = b;
        f.v[2] = c;
        f.normal = normalize(cross(p_[b] - p_[a], p_[c] - p_[a]));
        f.offset = dot(f.normal, p_[a]);
        const int fi = (int)tris_.size();
        for (int i = 0; i < 3; ++i) { edgeOwner_[directedEdge(f.v[i], f.v[(i + 1) % 3])] = fi; }
        tris_.push_back(std::move(f));
    }

    float above(const Tri& f, int pi) const { return dot(f.normal, p_[pi]) - f.offset; }

    // Each point goes to the candidate face it is farthest above (beyond the tolerance); a point within the
    // tolerance of some face but above none is kept for one retry.
    void distribute(const std::vector<int>& points, const std::vector<int>& candidates) {
        for (int pi : points) {
            int best = -1;
            float far = tol_, top = -FLT_MAX;
            for (int fi : candidates) {
                const float d = above(tris_[fi], pi);
                top = std::max(top, d);
                if (d > far) {
                    far = d;
                    best = fi;
                }
            }
            if (best >= 0) {
                tris_[best].outside.push_back(pi);
            } else if (top > 0.0f && !reclaimed_[pi]) {
                dropped_.push_back(pi);
            }
        }
    }

    bool coplanar(const Tri& seed, const Tri& f) const {
        if (dot(seed.normal, f.normal) < kCoplanarCos) { return false; }
        for (int v : f.v) {
            if (std::fabs(above(seed, v)) > tol_) { return false; }
        }
        return true;
    }

    int usedVertices() const {
        std::vector<bool> used(p_.size(), false);
        int n = 0;
        for (const Tri& f : tris_) {
            if (!f.alive) { continue; }
            for (int v : f.v) {
                if (!used[v]) {
                    used[v] = true;
                    ++n;
                }
            }
        }
        return n;
    }

    // Points dropped within the tolerance are tested once more against the finished faces.
    bool retryDropped() {
        std::vector<int> points, alive;
        points.swap(dropped_);
        for (int pi : points) { reclaimed_[pi] = true; }
        for (int fi = 0; fi < (int)tris_.size(); ++fi) {
            if (tris_[fi].alive) { alive.push_back(fi); }
        }
        distribute(points, alive);
        for (int fi : alive) {
            if (!tris_[fi].outside.empty()) { return true; }
        }
        return false;
    }

    // Whether face f, across edge a-b of the visible face `from`, must go as well: the eye is clearly above
    // it, the new face over a-b would be a sliver or fold back over it, or would face inward.
    bool mustGo(const Tri& from, const Tri& f, int a, int b, int eye) const {
        const float d = above(f, eye);
        if (d > tol_) { return true; }
        const Vec3 edge = normalize(p_[b] - p_[a]);
        const Vec3 r = p_[eye] - p_[a];
        const float h = length(r - edge * dot(r, edge));
        if (h <= tol_) { return true; }
        if (above(from, eye) <= tol_ && dot(r, cross(from.normal, edge)) <= 0.0f) { return true; }
        if (d <= 0.0f) { return false; }
        return dot(r, cross(f.normal, edge)) <= 0.0f || d > fold_ * h;
    }

    // Adds the eye, unless the horizon of the faces it removes is not a single loop (then nothing changes).
    bool addEye(int start, int eye) {
        std::vector<int> visible{ start };
        std::vector<bool> seen(tris_.size(), false);
        seen[start] = true;
        std::vector<std::pair<int, int>> horizon;
        for (size_t k = 0; k < visible.size(); ++k) {
            const Tri& f = tris_[visible[k]];
            for (int i = 0; i < 3; ++i) {
                const int a = f.v[i], b = f.v[(i + 1) % 3];
                const int twin = edgeOwner_.at(directedEdge(b, a));
                if (seen[twin]) { continue; }
                if (mustGo(f, tris_[twin], a, b, eye)) {
                    seen[twin] = true;
                    visible.push_back(twin);
                } else {
                    horizon.push_back({ a, b });
                }
            }
        }
        std::vector<std::pair<int, int>> kept;
        for (const auto& e : horizon) {
            if (!seen[edgeOwner_.at(directedEdge(e.second, e.first))]) { kept.push_back(e); }
        }
        horizon.swap(kept);
        if (!oneLoop(horizon)) { return false; }
        std::vector<int> homeless;
        for (int fi : visible) {
            Tri& f = tris_[fi];
            f.alive = false;
            for (int i = 0; i < 3; ++i) { edgeOwner_.erase(directedEdge(f.v[i], f.v[(i + 1) % 3])); }
            for (int pi : f.outside) {
                if (pi != eye) { homeless.push_back(pi); }
            }
            f.outside.clear();
        }
        std::vector<int> fresh;
        for (const auto& e : horizon) {
            fresh.push_back((int)tris_.size());
            addTri(e.first, e.second, eye);
        }
        distribute(homeless, fresh);
        return true;
    }

    // The horizon edges (a, b) must chain into one closed loop, each start vertex used once.
    static bool oneLoop(const std::vector<std::pair<int, int>>& horizon) {
        for (size_t i = 0; i < horizon.size(); ++i) {
            for (size_t j = 0; j < i; ++j) {
                if (horizon[i].first == horizon[j].first) { return false; }
            }
        }
        int v = horizon.empty() ? -1 : horizon[0].second;
        for (size_t steps = 1; steps < horizon.size(); ++steps) {
            size_t k = 0;
            while (k < horizon.size() && horizon[k].first != v) { ++k; }
            if (k == horizon.size() || k == 0) { return false; }
            v = horizon[k].second;
        }
        return !horizon.empty() && v == horizon[0].first;
    }

    // Every corner of the loop turns left about the normal, up to the tolerance.
    bool convexLoop(const std::vector<int>& loop, const Vec3& normal) const {
        const size_t n = loop.size();
        for (size_t i = 0; i < n; ++i) {
            const Vec3& a = p_[loop[i]];
            const Vec3& b = p_[loop[(i + 1) % n]];
            const Vec3& c = p_[loop[(i + 2) % n]];
            if (dot(cross(b - a, c - b), normal) < -tol_ * length(c - a)) { return false; }
        }
        return true;
    }

    // Grows a region from its seed one coplanar face at a time, keeping its outline one convex loop.
    std::vector<int> growConvex(int seed, std::vector<int>& region, int id) const {
        std::vector<int> members{ seed }, loop;
        outline(members, region, id, loop);
        for (size_t k = 0; k < members.size(); ++k) {
            for (int i = 0; i < 3; ++i) {
                const Tri& f = tris_[members[k]];
                const int twin = edgeOwner_.at(directedEdge(f.v[(i + 1) % 3], f.v[i]));
                if (region[twin] >= 0 || !coplanar(tris_[seed], tris_[twin])) { continue; }
                region[twin] = id;
                members.push_back(twin);
                std::vector<int> grown;
                if (outline(members, region, id, grown) && convexLoop(grown, tris_[seed].normal)) {
                    loop.swap(grown);
                } else {
                    region[twin] = -1;
                    members.pop_back();
                }
            }
        }
        return loop;
    }

    // The outline of a region as one simple loop from its lowest vertex; fails otherwise.
    bool outline(const std::vector<int>& members, const std::vector<int>& region, int id, std::vector<int>& loop) const {
        std::map<int, int> next;
        for (int fi : members) {
            const Tri& f = tris_[fi];
            for (int i = 0; i < 3; ++i) {
                const int a = f.v[i], b = f.v[(i + 1) % 3];
                if (region[edgeOwner_.at(directedEdge(b, a))] == id) { continue; }
                if (!next.emplace(a, b).second) { return false; }
            }
        }
        if (next.empty()) { return false; }
        const int start = next.begin()->first;
        int v = start;
        do {
            loop.push_back(v);
            auto it = next.find(v);
            if (it == next.end() || loop.size() > next.size()) { return false; }
            v = it->second;
        } while (v != start);
        return loop.size() == next.size();
    }

    const std::vector<Vec3>& p_;
    const std::vector<Vec3>& original_;
    float tol_;
    float fold_;  // sine of the steepest fold-back that leaves no corner more than the tolerance outside
    std::vector<Tri> tris_;
    std::unordered_map<uint64_t, int> edgeOwner_;  // directed edge -> the face it belongs to
    std::vector<int> dropped_;
    std::vector<bool> reclaimed_;
};

// Every point offset to each corner of a box spanned by `count` axes at +-t.
inline std::vector<Vec3> thickened(const std::vector<Vec3>& points, const Vec3* axes, int count, float t) {
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

// src/hull.cpp:332-400: tolerances from the cloud's size, the initial simplex from extreme points, degenerate
// clouds thickened once.
inline HullResult hullOf(const std::vector<Vec3>& points, int maxVertices, bool thickenFlat) {
    if (points.empty()) { return {}; }
    Vec3 lo = points[0], hi = points[0];
    int extreme[6] = {};
    for (int i = 0; i < (int)points.size(); ++i) {
        for (int k = 0; k < 3; ++k) {
            if (comp(points[i], k) < comp(points[extreme[2 * k]], k)) { extreme[2 * k] = i; }
            if (comp(points[i], k) > comp(points[extreme[2 * k + 1]], k)) { extreme[2 * k + 1] = i; }
        }
        lo = minVec(lo, points[i]);
        hi = maxVec(hi, points[i]);
    }
    const float size = length(hi - lo);
    float reach = 0.0f;
    for (int k = 0; k < 3; ++k) { reach += std::max(std::fabs(comp(lo, k)), std::fabs(comp(hi, k))); }
    if (!std::isfinite(size) || !std::isfinite(reach)) { return {}; }
    const float tol = std::max({ 1e-4f * size, 3.0f * FLT_EPSILON * reach, 1e-8f });
    const float slab = std::max({ 0.005f * size, 1e-4f, 10.0f * tol });

    int s[4] = { extreme[0], extreme[0], 0, 0 };
    float best = 0.0f;
    for (int i = 0; i < 6; ++i) {
        for (int j = i + 1; j < 6; ++j) {
            const float d = lengthSquared(points[extreme[i]] - points[extreme[j]]);
            if (d > best) {
                best = d;
                s[0] = extreme[i];
                s[1] = extreme[j];
            }
        }
    }
    if (best <= tol * tol) {
        if (!thickenFlat) { return {}; }
        const Vec3 axes[3] = { { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } };
        return hullOf(thickened(points, axes, 3, slab), maxVertices, false);
    }
    const Vec3 dir = normalize(points[s[1]] - points[s[0]]);
    best = 0.0f;
    for (int i = 0; i < (int)points.size(); ++i) {
        const float d = length(cross(points[i] - points[s[0]], dir));
        if (d > best) {
            best = d;
            s[2] = i;
        }
    }
    if (best <= tol) {
        if (!thickenFlat) { return {}; }
        const Vec3 u = perpendicular(dir);
        const Vec3 axes[2] = { u, cross(dir, u) };
        return hullOf(thickened(points, axes, 2, slab), maxVertices, false);
    }
    const Vec3 n = normalize(cross(points[s[1]] - points[s[0]], points[s[2]] - points[s[0]]));
    best = 0.0f;
    for (int i = 0; i < (int)points.size(); ++i) {
        const float d = std::fabs(dot(points[i] - points[s[0]], n));
        if (d > best) {
            best = d;
            s[3] = i;
        }
    }
    if (best <= tol) {
        if (!thickenFlat) { return {}; }
        return hullOf(thickened(points, &n, 1, slab), maxVertices, false);
    }
    // Built about the box centre, so the tolerance needs no allowance for distance from the origin.
    const Vec3 center = (lo + hi) * 0.5f;
    std::vector<Vec3> local;
    local.reserve(points.size());
    for (const Vec3& p : points) { local.push_back(p - center); }
    Quickhull q(local, points, std::max(1e-4f * size, 1e-8f), size);
    q.run(s, maxVertices);
    return q.result();
}

}  // namespace hull

// At least 4 vertices; non-finite points are skipped (src/hull.cpp:404-410).
inline HullResult computeHull(const std::vector<Vec3>& points, int maxVertices) {
    maxVertices = std::max(maxVertices, 4);
    std::vector<Vec3> kept;
    for (const Vec3& p : points) {
        if (std::isfinite(p.x) && std::isfinite(p.y) && std::isfinite(p.z)) { kept.push_back(p); }
    }
    return hull::hullOf(kept, maxVertices, true);
}

}  // namespace tfb
