// Triangle meshes for mesh shapes, built on the host (twofold::TriangleMesh, include/twofold/mesh.h:15).
//
// The device walks a mesh's tree and collides its triangles in the order they are stored, and contact order
// follows it, so the built mesh must be the reference's byte for byte (src/mesh.cpp): the same vertices in the
// same order, the same triangles dropped, normals, edge flags, tree nodes and triangle order. What decides
// those is kept exactly (which vertices count as equal and which one stands for them, the sliver test's
// arithmetic, the flag test's arithmetic, the split axis and the order triangles are ranked in along it, the
// order nodes are numbered in); how it is computed is this file's own: equal vertices are found by hashing
// their coordinates, edge neighbours by hashing their vertex pairs, and the tree is built without recursion.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <utility>
#include <vector>

#include "tf_types.cuh"

namespace tfb {

struct HostMesh {
    std::vector<Vec3> vertices;
    std::vector<uint32_t> indices;
    std::vector<Vec3> normals;
    // Bit k: edge k (corner k to k + 1) may give a contact its own normal on the front side; bit 3 + k: on
    // the back side.
    std::vector<uint8_t> edges;
    std::vector<MeshNode> nodes;

    void corners(int t, Vec3 out[3]) const {
        for (int k = 0; k < 3; ++k) { out[k] = vertices[indices[3 * t + k]]; }
    }
};

namespace mesh {

constexpr int kLeafTriangles = 4;
constexpr float kFoldSine = 0.087f;    // a neighbour folding away less than this leaves the edge no normal
constexpr float kSliverSine = 1e-3f;   // a triangle whose widest corner has a smaller sine is dropped
constexpr uint32_t kUnset = 0xffffffffu;

// Coordinates as a hash key under which equal vertices (==, so -0 equals +0) collide: adding +0 turns -0 into
// +0 and changes nothing else.
struct PointKey {
    uint32_t x, y, z;
    bool operator==(const PointKey& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct PointKeyHash {
    size_t operator()(const PointKey& k) const {
        uint64_t h = k.x * 0x9E3779B97F4A7C15ull;
        h ^= (h >> 29) + k.y * 0xBF58476D1CE4E5B9ull;
        h ^= (h >> 31) + k.z * 0x94D049BB133111EBull;
        return (size_t)(h ^ (h >> 32));
    }
};

inline PointKey keyOf(const Vec3& v) {
    const float c[3] = { v.x + 0.0f, v.y + 0.0f, v.z + 0.0f };
    PointKey k;
    std::memcpy(&k.x, &c[0], 4);
    std::memcpy(&k.y, &c[1], 4);
    std::memcpy(&k.z, &c[2], 4);
    return k;
}

inline bool finitePoint(const Vec3& v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }

// For each input vertex, the lowest-numbered finite vertex equal to it (itself if none comes before), or kUnset
// for a non-finite one (src/mesh.cpp: the merge in TriangleMesh::TriangleMesh).
inline std::vector<uint32_t> mergeEqual(const std::vector<Vec3>& v) {
    std::vector<uint32_t> rep(v.size(), kUnset);
    std::unordered_map<PointKey, uint32_t, PointKeyHash> seen;
    seen.reserve(v.size());
    for (uint32_t i = 0; i < (uint32_t)v.size(); ++i) {
        if (!finitePoint(v[i])) { continue; }
        rep[i] = seen.emplace(keyOf(v[i]), i).first->second;
    }
    return rep;
}

// Whether the triangle is too thin to keep: its widest corner (the one facing the longest side, the first of
// equals) has a sine below kSliverSine, in the reference's arithmetic.
inline bool sliver(const Vec3& p0, const Vec3& p1, const Vec3& p2) {
    const Vec3 p[3] = { p0, p1, p2 };
    int wide = 0;
    float longest = 0.0f;
    for (int k = 0; k < 3; ++k) {
        const float side = lengthSquared(p[(k + 2) % 3] - p[(k + 1) % 3]);
        if (side > longest) {
            longest = side;
            wide = k;
        }
    }
    const Vec3 e1 = p[(wide + 1) % 3] - p[wide];
    const Vec3 e2 = p[(wide + 2) % 3] - p[wide];
    return !(lengthSquared(cross(e1, e2)) > kSliverSine * kSliverSine * lengthSquared(e1) * lengthSquared(e2));
}

// Edge a -> b of a triangle with normal n, whose neighbour across it has `far` as its third corner: the edge
// may give its own normal on the front (bit 0) where the neighbour folds back, on the back (bit 3) where it
// folds forward, by more than kFoldSine (src/mesh.cpp: edgeFlags).
inline uint8_t foldFlags(const Vec3& a, const Vec3& b, const Vec3& n, const Vec3& far) {
    const Vec3 e = normalize(b - a);
    const Vec3 r = far - a;
    const float reach = length(r - e * dot(r, e));
    const float rise = dot(n, r);
    return (uint8_t)((rise < -kFoldSine * reach ? 1u : 0u) | (rise > kFoldSine * reach ? 8u : 0u));
}

// The edge flags of every triangle: an edge shared by exactly two triangles gets each side's fold flags; an
// open edge, or one shared by more, may give its own normal on both sides.
inline std::vector<uint8_t> edgeFlagsOf(const std::vector<Vec3>& v, const std::vector<uint32_t>& tri,
                                        const std::vector<Vec3>& normals) {
    const int count = (int)normals.size();
    std::vector<uint8_t> flags((size_t)count, 0);
    // Per undirected edge: its first two uses (triangle * 3 + corner) and how many there are.
    struct Uses {
        int first = -1, second = -1, n = 0;
    };
    std::unordered_map<uint64_t, Uses> byEdge;
    byEdge.reserve((size_t)count * 2);
    auto edgeKey = [&](int t, int k) {
        const uint32_t a = tri[3 * t + k], b = tri[3 * t + (k + 1) % 3];
        return ((uint64_t)std::min(a, b) << 32) | std::max(a, b);
    };
    for (int t = 0; t < count; ++t) {
        for (int k = 0; k < 3; ++k) {
            Uses& u = byEdge[edgeKey(t, k)];
            if (u.n == 0) {
                u.first = 3 * t + k;
            } else if (u.n == 1) {
                u.second = 3 * t + k;
            }
            ++u.n;
        }
    }
    for (int t = 0; t < count; ++t) {
        for (int k = 0; k < 3; ++k) {
            const Uses& u = byEdge[edgeKey(t, k)];
            if (u.n != 2) {
                flags[t] |= (uint8_t)(9u << k);
                continue;
            }
            const int other = u.first == 3 * t + k ? u.second : u.first;
            const int ot = other / 3, oc = other % 3;
            const Vec3& far = v[tri[3 * ot + (oc + 2) % 3]];
            flags[t] |= (uint8_t)(foldFlags(v[tri[3 * t + k]], v[tri[3 * t + (k + 1) % 3]], normals[t], far) << k);
        }
    }
    return flags;
}

// The tree over `count` triangles, without recursion. A node covers a range of the triangle order; one over
// more than kLeafTriangles is ranked along the axis of widest spread of triangle centres (ties by triangle
// number) and halved, its two children numbered next, the first half's subtree before the second's
// (src/mesh.cpp: Builder::build). Returns the triangle order the leaves hold.
inline std::vector<int> buildTree(const HostMesh& m, int count, std::vector<MeshNode>& nodes) {
    std::vector<int> order((size_t)count);
    std::vector<Vec3> centre((size_t)count);
    for (int t = 0; t < count; ++t) {
        order[t] = t;
        Vec3 c[3];
        m.corners(t, c);
        centre[t] = (c[0] + c[1] + c[2]) * (1.0f / 3.0f);
    }
    nodes.assign(1, MeshNode{});
    struct Job {
        int node, first, count;
    };
    std::vector<Job> jobs{ { 0, 0, count } };
    std::vector<std::pair<float, int>> ranked;
    while (!jobs.empty()) {
        const Job j = jobs.back();
        jobs.pop_back();
        MeshNode& n = nodes[j.node];
        Vec3 c[3];
        m.corners(order[j.first], c);
        n.lo = n.hi = c[0];
        for (int i = j.first; i < j.first + j.count; ++i) {
            m.corners(order[i], c);
            for (const Vec3& p : c) {
                n.lo = minVec(n.lo, p);
                n.hi = maxVec(n.hi, p);
            }
        }
        if (j.count <= kLeafTriangles) {
            n.first = j.first;
            n.count = j.count;
            continue;
        }
        Vec3 lo = centre[order[j.first]], hi = lo;
        for (int i = j.first; i < j.first + j.count; ++i) {
            lo = minVec(lo, centre[order[i]]);
            hi = maxVec(hi, centre[order[i]]);
        }
        const Vec3 spread = hi - lo;
        const int axis = spread.x >= spread.y && spread.x >= spread.z ? 0 : spread.y >= spread.z ? 1 : 2;
        ranked.clear();
        for (int i = j.first; i < j.first + j.count; ++i) { ranked.push_back({ comp(centre[order[i]], axis), order[i] }); }
        std::sort(ranked.begin(), ranked.end());
        for (int i = 0; i < j.count; ++i) { order[j.first + i] = ranked[i].second; }
        const int child = (int)nodes.size();
        nodes.push_back(MeshNode{});
        nodes.push_back(MeshNode{});
        nodes[j.node].first = child;
        nodes[j.node].count = 0;
        const int half = j.count / 2;
        // The second half waits under the first, so the first half's whole subtree is numbered first.
        jobs.push_back({ child + 1, j.first + half, j.count - half });
        jobs.push_back({ child, j.first, half });
    }
    return order;
}

}  // namespace mesh

// TriangleMesh::TriangleMesh (src/mesh.cpp:122-245): equal vertices merged, triangles that are invalid,
// repeat a vertex or are slivers dropped, vertices renumbered in order of first use by a kept triangle,
// normals, edge flags, the tree, and the triangles stored in the tree's order.
inline HostMesh buildMesh(const std::vector<Vec3>& vertices, const std::vector<uint32_t>& indices) {
    using namespace mesh;
    HostMesh m;
    const std::vector<uint32_t> rep = mergeEqual(vertices);
    std::vector<uint32_t> number(vertices.size(), kUnset);
    std::vector<uint32_t> tri;
    for (size_t t = 0; t + 2 < indices.size(); t += 3) {
        uint32_t c[3];
        bool ok = true;
        for (int k = 0; k < 3 && ok; ++k) {
            ok = indices[t + k] < vertices.size() && rep[indices[t + k]] != kUnset;
            if (ok) { c[k] = rep[indices[t + k]]; }
        }
        if (!ok || c[0] == c[1] || c[1] == c[2] || c[2] == c[0]) { continue; }
        if (sliver(vertices[c[0]], vertices[c[1]], vertices[c[2]])) { continue; }
        for (uint32_t x : c) {
            if (number[x] == kUnset) {
                number[x] = (uint32_t)m.vertices.size();
                m.vertices.push_back(vertices[x]);
            }
            tri.push_back(number[x]);
        }
    }
    const int count = (int)tri.size() / 3;
    if (count == 0) { return m; }

    std::vector<Vec3> normals((size_t)count);
    for (int t = 0; t < count; ++t) {
        const Vec3& a = m.vertices[tri[3 * t]];
        const Vec3& b = m.vertices[tri[3 * t + 1]];
        const Vec3& c = m.vertices[tri[3 * t + 2]];
        normals[t] = normalize(cross(b - a, c - a));
    }
    const std::vector<uint8_t> flags = edgeFlagsOf(m.vertices, tri, normals);

    m.indices = tri;
    const std::vector<int> order = buildTree(m, count, m.nodes);
    m.normals.resize((size_t)count);
    m.edges.resize((size_t)count);
    for (int i = 0; i < count; ++i) {
        const int t = order[i];
        for (int k = 0; k < 3; ++k) { m.indices[3 * i + k] = tri[3 * t + k]; }
        m.normals[i] = normals[t];
        m.edges[i] = flags[t];
    }
    return m;
}

}  // namespace tfb
