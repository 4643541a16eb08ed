// Triangle meshes built on the host as the reference builds them (src/mesh.cpp:122-245): duplicate
// vertices merged, degenerate and sliver triangles dropped, per-triangle normals, per-edge flags saying
// which side of an edge may give a contact its own normal, and a bounding-volume tree split at the median
// of the widest spread of triangle centers, its leaves' triangles stored in tree order. The same float
// operations in the same order, host code compiled without contraction, so the device collides against
// the reference's triangles, in its order.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
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

constexpr int kLeafSize = 4;
constexpr float kFlatEdge = 0.087f;  // sine below which a folding neighbor leaves an edge without a normal
constexpr float kSliver = 1e-3f;     // sine of a triangle's widest corner below which it is dropped

inline bool finite3(const Vec3& v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }

inline bool lessXyz(const Vec3& a, const Vec3& b) {
    if (a.x != b.x) { return a.x < b.x; }
    if (a.y != b.y) { return a.y < b.y; }
    return a.z < b.z;
}

inline float axisOf(const Vec3& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

// src/mesh.cpp:73-82.
inline uint8_t edgeFlags(const Vec3& a, const Vec3& b, const Vec3& normal, const Vec3& far) {
    const Vec3 e = normalize(b - a);
    const Vec3 r = far - a;
    const float reach = length(r - e * dot(r, e));
    const float rise = dot(normal, r);
    uint8_t flags = 0;
    if (rise < -kFlatEdge * reach) { flags |= 1; }
    if (rise > kFlatEdge * reach) { flags |= 8; }
    return flags;
}

// The tree over triangles in `order`, node by node (src/mesh.cpp:28-70).
struct TreeBuilder {
    HostMesh& d;
    std::vector<int> order;
    std::vector<Vec3> centers;

    void fit(MeshNode& n, int first, int count) {
        Vec3 c[3];
        d.corners(order[first], c);
        n.lo = n.hi = c[0];
        for (int i = first; i < first + count; ++i) {
            d.corners(order[i], c);
            for (const Vec3& v : c) {
                n.lo = minVec(n.lo, v);
                n.hi = maxVec(n.hi, v);
            }
        }
    }

    void build(int node, int first, int count) {
        fit(d.nodes[node], first, count);
        if (count <= kLeafSize) {
            d.nodes[node].first = first;
            d.nodes[node].count = count;
            return;
        }
        Vec3 lo = centers[order[first]], hi = lo;
        for (int i = first; i < first + count; ++i) {
            lo = minVec(lo, centers[order[i]]);
            hi = maxVec(hi, centers[order[i]]);
        }
        const Vec3 spread = hi - lo;
        const int axis = spread.x >= spread.y && spread.x >= spread.z ? 0 : spread.y >= spread.z ? 1 : 2;
        std::sort(order.begin() + first, order.begin() + first + count, [&](int a, int b) {
            const float ca = axisOf(centers[a], axis), cb = axisOf(centers[b], axis);
            return ca != cb ? ca < cb : a < b;
        });
        const int child = (int)d.nodes.size();
        d.nodes.push_back(MeshNode{});
        d.nodes.push_back(MeshNode{});
        d.nodes[node].first = child;
        d.nodes[node].count = 0;
        const int half = count / 2;
        build(child, first, half);
        build(child + 1, first + half, count - half);
    }
};

}

// TriangleMesh::TriangleMesh (src/mesh.cpp:122-245).
inline HostMesh buildMesh(const std::vector<Vec3>& vertices, const std::vector<uint32_t>& indices) {
    using namespace mesh;
    HostMesh d;
    std::vector<uint32_t> sorted;
    sorted.reserve(vertices.size());
    for (uint32_t i = 0; i < (uint32_t)vertices.size(); ++i) {
        if (finite3(vertices[i])) { sorted.push_back(i); }
    }
    std::sort(sorted.begin(), sorted.end(), [&](uint32_t a, uint32_t b) {
        if (lessXyz(vertices[a], vertices[b])) { return true; }
        if (lessXyz(vertices[b], vertices[a])) { return false; }
        return a < b;
    });
    // Every vertex maps to the first of the vertices equal to it.
    std::vector<uint32_t> first(vertices.size(), UINT32_MAX);
    for (size_t i = 0; i < sorted.size(); ++i) {
        const bool same = i > 0 && !lessXyz(vertices[sorted[i - 1]], vertices[sorted[i]]);
        first[sorted[i]] = same ? first[sorted[i - 1]] : sorted[i];
    }

    std::vector<uint32_t> remap(vertices.size(), UINT32_MAX);
    std::vector<uint32_t> tris;
    for (size_t t = 0; t + 2 < indices.size(); t += 3) {
        uint32_t v[3];
        bool valid = true;
        for (int k = 0; k < 3; ++k) {
            if (indices[t + k] >= vertices.size() || first[indices[t + k]] == UINT32_MAX) {
                valid = false;
                break;
            }
            v[k] = first[indices[t + k]];
        }
        if (!valid || v[0] == v[1] || v[1] == v[2] || v[2] == v[0]) { continue; }
        int wide = 0;
        float longest = 0.0f;
        for (int k = 0; k < 3; ++k) {
            const float opposite = lengthSquared(vertices[v[(k + 2) % 3]] - vertices[v[(k + 1) % 3]]);
            if (opposite > longest) {
                longest = opposite;
                wide = k;
            }
        }
        const Vec3 e1 = vertices[v[(wide + 1) % 3]] - vertices[v[wide]];
        const Vec3 e2 = vertices[v[(wide + 2) % 3]] - vertices[v[wide]];
        if (!(lengthSquared(cross(e1, e2)) > kSliver * kSliver * lengthSquared(e1) * lengthSquared(e2))) { continue; }
        for (int k = 0; k < 3; ++k) {
            if (remap[v[k]] == UINT32_MAX) {
                remap[v[k]] = (uint32_t)d.vertices.size();
                d.vertices.push_back(vertices[v[k]]);
            }
            tris.push_back(remap[v[k]]);
        }
    }
    const int count = (int)tris.size() / 3;
    if (count == 0) { return d; }

    std::vector<Vec3> normals((size_t)count);
    std::vector<uint8_t> edges((size_t)count, 0);
    for (int t = 0; t < count; ++t) {
        const Vec3 a = d.vertices[tris[3 * t]], b = d.vertices[tris[3 * t + 1]], c = d.vertices[tris[3 * t + 2]];
        normals[t] = normalize(cross(b - a, c - a));
    }

    // Edges by their two vertices: one with exactly one neighbor takes its own normal only on the side
    // where the neighbor folds away; an open edge, or one shared by more than two triangles, on both.
    struct EdgeRef {
        uint64_t key;
        int tri;
        int corner;
    };
    std::vector<EdgeRef> refs;
    refs.reserve(tris.size());
    for (int t = 0; t < count; ++t) {
        for (int k = 0; k < 3; ++k) {
            const uint32_t a = tris[3 * t + k], b = tris[3 * t + (k + 1) % 3];
            refs.push_back({ ((uint64_t)std::min(a, b) << 32) | std::max(a, b), t, k });
        }
    }
    std::sort(refs.begin(), refs.end(), [](const EdgeRef& x, const EdgeRef& y) {
        if (x.key != y.key) { return x.key < y.key; }
        return x.tri != y.tri ? x.tri < y.tri : x.corner < y.corner;
    });
    for (size_t i = 0; i < refs.size();) {
        size_t j = i;
        while (j < refs.size() && refs[j].key == refs[i].key) { ++j; }
        for (size_t k = i; k < j; ++k) {
            const EdgeRef& r = refs[k];
            if (j - i != 2) {
                edges[r.tri] |= (uint8_t)(9u << r.corner);
                continue;
            }
            const EdgeRef& o = refs[k == i ? i + 1 : i];
            const Vec3 a = d.vertices[tris[3 * r.tri + r.corner]];
            const Vec3 b = d.vertices[tris[3 * r.tri + (r.corner + 1) % 3]];
            const Vec3 far = d.vertices[tris[3 * o.tri + (o.corner + 2) % 3]];
            edges[r.tri] |= (uint8_t)(edgeFlags(a, b, normals[r.tri], far) << r.corner);
        }
        i = j;
    }

    d.indices = tris;
    TreeBuilder builder{ d, std::vector<int>((size_t)count), std::vector<Vec3>((size_t)count) };
    for (int t = 0; t < count; ++t) {
        builder.order[t] = t;
        Vec3 c[3];
        d.corners(t, c);
        builder.centers[t] = (c[0] + c[1] + c[2]) * (1.0f / 3.0f);
    }
    d.nodes.reserve(2 * (size_t)count / kLeafSize + 1);
    d.nodes.push_back(MeshNode{});
    builder.build(0, 0, count);

    // Triangles in tree order.
    d.indices.resize(tris.size());
    d.normals.resize((size_t)count);
    d.edges.resize((size_t)count);
    for (int i = 0; i < count; ++i) {
        const int t = builder.order[i];
        for (int k = 0; k < 3; ++k) { d.indices[3 * i + k] = tris[3 * t + k]; }
        d.normals[i] = normals[t];
        d.edges[i] = edges[t];
    }
    return d;
}

}
