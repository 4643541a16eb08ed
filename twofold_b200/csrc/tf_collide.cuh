// Narrowphase for 3D convex pairs: half-space, sphere and polyhedron manifolds.
//
// One thread collides one shape pair. Each function restates the reference function it names
// (src/collide3d.cpp, src/distance.cpp) with the same arithmetic in the same order and the same strict
// tie-breaking in index order, so manifolds, point counts and feature ids come out bit-identical. The
// reference's 4-wide lane scans (leastAbove, the queryEdges arc tests) are order-preserving scans here:
// their results do not depend on the lane width (src/collide3d.cpp:110-130, 249-270).
//
// A polyhedron seen in the other shape's frame is not copied: its vertices, normals, offsets and arcs are
// recomputed from the shared tables when read, which yields the same bits as the reference's stored copy
// (src/collide3d.cpp:48-76).
#pragma once

#include "tf_body.cuh"

namespace tfb {

constexpr float kParallelEdges = 0.05f;
constexpr int kMaxClip = 64;      // clip polygon vertices
constexpr int kMaxReduce = 64;    // candidate manifold points
constexpr int kMaxEdges = 192;    // polyhedron edges
constexpr int kMaxVerts = 128;    // polyhedron vertices

struct MPoint {
    Vec3 position;
    float separation;
    float predicted;
};

struct Manifold {
    Vec3 normal;
    MPoint points[4];
    int count;
    int featKind, featA, featB;
};

// Velocities of the two bodies over the coming step (src/internal.h:354-373).
struct Motion {
    Vec3 linearA, angularA, centerA;
    Vec3 linearB, angularB, centerB;
    float dt;
    bool fast;

    TF_HD float predict(const Vec3& p, const Vec3& n, float separation) const {
        const Vec3 va = linearA + cross(angularA, p - centerA);
        const Vec3 vb = linearB + cross(angularB, p - centerB);
        return separation + dt * dot(n, vb - va);
    }
    TF_HD Motion swapped() const { return { linearB, angularB, centerB, linearA, angularA, centerA, dt, fast }; }
};

// Face and edge numbering of every box (src/collide3d.cpp:456-476), filled on the host.
struct BoxTopology {
    int face[3][2];
    int edge[3][2][2];
};

// A polyhedron in the frame of the pair's first shape: its own frame, or transformed by (r, p).
struct FramePoly {
    const PolyTables* t;
    const DPoly* P;
    bool moved;
    Mat3 r;
    Vec3 p;
    Vec3 centroid, lo, hi;

    TF_HD int vertexCount() const { return P->vCount; }
    TF_HD int faceCount() const { return P->fCount; }
    TF_HD int edgeCount() const { return P->eCount; }
    TF_HD Vec3 v(int k) const {
        const Vec3 x = t->verts[P->vFirst + k];
        return moved ? r * x + p : x;
    }
    TF_HD Vec3 n(int i) const {
        const Vec3 x = t->normals[P->fFirst + i];
        return moved ? r * x : x;
    }
    TF_HD float d(int i) const {
        if (!moved) { return t->offsets[P->fFirst + i]; }
        return dot(n(i), v(index(face(i).first)));
    }
    TF_HD Vec3 arc(int i) const {
        const Vec3 x = t->arcs[P->eFirst + i];
        return moved ? r * x : x;
    }
    TF_HD DFace face(int i) const { return t->faces[P->fFirst + i]; }
    TF_HD int index(int k) const { return t->indices[P->iFirst + k]; }
    TF_HD DEdge edge(int i) const { return t->edges[P->eFirst + i]; }
};

TF_HD FramePoly ownFrame(const PolyTables& t, int poly) {
    FramePoly f;
    f.t = &t;
    f.P = &t.polys[poly];
    f.moved = false;
    f.r = mid();
    f.p = zero3();
    f.centroid = f.P->centroid;
    f.lo = f.P->lo;
    f.hi = f.P->hi;
    return f;
}

TF_HD FramePoly otherFrame(const PolyTables& t, int poly, const Transform& xf) {
    FramePoly f;
    f.t = &t;
    f.P = &t.polys[poly];
    f.moved = true;
    f.r = toMat3(xf.q);
    f.p = xf.p;
    f.lo = f.hi = f.r * t.verts[f.P->vFirst] + xf.p;
    for (int i = 0; i < f.P->vCount; ++i) {
        const Vec3 w = f.r * t.verts[f.P->vFirst + i] + xf.p;
        f.lo = minVec(f.lo, w);
        f.hi = maxVec(f.hi, w);
    }
    f.centroid = f.r * f.P->centroid + xf.p;
    return f;
}

// src/collide3d.cpp:77-88.
TF_HD int supportFace(const FramePoly& p, const Vec3& n) {
    int best = 0;
    float most = dot(p.n(0), n);
    for (int i = 1; i < p.faceCount(); ++i) {
        const float d = dot(p.n(i), n);
        if (d > most) {
            most = d;
            best = i;
        }
    }
    return best;
}

// minf of s and every dot of n with a vertex, scanned in vertex order; the first dot at or below bound ends
// the scan and is the result (src/collide3d.cpp:110-130).
TF_HD float leastAbove(const FramePoly& b, const Vec3& n, float s, float bound) {
    float low = s;
    for (int k = 0; k < b.vertexCount(); ++k) {
        const float d = dot(n, b.v(k));
        if (!(d > bound) && d == d) { return d; }
        low = minf(low, d);
    }
    return low;
}

struct FaceQuery {
    int index;
    float separation;
};

struct EdgeQuery {
    int a, b;
    float separation;
    Vec3 axis;
    bool pruned;
};

TF_HD FaceQuery noFace() { return { -1, -FLT_MAX }; }
TF_HD EdgeQuery noEdge() { return { -1, -1, -FLT_MAX, zero3(), false }; }

// src/collide3d.cpp:146-179.
TF_HD FaceQuery queryFaces(const FramePoly& a, const FramePoly& b, float limit) {
    const Vec3 toward = b.centroid - a.centroid;
    int deep = 0;
    float least = dot(b.v(0), toward);
    for (int k = 1; k < b.vertexCount(); ++k) {
        const float d = dot(b.v(k), toward);
        if (d < least) {
            least = d;
            deep = k;
        }
    }
    const int first = supportFace(a, toward);
    FaceQuery q = noFace();
    const Vec3 deepV = b.v(deep);
    for (int j = -1; j < a.faceCount(); ++j) {
        if (j == first) { continue; }
        const int i = j < 0 ? first : j;
        const Vec3 n = a.n(i);
        const float ad = a.d(i);
        const float bound = q.separation + ad;
        float s = dot(n, deepV);
        if (s > bound) { s = leastAbove(b, n, s, bound); }
        s -= ad;
        if (s > q.separation) {
            q.separation = s;
            q.index = i;
            if (s > limit) { break; }
        }
    }
    return q;
}

// The edges of p not wholly past one side of the box (src/collide3d.cpp:183-197).
TF_HD int edgesInBox(const FramePoly& p, const Vec3& lo, const Vec3& hi, uint8_t* past, int16_t* out) {
    const int nv = p.vertexCount() < kMaxVerts ? p.vertexCount() : kMaxVerts;
    for (int k = 0; k < nv; ++k) {
        const Vec3 v = p.v(k);
        past[k] = (uint8_t)((v.x > hi.x) | (v.x < lo.x) << 1 | (v.y > hi.y) << 2 | (v.y < lo.y) << 3 |
                            (v.z > hi.z) << 4 | (v.z < lo.z) << 5);
    }
    int n = 0;
    for (int i = 0; i < p.edgeCount() && n < kMaxEdges; ++i) {
        const DEdge e = p.edge(i);
        if (past[e.v0] & past[e.v1]) { continue; }
        out[n++] = (int16_t)i;
    }
    return n;
}

// src/collide3d.cpp:219-231.
TF_HD bool edgeAxis(const FramePoly& a, const FramePoly& b, int i, int j, Vec3& axis, float& separation) {
    const DEdge ea = a.edge(i);
    const DEdge eb = b.edge(j);
    const Vec3 pa = a.v(ea.v0);
    const Vec3 pb = b.v(eb.v0);
    axis = cross(a.v(ea.v1) - pa, b.v(eb.v1) - pb);
    const float len = length(axis);
    if (len < kParallelEdges * ea.length * eb.length) { return false; }
    axis = axis / len;
    if (dot(axis, pa - a.centroid) < 0.0f) { axis = -axis; }
    separation = dot(axis, pb - pa);
    return true;
}

// src/collide3d.cpp:236-273.
TF_HD EdgeQuery queryEdges(const FramePoly& a, const FramePoly& b, float reach) {
    EdgeQuery q = noEdge();
    const Vec3 grow{ reach, reach, reach };
    const Vec3 lo = maxVec(a.lo, b.lo) - grow, hi = minVec(a.hi, b.hi) + grow;
    uint8_t past[kMaxVerts];
    int16_t nearA[kMaxEdges], nearB[kMaxEdges];
    const int na = edgesInBox(a, lo, hi, past, nearA);
    const int nb = edgesInBox(b, lo, hi, past, nearB);
    q.pruned = na < a.edgeCount() || nb < b.edgeCount();
    for (int x = 0; x < na; ++x) {
        const int i = nearA[x];
        const DEdge ea = a.edge(i);
        const Vec3 ua = a.n(ea.f0), va = a.n(ea.f1), ga = a.arc(i);
        for (int y = 0; y < nb; ++y) {
            const int j = nearB[y];
            const DEdge eb = b.edge(j);
            const float cba = dot(b.n(eb.f0), ga), dba = dot(b.n(eb.f1), ga);
            const Vec3 gb = b.arc(j);
            const float bdc = dot(va, gb);
            if (!((0.0f > cba * dba) & (0.0f > dot(ua, gb) * bdc) & (0.0f > cba * bdc))) { continue; }
            Vec3 axis;
            float s;
            if (!edgeAxis(a, b, i, j, axis, s)) { continue; }
            if (s > q.separation) {
                q.separation = s;
                q.a = i;
                q.b = j;
                q.axis = axis;
            }
        }
    }
    return q;
}

// src/collide3d.cpp:275-288. Returns the new vertex count.
TF_HD int clipPolygon(Vec3* poly, int count, Vec3* scratch, const Vec3& n, const Vec3& origin) {
    if (count == 0) { return 0; }
    int out = 0;
    for (int i = 0; i < count; ++i) {
        const Vec3 p = poly[i];
        const Vec3 q = poly[(i + 1) % count];
        const float dp = dot(n, p - origin);
        const float dq = dot(n, q - origin);
        if (dp <= 0.0f && out < kMaxClip) { scratch[out++] = p; }
        if ((dp <= 0.0f) != (dq <= 0.0f) && out < kMaxClip) { scratch[out++] = p + (q - p) * (dp / (dp - dq)); }
    }
    for (int i = 0; i < out; ++i) { poly[i] = scratch[i]; }
    return out;
}

// Picks up to four points: deepest predicted, farthest, largest area, farthest outside, then the deepest
// of the rest (src/collide3d.cpp:1497-1575).
TF_HD void reduceManifold(const MPoint* pts, int n, const Vec3& normal, float band, Manifold& m, float tie, bool fast) {
    m.normal = normal;
    m.count = 0;
    if (n <= 4) {
        for (int i = 0; i < n; ++i) { m.points[m.count++] = pts[i]; }
        return;
    }
    int i0 = 0;
    for (int i = 1; i < n; ++i) {
        if (pts[i].predicted < pts[i0].predicted) { i0 = i; }
    }
    for (int i = 0; i < i0; ++i) {
        if (pts[i].predicted <= pts[i0].predicted + tie) {
            i0 = i;
            break;
        }
    }
    const Vec3 p0 = pts[i0].position;
    const float limit = fast ? maxf(pts[i0].predicted + band, 0.0f) : pts[i0].predicted + band;
    int chosen[4] = { i0, i0, i0, i0 };
    auto used = [&](int i) { return i == chosen[0] || i == chosen[1] || i == chosen[2] || i == chosen[3]; };
    m.points[m.count++] = pts[i0];

    int i1 = n;
    float best = 0.0f;
    for (int i = 0; i < n; ++i) {
        if (pts[i].predicted > limit) { continue; }
        const float d = lengthSquared(pts[i].position - p0);
        if (d > best) {
            best = d;
            i1 = i;
        }
    }
    int i2 = n;
    float area = 0.0f;
    if (i1 < n) {
        chosen[1] = i1;
        m.points[m.count++] = pts[i1];
        const Vec3 p1 = pts[i1].position;
        for (int i = 0; i < n; ++i) {
            if (used(i) || pts[i].predicted > limit) { continue; }
            const float a = dot(cross(p1 - p0, pts[i].position - p0), normal);
            if (fabsf(a) > fabsf(area)) {
                area = a;
                i2 = i;
            }
        }
    }
    if (i2 < n) {
        chosen[2] = i2;
        m.points[m.count++] = pts[i2];
        const float sign = area < 0.0f ? -1.0f : 1.0f;
        const Vec3 tri[3] = { p0, m.points[1].position, pts[i2].position };
        int i3 = n;
        float outside = 0.0f;
        for (int i = 0; i < n; ++i) {
            if (used(i) || pts[i].predicted > limit) { continue; }
            for (int e = 0; e < 3; ++e) {
                const Vec3& a = tri[e];
                const Vec3& b = tri[(e + 1) % 3];
                const float s = -sign * dot(cross(b - a, pts[i].position - a), normal);
                if (s > outside) {
                    outside = s;
                    i3 = i;
                }
            }
        }
        if (i3 < n) {
            chosen[3] = i3;
            m.points[m.count++] = pts[i3];
        }
    }
    while (m.count < 4) {
        int next = n;
        for (int i = 0; i < n; ++i) {
            if (used(i)) { continue; }
            if (next == n || pts[i].predicted < pts[next].predicted) { next = i; }
        }
        if (next == n) { break; }
        chosen[m.count] = next;
        m.points[m.count++] = pts[next];
    }
}

// src/collide3d.cpp:296-344.
TF_HD void faceContact(const FramePoly& ref, int refFace, const FramePoly& inc, bool flip, const Transform& xf,
                       float margin, float band, const Motion& motion, Manifold& m) {
    const Vec3 refN = ref.n(refFace);
    const float refD = ref.d(refFace);
    const Vec3 worldN = rotate(xf.q, refN);

    int incFace = 0;
    float minDot = FLT_MAX;
    for (int i = 0; i < inc.faceCount(); ++i) {
        const float d = dot(inc.n(i), refN);
        if (d < minDot) {
            minDot = d;
            incFace = i;
        }
    }
    Vec3 poly[kMaxClip], scratch[kMaxClip];
    const DFace fi = inc.face(incFace);
    int count = 0;
    for (int k = 0; k < fi.count && count < kMaxClip; ++k) { poly[count++] = inc.v(inc.index(fi.first + k)); }
    const DFace fr = ref.face(refFace);
    for (int k = 0; k < fr.count; ++k) {
        const Vec3 a = ref.v(ref.index(fr.first + k));
        const Vec3 b = ref.v(ref.index(fr.first + (k + 1) % fr.count));
        count = clipPolygon(poly, count, scratch, cross(b - a, refN), a);
    }
    MPoint pts[kMaxClip];
    int np = 0;
    for (int k = 0; k < count; ++k) {
        const Vec3 p = poly[k];
        const float s = dot(refN, p) - refD;
        if (s > margin) { continue; }
        const Vec3 w = apply(xf, p);
        pts[np++] = { w - worldN * (0.5f * s), s, motion.predict(w, worldN, s) };
    }
    if (np == 0) {
        Vec3 deepest = inc.v(0);
        for (int k = 1; k < inc.vertexCount(); ++k) {
            const Vec3 vk = inc.v(k);
            if (dot(refN, vk) < dot(refN, deepest)) { deepest = vk; }
        }
        const float s = dot(refN, deepest) - refD;
        if (s <= margin) {
            const Vec3 w = apply(xf, deepest);
            pts[np++] = { w - worldN * (0.5f * s), s, motion.predict(w, worldN, s) };
        }
    }
    reduceManifold(pts, np, flip ? -worldN : worldN, band, m, 0.0f, motion.fast);
}

// src/collide3d.cpp:346-375.
TF_HD void closestOnSegments(const Vec3& p1, const Vec3& q1, const Vec3& p2, const Vec3& q2, Vec3& c1, Vec3& c2) {
    const Vec3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    const float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    float s = 0.0f, t = 0.0f;
    if (a <= FLT_EPSILON && e <= FLT_EPSILON) {
        c1 = p1;
        c2 = p2;
        return;
    }
    if (a <= FLT_EPSILON) {
        t = minf(maxf(f / e, 0.0f), 1.0f);
    } else {
        const float c = dot(d1, r);
        if (e <= FLT_EPSILON) {
            s = minf(maxf(-c / a, 0.0f), 1.0f);
        } else {
            const float b = dot(d1, d2);
            const float denom = a * e - b * b;
            s = denom != 0.0f ? minf(maxf((b * f - c * e) / denom, 0.0f), 1.0f) : 0.0f;
            t = (b * s + f) / e;
            if (t < 0.0f) {
                t = 0.0f;
                s = minf(maxf(-c / a, 0.0f), 1.0f);
            } else if (t > 1.0f) {
                t = 1.0f;
                s = minf(maxf((b - c) / a, 0.0f), 1.0f);
            }
        }
    }
    c1 = p1 + d1 * s;
    c2 = p2 + d2 * t;
}

// src/collide3d.cpp:377-414.
TF_HD void edgeContact(const FramePoly& a, const FramePoly& b, const EdgeQuery& eq, const Transform& xf, float margin,
                       float band, const Motion& motion, Manifold& m) {
    const Vec3 n = eq.axis;
    const Vec3 worldN = rotate(xf.q, n);
    const int fa = supportFace(a, n);
    const Vec3 na = a.n(fa);
    const float cosA = dot(na, n);
    MPoint pts[kMaxClip];
    int np = 0;
    if (cosA > 0.0f) {
        Vec3 poly[kMaxClip], scratch[kMaxClip];
        const DFace fi = b.face(supportFace(b, -n));
        int count = 0;
        for (int k = 0; k < fi.count && count < kMaxClip; ++k) { poly[count++] = b.v(b.index(fi.first + k)); }
        const DFace fr = a.face(fa);
        for (int k = 0; k < fr.count; ++k) {
            const Vec3 p = a.v(a.index(fr.first + k));
            const Vec3 q = a.v(a.index(fr.first + (k + 1) % fr.count));
            count = clipPolygon(poly, count, scratch, cross(q - p, n), p);
        }
        const float ad = a.d(fa);
        for (int k = 0; k < count; ++k) {
            const Vec3 p = poly[k];
            const float s = maxf((dot(na, p) - ad) / cosA, eq.separation);
            if (s > margin) { continue; }
            const Vec3 w = apply(xf, p);
            pts[np++] = { w - worldN * (0.5f * s), s, motion.predict(w, worldN, s) };
        }
    }
    if (np >= 2) {
        reduceManifold(pts, np, worldN, band, m, 0.0f, motion.fast);
        return;
    }
    const DEdge ea = a.edge(eq.a);
    const DEdge eb = b.edge(eq.b);
    Vec3 c1, c2;
    closestOnSegments(a.v(ea.v0), a.v(ea.v1), b.v(eb.v0), b.v(eb.v1), c1, c2);
    m.normal = worldN;
    m.points[0] = { apply(xf, (c1 + c2) * 0.5f), eq.separation, 0.0f };
    m.count = 1;
}

// src/collide3d.cpp:425-439.
TF_HD EdgeQuery reusedEdges(const FramePoly& a, const FramePoly& b, int kind, int fa, int fb) {
    EdgeQuery q = noEdge();
    if (kind != kFeatEdges) { return q; }
    const DEdge ea = a.edge(fa);
    const DEdge eb = b.edge(fb);
    const Vec3 ga = a.arc(fa), gb = b.arc(fb);
    const float cba = dot(b.n(eb.f0), ga), dba = dot(b.n(eb.f1), ga);
    const float adc = dot(a.n(ea.f0), gb), bdc = dot(a.n(ea.f1), gb);
    if (cba * dba >= 0.0f || adc * bdc >= 0.0f || cba * bdc >= 0.0f) { return q; }
    if (edgeAxis(a, b, fa, fb, q.axis, q.separation)) {
        q.a = fa;
        q.b = fb;
    }
    return q;
}

// The face and edge queries of two boxes in closed form, b in the frame of a (src/collide3d.cpp:481-596).
TF_HD bool boxQueries(const BoxTopology& topology, const Vec3& halfA, const Vec3& halfB, const Transform& x,
                      float margin, FaceQuery& fa, FaceQuery& fb, EdgeQuery& eq, bool& unsure) {
    const Mat3 rot = toMat3(x.q);
    const float r[3][3] = { { rot.r[0].x, rot.r[0].y, rot.r[0].z },
                            { rot.r[1].x, rot.r[1].y, rot.r[1].z },
                            { rot.r[2].x, rot.r[2].y, rot.r[2].z } };
    float ar[3][3];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) { ar[i][j] = fabsf(r[i][j]); }
    }
    const float t[3] = { x.p.x, x.p.y, x.p.z };
    const float ha[3] = { halfA.x, halfA.y, halfA.z }, hb[3] = { halfB.x, halfB.y, halfB.z };

    int faceA = 0, faceB = 0;
    for (int i = 0; i < 3; ++i) {
        const float s = fabsf(t[i]) - ha[i] - (hb[0] * ar[i][0] + hb[1] * ar[i][1] + hb[2] * ar[i][2]);
        if (s > margin) { return false; }
        if (s > fa.separation) {
            fa.separation = s;
            faceA = i;
        }
    }
    float tb[3];
    for (int j = 0; j < 3; ++j) {
        tb[j] = t[0] * r[0][j] + t[1] * r[1][j] + t[2] * r[2][j];
        const float s = fabsf(tb[j]) - hb[j] - (ha[0] * ar[0][j] + ha[1] * ar[1][j] + ha[2] * ar[2][j]);
        if (s > margin) { return false; }
        if (s > fb.separation) {
            fb.separation = s;
            faceB = j;
        }
    }

    int edgeI = -1, edgeJ = -1;
    float edgeSign = 1.0f, edgeLength = 1.0f;
    for (int i = 0; i < 3; ++i) {
        const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
        for (int j = 0; j < 3; ++j) {
            const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            const float l1 = -r[i2][j], l2 = r[i1][j];
            if (l1 == 0.0f || l2 == 0.0f || r[i][j1] == 0.0f || r[i][j2] == 0.0f) { continue; }
            const float len = sqrtf(l1 * l1 + l2 * l2);
            if (len < kParallelEdges) { continue; }
            const float d = t[i1] * l1 + t[i2] * l2;
            const float ra = ha[i1] * ar[i2][j] + ha[i2] * ar[i1][j];
            const float rb = hb[j1] * ar[i][j2] + hb[j2] * ar[i][j1];
            const float s = (fabsf(d) - ra - rb) / len;
            if (s > margin) { return false; }
            if (s > eq.separation) {
                eq.separation = s;
                edgeI = i;
                edgeJ = j;
                edgeSign = d < 0.0f ? -1.0f : 1.0f;
                edgeLength = len;
            }
        }
    }

    fa.index = topology.face[faceA][t[faceA] >= 0.0f];
    fb.index = topology.face[faceB][tb[faceB] < 0.0f];
    if (edgeI >= 0) {
        const int i = edgeI, j = edgeJ;
        const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
        const float l1 = -r[i2][j] * edgeSign, l2 = r[i1][j] * edgeSign;
        float n[3];
        n[i] = 0.0f;
        n[i1] = l1 / edgeLength;
        n[i2] = l2 / edgeLength;
        eq.axis = { n[0], n[1], n[2] };
        const float m1 = r[i][j2] * edgeSign, m2 = -r[i][j1] * edgeSign;
        eq.a = topology.edge[i][l1 > 0.0f][l2 > 0.0f];
        eq.b = topology.edge[j][m1 < 0.0f][m2 < 0.0f];
    }

    unsure = false;
    const float gap = maxf(maxf(fa.separation, fb.separation), eq.separation);
    if (gap <= 0.0f) { return true; }
    if (edgeI >= 0 && gap == eq.separation) {
        const int i = edgeI, j = edgeJ;
        const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
        const float sideB1 = r[i][j2] * edgeSign < 0.0f ? hb[j1] : -hb[j1];
        const float sideB2 = -r[i][j1] * edgeSign < 0.0f ? hb[j2] : -hb[j2];
        float w[3];
        for (int k = 0; k < 3; ++k) { w[k] = -t[k] - sideB1 * r[k][j1] - sideB2 * r[k][j2]; }
        w[i1] += -r[i2][j] * edgeSign > 0.0f ? ha[i1] : -ha[i1];
        w[i2] += r[i1][j] * edgeSign > 0.0f ? ha[i2] : -ha[i2];
        const float b = r[i][j], f = w[0] * r[0][j] + w[1] * r[1][j] + w[2] * r[2][j];
        const float s = (b * f - w[i]) / (1.0f - b * b);
        unsure = fabsf(s) > ha[i] || fabsf(f + s * b) > hb[j];
    } else if (gap == fa.separation) {
        const int i = faceA;
        const float side = t[i] < 0.0f ? -1.0f : 1.0f;
        for (int k = 0; k < 3 && !unsure; ++k) {
            if (k == i) { continue; }
            float v = t[k];
            for (int j = 0; j < 3; ++j) { v += side * r[i][j] > 0.0f ? -hb[j] * r[k][j] : hb[j] * r[k][j]; }
            unsure = fabsf(v) > ha[k];
        }
    } else {
        const int j = faceB;
        const float side = tb[j] < 0.0f ? -1.0f : 1.0f;
        for (int k = 0; k < 3 && !unsure; ++k) {
            if (k == j) { continue; }
            float v = -tb[k];
            for (int i = 0; i < 3; ++i) { v += side * r[i][j] > 0.0f ? ha[i] * r[i][k] : -ha[i] * r[i][k]; }
            unsure = fabsf(v) > hb[k];
        }
    }
    return true;
}

// ---------------------------------------------------------------------------------------------------------
// GJK (src/distance.cpp): support points in float, simplex weights in double.

// A shape as GJK sees it (src/internal.h:203-211): points (with a rounding radius), a half-space, or a
// cylinder of radius rim and half height halfHeight about its local z.
struct Convex {
    const Vec3* points;
    int count;
    float radius;
    bool halfSpace;
    bool cylinder;
    float rim, halfHeight;
};

// src/shape.cpp:142-147: the point of a cylinder farthest along d, in its own frame.
TF_HD Vec3 cylinderSupport(float radius, float halfHeight, const Vec3& d) {
    const float z = d.z < 0.0f ? -halfHeight : halfHeight;
    const float side = sqrtf(d.x * d.x + d.y * d.y);
    if (side == 0.0f) { return Vec3{ 0.0f, 0.0f, z }; }
    return Vec3{ d.x * (radius / side), d.y * (radius / side), z };
}

struct GVertex {
    Vec3 a, b, w;
};

struct DPt {
    double x, y, z;
};

TF_HD DPt dpt(const Vec3& v) { return { (double)v.x, (double)v.y, (double)v.z }; }
TF_HD DPt operator+(const DPt& a, const DPt& b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
TF_HD DPt operator-(const DPt& a, const DPt& b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
TF_HD DPt operator*(const DPt& a, double s) { return { a.x * s, a.y * s, a.z * s }; }
TF_HD double dot(const DPt& a, const DPt& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
TF_HD DPt cross(const DPt& a, const DPt& b) {
    return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x };
}
TF_HD Vec3 toVec(const DPt& p) { return { (float)p.x, (float)p.y, (float)p.z }; }

struct Simplex {
    GVertex v[4];
    double u[4];
    int count;
};

TF_HD Vec3 gjkSupport(const Convex& c, const Transform& xf, const Vec3& d) {
    const Vec3 local = unrotate(xf.q, d);
    if (c.cylinder) { return apply(xf, cylinderSupport(c.rim, c.halfHeight, local)); }
    int best = 0;
    float most = dot(c.points[0], local);
    for (int i = 1; i < c.count; ++i) {
        const float s = dot(c.points[i], local);
        if (s > most) {
            most = s;
            best = i;
        }
    }
    return apply(xf, c.points[best]);
}

TF_HD void segmentWeights(const DPt& a, const DPt& b, double& ua, double& ub) {
    const DPt e = b - a;
    const double ee = dot(e, e);
    double t = 0.0;
    if (ee > 0.0) {
        t = -dot(a, e) / ee;
        t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
    }
    ua = 1.0 - t;
    ub = t;
}

// Ericson's closest point on a triangle as barycentric weights (src/distance.cpp:41-102).
TF_HD void triangleWeights(const DPt& a, const DPt& b, const DPt& c, double u[3]) {
    u[0] = u[1] = u[2] = 0.0;
    const DPt ab = b - a, ac = c - a;
    const double d1 = -dot(ab, a), d2 = -dot(ac, a);
    if (d1 <= 0.0 && d2 <= 0.0) {
        u[0] = 1.0;
        return;
    }
    const double d3 = -dot(ab, b), d4 = -dot(ac, b);
    if (d3 >= 0.0 && d4 <= d3) {
        u[1] = 1.0;
        return;
    }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        segmentWeights(a, b, u[0], u[1]);
        return;
    }
    const double d5 = -dot(ab, c), d6 = -dot(ac, c);
    if (d6 >= 0.0 && d5 <= d6) {
        u[2] = 1.0;
        return;
    }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        segmentWeights(a, c, u[0], u[2]);
        return;
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && d4 - d3 >= 0.0 && d5 - d6 >= 0.0) {
        segmentWeights(b, c, u[1], u[2]);
        return;
    }
    const double sum = va + vb + vc;
    if (sum > DBL_MIN) {
        u[0] = va / sum;
        u[1] = vb / sum;
        u[2] = vc / sum;
        return;
    }
    const DPt* p[3] = { &a, &b, &c };
    double best = DBL_MAX;
    for (int i = 0; i < 3; ++i) {
        const int j = (i + 1) % 3;
        double ui, uj;
        segmentWeights(*p[i], *p[j], ui, uj);
        const DPt q = *p[i] * ui + *p[j] * uj;
        if (dot(q, q) < best) {
            best = dot(q, q);
            u[0] = u[1] = u[2] = 0.0;
            u[i] = ui;
            u[j] = uj;
        }
    }
}

// src/distance.cpp:104-124.
TF_HD bool tetrahedronWeights(const DPt w[4], double u[4]) {
    const int faces[4][4] = { { 0, 1, 2, 3 }, { 0, 3, 1, 2 }, { 0, 2, 3, 1 }, { 1, 3, 2, 0 } };
    bool outside = false;
    double best = DBL_MAX;
    for (int k = 0; k < 4; ++k) {
        const int* f = faces[k];
        const DPt n = cross(w[f[1]] - w[f[0]], w[f[2]] - w[f[0]]);
        const DPt apex = w[f[3]] - w[f[0]];
        const double height = dot(apex, n);
        if (-dot(w[f[0]], n) * height > 0.0 && height * height > 1e-8 * dot(n, n) * dot(apex, apex)) { continue; }
        outside = true;
        double t[3];
        triangleWeights(w[f[0]], w[f[1]], w[f[2]], t);
        const DPt q = w[f[0]] * t[0] + w[f[1]] * t[1] + w[f[2]] * t[2];
        if (dot(q, q) < best) {
            best = dot(q, q);
            u[0] = u[1] = u[2] = u[3] = 0.0;
            for (int i = 0; i < 3; ++i) { u[f[i]] = t[i]; }
        }
    }
    return outside;
}

// src/distance.cpp:127-147.
TF_HD bool solveSimplex(Simplex& s) {
    double u[4] = { 1.0, 0.0, 0.0, 0.0 };
    if (s.count == 2) {
        segmentWeights(dpt(s.v[0].w), dpt(s.v[1].w), u[0], u[1]);
    } else if (s.count == 3) {
        triangleWeights(dpt(s.v[0].w), dpt(s.v[1].w), dpt(s.v[2].w), u);
    } else if (s.count == 4) {
        const DPt w[4] = { dpt(s.v[0].w), dpt(s.v[1].w), dpt(s.v[2].w), dpt(s.v[3].w) };
        if (!tetrahedronWeights(w, u)) { return false; }
    }
    int kept = 0;
    for (int i = 0; i < s.count; ++i) {
        if (u[i] <= 0.0) { continue; }
        s.v[kept] = s.v[i];
        s.u[kept] = u[i];
        ++kept;
    }
    s.count = kept;
    return true;
}

TF_HD Vec3 simplexClosest(const Simplex& s) {
    DPt v{ 0.0, 0.0, 0.0 };
    for (int i = 0; i < s.count; ++i) { v = v + dpt(s.v[i].w) * s.u[i]; }
    return toVec(v);
}

enum Verdict { kOpen = 0, kWithin = 1, kBeyond = 2 };

// GJK from the first points (src/distance.cpp:193-245).
TF_HD int gjkSearch(const Convex& a, const Transform& xa, const Convex& b, const Transform& xb, float limit, Simplex& s,
                    Vec3& v, bool& overlap, const Vec3& start = Vec3{ 0.0f, 0.0f, 0.0f }) {
    const bool bounded = limit >= 0.0f;
    if (lengthSquared(start) > 0.0f) {
        s.v[0].a = gjkSupport(a, xa, start);
        s.v[0].b = gjkSupport(b, xb, -start);
    } else {
        s.v[0].a = a.cylinder ? apply(xa, Vec3{ a.rim, 0.0f, a.halfHeight }) : apply(xa, a.points[0]);
        s.v[0].b = b.cylinder ? apply(xb, Vec3{ b.rim, 0.0f, b.halfHeight }) : apply(xb, b.points[0]);
    }
    s.v[0].w = s.v[0].b - s.v[0].a;
    s.u[0] = 1.0;
    s.count = 1;
    v = s.v[0].w;
    overlap = false;
    for (int iter = 0; iter < 32; ++iter) {
        const float vv = dot(v, v);
        if (vv < 1.0e-14f) {
            overlap = true;
            return bounded ? kWithin : kOpen;
        }
        if (bounded && vv <= limit * limit) { return kWithin; }
        GVertex n;
        n.a = gjkSupport(a, xa, v);
        n.b = gjkSupport(b, xb, -v);
        n.w = n.b - n.a;
        const float vw = dot(v, n.w);
        if (bounded && vw > 0.0f && vw * vw > limit * limit * vv) { return kBeyond; }
        if (vv - vw <= 1.0e-6f * vv) { break; }
        bool repeated = false;
        for (int i = 0; i < s.count; ++i) { repeated = repeated || lengthSquared(s.v[i].w - n.w) < 1.0e-14f; }
        if (repeated) { break; }
        const Simplex previous = s;
        s.v[s.count++] = n;
        if (!solveSimplex(s)) {
            overlap = true;
            return bounded ? kWithin : kOpen;
        }
        const Vec3 next = simplexClosest(s);
        if (dot(next, next) >= vv) {
            s = previous;
            break;
        }
        v = next;
    }
    return kOpen;
}

// Whether the shapes are further apart than limit, for shapes with points (src/distance.cpp:248-256).
TF_HD bool apart(const Convex& a, const Transform& xa, const Convex& b, const Transform& xb, float limit) {
    Simplex s;
    Vec3 v;
    bool overlap;
    const int verdict = gjkSearch(a, xa, b, xb, limit + a.radius + b.radius, s, v, overlap);
    if (verdict != kOpen) { return verdict == kBeyond; }
    return length(v) - a.radius - b.radius > limit;
}

// ---------------------------------------------------------------------------------------------------------

// Everything a pair collision needs from the batch.
// A cylinder's cap as 24 points, and the turn between neighbouring points (src/collide3d.cpp:720-737,
// 1157-1168): cosines and sines taken on the host with the C library, as the reference takes them.
constexpr int kCapPoints = 24;
struct CapCircle {
    float cos[kCapPoints], sin[kCapPoints];
    float turnCos, turnSin;
};

struct CollideCtx {
    PolyTables pt;
    MeshTables mt;
    BoxTopology boxes;
    Tolerances tol;
    CapCircle cap;
};

TF_HD Convex convexOf(const CollideCtx& cx, const DShape& s) {
    Convex c;
    c.halfSpace = s.kind == kHalfSpace;
    c.radius = 0.0f;
    c.points = nullptr;
    c.count = 0;
    c.cylinder = s.kind == kCylinder;
    c.rim = c.cylinder ? s.radius : 0.0f;
    c.halfHeight = c.cylinder ? s.halfHeight : 0.0f;
    if (s.kind == kSphere) {
        c.points = &s.centroid;
        c.count = 1;
        c.radius = s.radius;
    } else if (s.kind == kConvex) {
        const DPoly& P = cx.pt.polys[s.poly];
        c.points = cx.pt.verts + P.vFirst;
        c.count = P.vCount;
    }
    return c;
}

// Picks the deciding axis and clips along it (src/collide3d.cpp:599-613).
TF_HD void convexContact(const FramePoly& a, const FramePoly& b, const FaceQuery& fa, const FaceQuery& fb,
                         const EdgeQuery& eq, const Transform& xa, float margin, const Tolerances& tol,
                         const Motion& motion, Manifold& m) {
    const float absTol = 0.5f * tol.linearSlop;
    if (eq.a >= 0 && eq.separation > 0.9f * maxf(fa.separation, fb.separation) + absTol) {
        edgeContact(a, b, eq, xa, margin, tol.linearSlop, motion, m);
        m.featKind = kFeatEdges;
        m.featA = eq.a;
        m.featB = eq.b;
    } else if (fb.separation > 0.98f * fa.separation + absTol) {
        faceContact(b, fb.index, a, true, xa, margin, tol.linearSlop, motion.swapped(), m);
        m.featKind = kFeatFaceB;
        m.featA = -1;
        m.featB = fb.index;
    } else {
        faceContact(a, fa.index, b, false, xa, margin, tol.linearSlop, motion, m);
        m.featKind = kFeatFaceA;
        m.featA = fa.index;
        m.featB = -1;
    }
}

// src/collide3d.cpp:615-648. reuseKind/A/B name the feature a fast pair met on, or kFeatNone.
TF_HD void collideConvex(const CollideCtx& cx, const DShape& sa, const Transform& xa, const DShape& sb,
                         const Transform& xb, float margin, const Motion& motion, Manifold& m, int reuseKind,
                         int reuseA, int reuseB) {
    const Transform x{ unrotate(xa.q, xb.p - xa.p), conjugate(xa.q) * xb.q };
    const FramePoly a = ownFrame(cx.pt, sa.poly);
    if (sa.geometry == 1 && sb.geometry == 1) {
        FaceQuery fa = noFace(), fb = noFace();
        EdgeQuery eq = noEdge();
        bool unsure;
        if (!boxQueries(cx.boxes, sa.halfExtents, sb.halfExtents, x, margin, fa, fb, eq, unsure)) { return; }
        if (unsure && apart(convexOf(cx, sa), xa, convexOf(cx, sb), xb, margin)) { return; }
        convexContact(a, otherFrame(cx.pt, sb.poly, x), fa, fb, eq, xa, margin, cx.tol, motion, m);
        return;
    }
    const FramePoly b = otherFrame(cx.pt, sb.poly, x);
    const FaceQuery fa = queryFaces(a, b, margin);
    if (fa.separation > margin) { return; }
    const FaceQuery fb = queryFaces(b, a, margin);
    if (fb.separation > margin) { return; }
    const bool reuse = reuseKind != kFeatNone;
    EdgeQuery eq = reuse ? reusedEdges(a, b, reuseKind, reuseA, reuseB) : noEdge();
    if (eq.separation > margin) { return; }
    if (!reuse || (reuseKind == kFeatEdges && eq.a < 0)) {
        const float reach = maxf(margin, -maxf(fa.separation, fb.separation));
        eq = queryEdges(a, b, reach);
        if (eq.separation > margin) { return; }
        if (eq.pruned && apart(convexOf(cx, sa), xa, convexOf(cx, sb), xb, margin)) { return; }
    }
    convexContact(a, b, fa, fb, eq, xa, margin, cx.tol, motion, m);
}

// Normal from the polyhedron to the sphere (src/collide3d.cpp:651-706).
TF_HD void collideSpherePoly(const CollideCtx& cx, const DShape& poly, const Transform& xp, const Vec3& center, float r,
                             float margin, Manifold& m) {
    const DPoly& P = cx.pt.polys[poly.poly];
    const Vec3* verts = cx.pt.verts + P.vFirst;
    const Vec3* normals = cx.pt.normals + P.fFirst;
    const float* offsets = cx.pt.offsets + P.fFirst;
    const DFace* faces = cx.pt.faces + P.fFirst;
    const int32_t* indices = cx.pt.indices + P.iFirst;
    const Vec3 c = applyInverse(xp, center);
    int best = -1;
    float bestSep = -FLT_MAX;
    bool outside = false;
    for (int i = 0; i < P.fCount; ++i) {
        const float s = dot(normals[i], c) - offsets[i];
        if (s > r + margin) { return; }
        if (s > 0.0f) { outside = true; }
        if (s > bestSep) {
            bestSep = s;
            best = i;
        }
    }
    if (best < 0) { return; }
    if (!outside) {
        const Vec3 n = normals[best];
        m.normal = rotate(xp.q, n);
        m.points[0] = { apply(xp, c - n * (0.5f * (bestSep + r))), bestSep - r, 0.0f };
        m.count = 1;
        return;
    }
    Vec3 closest = zero3();
    float closestSq = FLT_MAX;
    for (int i = 0; i < P.fCount; ++i) {
        const DFace f = faces[i];
        const Vec3 fn = normals[i];
        const float s = dot(fn, c) - offsets[i];
        if (s <= 0.0f) { continue; }
        const Vec3 proj = c - fn * s;
        bool inside = true;
        for (int k = 0; k < f.count; ++k) {
            const Vec3 a = verts[indices[f.first + k]];
            const Vec3 b = verts[indices[f.first + (k + 1) % f.count]];
            if (dot(cross(b - a, fn), proj - a) > 0.0f) {
                inside = false;
                const Vec3 ab = b - a;
                const float t = minf(maxf(dot(c - a, ab) / maxf(dot(ab, ab), FLT_MIN), 0.0f), 1.0f);
                const Vec3 q = a + ab * t;
                const float dsq = lengthSquared(c - q);
                if (dsq < closestSq) {
                    closestSq = dsq;
                    closest = q;
                }
            }
        }
        if (inside && s * s < closestSq) {
            closestSq = s * s;
            closest = proj;
        }
    }
    const float dist = sqrtf(closestSq);
    const float sep = dist - r;
    if (sep > margin || dist <= 0.0f) { return; }
    const Vec3 n = (c - closest) / dist;
    m.normal = rotate(xp.q, n);
    m.points[0] = { apply(xp, (closest + c - n * r) * 0.5f), sep, 0.0f };
    m.count = 1;
}

// src/collide3d.cpp:708-717.
TF_HD void collideSpheres(const Vec3& ca, float ra, const Vec3& cb, float rb, float margin, Manifold& m) {
    const Vec3 d = cb - ca;
    const float dist = length(d);
    const float sep = dist - ra - rb;
    if (sep > margin) { return; }
    const Vec3 n = dist > 0.0f ? d / dist : Vec3{ 0, 1, 0 };
    m.normal = n;
    m.points[0] = { ca + n * (ra + 0.5f * sep), sep, 0.0f };
    m.count = 1;
}

}
