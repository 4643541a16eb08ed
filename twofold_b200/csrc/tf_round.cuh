// Pairs with a cylinder (src/collide3d.cpp:720-1307): a cylinder or a polyhedron as a "solid", separating
// directions from face normals, cylinder axes and edge-axis cross products, GJK directions where a rim meets
// an edge, a climb toward the deepest direction in a deep overlap, and contacts clipped from the features
// each solid turns toward the other: a face, a cap as 24 points, a side line or a vertex.
#pragma once

#include "tf_collide.cuh"

namespace tfb {

constexpr float kFlatFace = 0.9998f;  // src/collide3d.cpp:739
constexpr int kMaxFeature = kMaxClip;  // points of one feature (a cap has kCapPoints)

// The point of the triangle closest to p, and its feature: corner k is k, edge k is 3 + k, the face 6
// (src/collide3d.cpp:987-1024).
TF_HD Vec3 closestOnTriangle(const Vec3 c[3], const Vec3& p, int& feature) {
    const Vec3 ab = c[1] - c[0], ac = c[2] - c[0], ap = p - c[0];
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) {
        feature = 0;
        return c[0];
    }
    const Vec3 bp = p - c[1];
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) {
        feature = 1;
        return c[1];
    }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        feature = 3;
        return c[0] + ab * (d1 / (d1 - d3));
    }
    const Vec3 cp = p - c[2];
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) {
        feature = 2;
        return c[2];
    }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        feature = 5;
        return c[0] + ac * (d2 / (d2 - d6));
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && d4 - d3 >= 0.0f && d5 - d6 >= 0.0f) {
        feature = 4;
        return c[1] + (c[2] - c[1]) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)));
    }
    feature = 6;
    const float denom = 1.0f / (va + vb + vc);
    return c[0] + ab * (vb * denom) + ac * (vc * denom);
}

// A cylinder or a polyhedron in the frame of the pair (src/collide3d.cpp:742-747).
struct Solid {
    bool cylinder;
    Vec3 center, axis, side;
    float radius, halfHeight;
    FramePoly poly;
};

TF_HD Solid cylinderSolid(const DShape& s, const Transform& xf) {
    Solid c;
    c.cylinder = true;
    c.center = xf.p;
    c.axis = rotate(xf.q, Vec3{ 0, 0, 1 });
    c.side = rotate(xf.q, Vec3{ 1, 0, 0 });
    c.radius = s.radius;
    c.halfHeight = s.halfHeight;
    return c;
}

TF_HD Solid polySolid(const FramePoly& p) {
    Solid s;
    s.cylinder = false;
    s.center = s.axis = s.side = zero3();
    s.radius = s.halfHeight = 0.0f;
    s.poly = p;
    return s;
}

TF_HD Solid solidOf(const CollideCtx& cx, const DShape& s, const Transform& xf) {
    if (s.kind == kCylinder) { return cylinderSolid(s, xf); }
    return polySolid(otherFrame(cx.pt, s.poly, xf));
}

// src/collide3d.cpp:767-775.
TF_HD float extentAlong(const Solid& s, const Vec3& d) {
    if (s.cylinder) {
        const float a = dot(s.axis, d);
        return dot(s.center, d) + s.halfHeight * fabsf(a) + s.radius * sqrtf(maxf(1.0f - a * a, 0.0f));
    }
    float most = dot(s.poly.v(0), d);
    for (int k = 1; k < s.poly.vertexCount(); ++k) { most = maxf(most, dot(s.poly.v(k), d)); }
    return most;
}

// The least and most a solid reaches along d (src/collide3d.cpp:778-794).
TF_HD void rangeAlong(const Solid& s, const Vec3& d, float& least, float& most) {
    if (s.cylinder) {
        const float a = dot(s.axis, d);
        const float c = dot(s.center, d);
        const float h = s.halfHeight * fabsf(a);
        const float r = s.radius * sqrtf(maxf(1.0f - a * a, 0.0f));
        most = c + h + r;
        least = -(-c + h + r);
        return;
    }
    most = least = dot(s.poly.v(0), d);
    for (int k = 1; k < s.poly.vertexCount(); ++k) {
        const float x = dot(s.poly.v(k), d);
        most = maxf(most, x);
        least = minf(least, x);
    }
}

// src/collide3d.cpp:796-809.
TF_HD Vec3 supportPoint(const Solid& s, const Vec3& d) {
    if (s.cylinder) {
        const float a = dot(s.axis, d);
        const Vec3 radial = d - s.axis * a;
        const float len = length(radial);
        const Vec3 rim = len > 1e-6f ? radial * (s.radius / len) : zero3();
        return s.center + s.axis * (a < 0.0f ? -s.halfHeight : s.halfHeight) + rim;
    }
    int best = 0;
    for (int k = 1; k < s.poly.vertexCount(); ++k) {
        if (dot(s.poly.v(k), d) > dot(s.poly.v(best), d)) { best = k; }
    }
    return s.poly.v(best);
}

// The part of a solid farthest along d: a face with its outward normal, an edge or a point. A cylinder
// gives a cap within 45 degrees of its axis, else the line of its side (src/collide3d.cpp:813-855).
// Returns the point count; normal is set for a face or a cap only.
TF_HD int featureAlong(const CapCircle& circle, const Solid& s, const Vec3& d, float band, Vec3* out, Vec3& normal) {
    int n = 0;
    if (s.cylinder) {
        const float a = dot(s.axis, d);
        const Vec3 radial = d - s.axis * a;
        const float len = length(radial);
        if (fabsf(a) > len) {
            normal = a < 0.0f ? -s.axis : s.axis;
            // A tilted cap starts at its deepest point, so that point is exact; a level one keeps the same
            // points as it turns, so its contacts carry over between steps.
            const Vec3 u = 2.0f * s.radius * len > band ? radial / len : s.side;
            const Vec3 v = cross(normal, u);
            const Vec3 c = s.center + normal * s.halfHeight;
            for (int k = 0; k < kCapPoints; ++k) { out[n++] = c + (u * circle.cos[k] + v * circle.sin[k]) * s.radius; }
        } else {
            const Vec3 p = s.center + radial * (s.radius / len);
            out[n++] = p - s.axis * s.halfHeight;
            out[n++] = p + s.axis * s.halfHeight;
        }
        return n;
    }
    const FramePoly& p = s.poly;
    const int f = supportFace(p, d);
    if (dot(p.n(f), d) >= kFlatFace) {
        normal = p.n(f);
        const DFace face = p.face(f);
        for (int k = 0; k < face.count && n < kMaxFeature; ++k) { out[n++] = p.v(p.index(face.first + k)); }
        return n;
    }
    int first = 0, second = -1;
    for (int k = 1; k < p.vertexCount(); ++k) {
        if (dot(p.v(k), d) > dot(p.v(first), d)) {
            second = first;
            first = k;
        } else if (second < 0 || dot(p.v(k), d) > dot(p.v(second), d)) {
            second = k;
        }
    }
    out[n++] = p.v(first);
    if (second >= 0 && dot(p.v(second), d) >= dot(p.v(first), d) - band) { out[n++] = p.v(second); }
    return n;
}

struct Separation {
    Vec3 normal;
    float gap;
};

TF_HD Separation noSeparation() { return Separation{ zero3(), -FLT_MAX }; }

// src/collide3d.cpp:861-870.
TF_HD void tryAxis(const Solid& a, const Solid& b, const Vec3& d, Separation& best) {
    const float len = length(d);
    if (len < 1e-6f) { return; }
    const Vec3 n = d / len;
    const float gap = -extentAlong(a, n) - extentAlong(b, -n);
    if (gap > best.gap) {
        best.normal = n;
        best.gap = gap;
    }
}

// d, then -d (src/collide3d.cpp:873-888).
TF_HD void tryAxes(const Solid& a, const Solid& b, const Vec3& d, Separation& best) {
    const float len = length(d);
    if (len < 1e-6f) { return; }
    const Vec3 n = d / len;
    float leastA, mostA, leastB, mostB;
    rangeAlong(a, n, leastA, mostA);
    rangeAlong(b, n, leastB, mostB);
    if (leastB - mostA > best.gap) {
        best.normal = n;
        best.gap = leastB - mostA;
    }
    if (leastA - mostB > best.gap) {
        best.normal = -n;
        best.gap = leastA - mostB;
    }
}

// The best of the directions along which a flat or straight pair of features can touch; stops once one
// separates the solids by more than limit (src/collide3d.cpp:893-926).
TF_HD Separation featureAxes(const Solid& a, const Solid& b, float limit) {
    Separation best = noSeparation();
    for (int i = 0; !a.cylinder && i < a.poly.faceCount() && best.gap <= limit; ++i) { tryAxis(a, b, a.poly.n(i), best); }
    for (int i = 0; !b.cylinder && i < b.poly.faceCount() && best.gap <= limit; ++i) { tryAxis(a, b, -b.poly.n(i), best); }
    if (a.cylinder) { tryAxes(a, b, a.axis, best); }
    if (b.cylinder) { tryAxes(a, b, b.axis, best); }
    if (best.gap > limit) { return best; }
    if (a.cylinder && b.cylinder) {
        const Vec3 c = cross(a.axis, b.axis);
        if (length(c) > kParallelEdges) {
            tryAxes(a, b, c, best);
        } else {
            const Vec3 d = b.center - a.center;
            tryAxis(a, b, d - a.axis * dot(d, a.axis), best);
        }
        return best;
    }
    const Solid& cyl = a.cylinder ? a : b;
    const FramePoly& p = a.cylinder ? b.poly : a.poly;
    for (int i = 0; i < p.edgeCount(); ++i) {
        if (best.gap > limit) { break; }
        const DEdge e = p.edge(i);
        const Vec3 edge = p.v(e.v1) - p.v(e.v0);
        Vec3 c = cross(edge, cyl.axis);
        if (length(c) <= kParallelEdges * e.length) {
            const Vec3 d = p.v(e.v0) - cyl.center;
            c = d - cyl.axis * dot(d, cyl.axis);
        }
        tryAxes(a, b, c, best);
    }
    return best;
}

// distance() (src/distance.cpp:269-305) from a start direction: the normal from a to b and the gap.
TF_HD void convexDistance(const Convex& a, const Transform& xa, const Convex& b, const Transform& xb, const Vec3& start,
                          Vec3& normal, float& distance) {
    Simplex s;
    Vec3 v;
    bool overlap;
    gjkSearch(a, xa, b, xb, -1.0f, s, v, overlap, start);
    const float gap = overlap ? 0.0f : length(v);
    normal = gap > 0.0f ? v * (1.0f / gap) : Vec3{ 0, 0, 1 };
    distance = gap - a.radius - b.radius;
}

// GJK directions between the shapes and between their cores, cylinders shrunk into a rounded core; near
// touching the first is poorly placed and the second takes over (src/collide3d.cpp:929-947).
TF_HD int distanceAxes(Convex ca, const Transform& xa, Convex cb, const Transform& xb, const Vec3& start,
                       const Tolerances& tol, Vec3 n[2]) {
    int count = 0;
    Vec3 normal;
    float distance;
    convexDistance(ca, xa, cb, xb, start, normal, distance);
    if (distance > 0.0f) { n[count++] = normal; }
    if (distance > tol.linearSlop) { return count; }
    float shrunk = 0.0f;
    Convex* both[2] = { &ca, &cb };
    for (int k = 0; k < 2; ++k) {
        Convex* c = both[k];
        if (!c->cylinder) { continue; }
        const float core = 0.25f * minf(c->rim, c->halfHeight);
        c->rim -= core;
        c->halfHeight -= core;
        c->radius += core;
        shrunk += core;
    }
    convexDistance(ca, xa, cb, xb, zero3(), normal, distance);
    if (distance + shrunk > 0.0f) { n[count++] = normal; }
    return count;
}

// src/collide3d.cpp:949-954.
TF_HD Vec3 centerOf(const Solid& s) {
    if (s.cylinder) { return s.center; }
    Vec3 c = zero3();
    for (int k = 0; k < s.poly.vertexCount(); ++k) { c = c + s.poly.v(k); }
    return c / (float)s.poly.vertexCount();
}

// Tilts from start while that separates the solids more; each step only comes closer to the true direction
// (src/collide3d.cpp:958-975).
TF_HD Separation climb(const Solid& a, const Solid& b, Separation start) {
    const float kDiagonal = 0.70710678f;
    const float turns[8][2] = { { 1, 0 }, { kDiagonal, kDiagonal }, { 0, 1 }, { -kDiagonal, kDiagonal },
                                { -1, 0 }, { -kDiagonal, -kDiagonal }, { 0, -1 }, { kDiagonal, -kDiagonal } };
    Separation best = start;
    float step = 0.1f;
    for (int i = 0; i < 64 && step > 1e-3f; ++i) {
        const Vec3 u = perpendicular(best.normal), v = cross(best.normal, u);
        Separation next = best;
        for (int t = 0; t < 8; ++t) { tryAxis(a, b, best.normal + (u * turns[t][0] + v * turns[t][1]) * step, next); }
        if (next.gap > best.gap) {
            best = next;
        } else {
            step *= 0.5f;
        }
    }
    return best;
}

// src/collide3d.cpp:977-984.
TF_HD Vec3 closestOnCylinder(const Solid& s, const Vec3& p) {
    const Vec3 d = p - s.center;
    const float along = dot(d, s.axis);
    Vec3 radial = d - s.axis * along;
    const float len = length(radial);
    if (len > s.radius) { radial = radial * (s.radius / len); }
    return s.center + s.axis * minf(maxf(along, -s.halfHeight), s.halfHeight) + radial;
}

// Distance from the segment pq to the triangle, with the closest point on each (src/collide3d.cpp:1027-1059).
TF_HD float segmentToTriangle(const Vec3 c[3], const Vec3& p, const Vec3& q, Vec3& onSegment, Vec3& onTriangle) {
    const Vec3 n = cross(c[1] - c[0], c[2] - c[0]);
    const float hp = dot(n, p - c[0]), hq = dot(n, q - c[0]);
    int feature;
    if ((hp < 0.0f) != (hq < 0.0f)) {
        const Vec3 x = p + (q - p) * (hp / (hp - hq));
        closestOnTriangle(c, x, feature);
        if (feature == 6) {
            onSegment = onTriangle = x;
            return 0.0f;
        }
    }
    onSegment = p;
    onTriangle = closestOnTriangle(c, p, feature);
    float best = length(p - onTriangle);
    const Vec3 fromQ = closestOnTriangle(c, q, feature);
    if (length(q - fromQ) < best) {
        best = length(q - fromQ);
        onSegment = q;
        onTriangle = fromQ;
    }
    for (int k = 0; k < 3; ++k) {
        Vec3 s, t;
        closestOnSegments(p, q, c[k], c[(k + 1) % 3], s, t);
        if (length(s - t) < best) {
            best = length(s - t);
            onSegment = s;
            onTriangle = t;
        }
    }
    return best;
}

// False when the solids are further apart than margin (src/collide3d.cpp:1063-1136). A GJK direction wins
// only where no flat or straight feature pair comes close, such as a rim on an edge; in a deep overlap the
// best axis climbs toward the direction a curved pair touches along. A triangle solid has three vertices.
TF_HD bool separate(const Solid& a, const Solid& b, const Convex& ca, const Transform& xa, const Convex& cb,
                    const Transform& xb, const Quat& toFrame, float margin, const Tolerances& tol, Separation& best) {
    best = featureAxes(a, b, margin);
    if (best.gap > margin) { return false; }
    float apart = FLT_MAX;
    Vec3 between = zero3();
    if (!a.cylinder && a.poly.vertexCount() == 3) {
        const Vec3 tri[3] = { a.poly.v(0), a.poly.v(1), a.poly.v(2) };
        // A cylinder lies within the capsule around its axis; where the capsule is closest between the caps,
        // its side is the cylinder's, and the direction between the closest points separates by exactly
        // their distance.
        if (b.cylinder) {
            const Vec3 h = b.axis * b.halfHeight;
            Vec3 onAxis, onTriangle;
            const float reach = segmentToTriangle(tri, b.center - h, b.center + h, onAxis, onTriangle) - b.radius;
            if (reach > margin + 0.1f * tol.linearSlop) {
                best.gap = reach;
                return false;
            }
            if (reach > 0.0f && fabsf(dot(onAxis - b.center, b.axis)) < 0.999f * b.halfHeight) {
                Separation side = noSeparation();
                tryAxis(a, b, onAxis - onTriangle, side);
                if (side.gap > best.gap + 0.1f * tol.linearSlop) { best = side; }
                apart = reach;
            }
        }
        // No axis separates the solids by more than two of their points are apart: once a pair found by
        // projecting back and forth comes as close as the best axis, a GJK direction cannot win.
        Vec3 p = supportPoint(b, -best.normal);
        for (int i = 0; i < 16 && apart > best.gap + 0.1f * tol.linearSlop; ++i) {
            int feature;
            const Vec3 q = closestOnTriangle(tri, p, feature);
            apart = length(p - q);
            if (!b.cylinder || apart <= best.gap + 0.1f * tol.linearSlop) { break; }
            between = p - q;
            if (i >= 2 && apart > tol.linearSlop) {
                Separation pair = noSeparation();
                tryAxis(a, b, between, pair);
                if (pair.gap >= apart - 0.01f * tol.linearSlop) {
                    if (pair.gap > best.gap + 0.1f * tol.linearSlop) { best = pair; }
                    apart = best.gap;
                    break;
                }
            }
            p = closestOnCylinder(b, q);
        }
    }
    if (apart > best.gap + 0.1f * tol.linearSlop) {
        Vec3 n[2];
        const int count = distanceAxes(ca, xa, cb, xb, rotate(toFrame, between), tol, n);
        Separation curved = noSeparation();
        for (int i = 0; i < count; ++i) { tryAxis(a, b, unrotate(toFrame, n[i]), curved); }
        if (curved.gap > best.gap + 0.1f * tol.linearSlop) { best = curved; }
    }
    if (best.gap < -2.0f * tol.speculative) {
        // The gap has several peaks: a rim pressed into the other solid peaks near its cap normal or its side.
        Separation climbed = climb(a, b, best);
        const Vec3 d = centerOf(b) - centerOf(a);
        const Solid* both[2] = { &a, &b };
        for (int k = 0; k < 2; ++k) {
            const Solid* s = both[k];
            if (!s->cylinder) { continue; }
            Separation cap = noSeparation(), side = noSeparation();
            tryAxes(a, b, s->axis, cap);
            tryAxis(a, b, d - s->axis * dot(d, s->axis), side);
            const Separation starts[2] = { cap, side };
            for (int x = 0; x < 2; ++x) {
                if (starts[x].gap == -FLT_MAX) { continue; }
                const Separation peak = climb(a, b, starts[x]);
                if (peak.gap > climbed.gap) { climbed = peak; }
            }
        }
        if (climbed.gap > best.gap + 0.1f * tol.linearSlop) { best = climbed; }
    }
    return best.gap <= margin;
}

// src/collide3d.cpp:1138-1148. Returns the new point count (0 or 2).
TF_HD int clipSegment(Vec3* seg, const Vec3& n, const Vec3& origin) {
    const float dp = dot(n, seg[0] - origin), dq = dot(n, seg[1] - origin);
    if (dp > 0.0f && dq > 0.0f) { return 0; }
    if (dp > 0.0f) {
        seg[0] = seg[0] + (seg[1] - seg[0]) * (dp / (dp - dq));
    } else if (dq > 0.0f) {
        seg[1] = seg[1] + (seg[0] - seg[1]) * (dq / (dq - dp));
    }
    return 2;
}

// The side lines one cap point either side of the one along d; a spinning cylinder brings them into
// contact within a step (src/collide3d.cpp:1157-1168).
TF_HD void turnLines(const CapCircle& circle, const Solid& s, const Vec3& d, Vec3 out[4]) {
    const Vec3 radial = normalize(d - s.axis * dot(s.axis, d));
    const Vec3 across = cross(s.axis, radial);
    const float signs[2] = { -1.0f, 1.0f };
    for (int k = 0; k < 2; ++k) {
        const Vec3 p = s.center + (radial * circle.turnCos + across * (signs[k] * circle.turnSin)) * s.radius;
        out[2 * k] = p - s.axis * s.halfHeight;
        out[2 * k + 1] = p + s.axis * s.halfHeight;
    }
}

// Contacts of solids that separate by gap along n, from a to b: whichever feature is a face clips the other,
// and of a face pair the one facing better along n clips (src/collide3d.cpp:1171-1264).
TF_HD void solidContact(const CapCircle& circle, const Solid& a, const Solid& b, const Vec3& n, float gap,
                        const Transform& xf, float margin, float band, const Motion& motion, Manifold& m) {
    Vec3 fa[kMaxFeature], fb[kMaxFeature];
    Vec3 na = zero3(), nb = zero3();
    const int nfa = featureAlong(circle, a, n, band, fa, na);
    const int nfb = featureAlong(circle, b, -n, band, fb, nb);
    const Vec3 worldN = rotate(xf.q, n);
    MPoint pts[kMaxClip + 16];
    int np = 0;
    // No point needs a deeper push than the separating direction allows.
    auto add = [&](const Vec3& onA, const Vec3& onB, float s) {
        s = maxf(s, gap);
        if (s > margin || np >= kMaxClip + 16) { return; }
        const Vec3 w = apply(xf, (onA + onB) * 0.5f);
        pts[np++] = MPoint{ w, s, motion.predict(w, worldN, s) };
    };
    const bool faceA = nfa >= 3, faceB = nfb >= 3;
    const bool refA = faceA && (!faceB || dot(na, n) >= -dot(nb, n));
    auto clipToFace = [&](const Vec3* feature, int count) {
        const Vec3* ref = refA ? fa : fb;
        const int nref = refA ? nfa : nfb;
        const Vec3 refN = refA ? na : nb;
        const Vec3 out = refA ? n : -n;
        const float facing = dot(refN, out);
        Vec3 inc[kMaxClip], scratch[kMaxClip];
        int ni = 0;
        for (int k = 0; k < count && ni < kMaxClip; ++k) { inc[ni++] = feature[k]; }
        for (int k = 0; k < nref && ni > 0; ++k) {
            const Vec3 side = cross(ref[(k + 1) % nref] - ref[k], refN);
            if (ni >= 3) {
                ni = clipPolygon(inc, ni, scratch, side, ref[k]);
            } else if (ni == 2) {
                ni = clipSegment(inc, side, ref[k]);
            } else if (dot(side, inc[0] - ref[k]) > 0.0f) {
                ni = 0;
            }
        }
        for (int k = 0; k < ni; ++k) {
            const Vec3 q = inc[k];
            const float s = dot(refN, q - ref[0]) / facing;
            const Vec3 onRef = q - out * s;
            if (refA) {
                add(onRef, q, s);
            } else {
                add(q, onRef, s);
            }
        }
    };
    // Lines closer to parallel than kParallelEdges touch along their overlap, others at their closest points.
    auto linePair = [&](const Vec3& a0, const Vec3& a1, const Vec3& b0, const Vec3& b1) {
        const Vec3 da = a1 - a0, db = b1 - b0;
        const float la = dot(da, da), lb = dot(db, db);
        if (la > 0.0f && lb > 0.0f && length(cross(da, db)) <= kParallelEdges * sqrtf(la * lb)) {
            const float t0 = dot(b0 - a0, da) / la, t1 = dot(b1 - a0, da) / la;
            const float lo = maxf(minf(t0, t1), 0.0f), hi = minf(maxf(t0, t1), 1.0f);
            if (lo <= hi) {
                const float ts[2] = { lo, hi };
                for (int k = 0; k < 2; ++k) {
                    const Vec3 onA = a0 + da * ts[k];
                    const Vec3 onB = b0 + db * minf(maxf(dot(onA - b0, db) / lb, 0.0f), 1.0f);
                    add(onA, onB, dot(onB - onA, n));
                }
                return;
            }
        }
        // Lines tilted against n reach deeper at their ends than where they pass closest.
        Vec3 onA, onB;
        closestOnSegments(a0, a1, b0, b1, onA, onB);
        add(onA, onB, minf(dot(b0, n), dot(b1, n)) - maxf(dot(a0, n), dot(a1, n)));
    };

    const Solid& incident = refA ? b : a;
    const Vec3* incFeature = refA ? fb : fa;
    const int nInc = refA ? nfb : nfa;
    if (faceA || faceB) {
        clipToFace(incFeature, nInc);
    } else if (nfa == 2 && nfb == 2) {
        linePair(fa[0], fa[1], fb[0], fb[1]);
    }
    if (np == 0) {
        const Vec3 onB = nfa == 1 && nfb != 1 ? fa[0] + n * gap : supportPoint(b, -n);
        add(onB - n * gap, onB, gap);
    }
    Vec3 turn[4];
    if ((faceA || faceB) && incident.cylinder && nInc == 2) {
        turnLines(circle, incident, refA ? -n : n, turn);
        for (int k = 0; k < 2; ++k) { clipToFace(&turn[2 * k], 2); }
    } else if (!faceA && !faceB && nfa == 2 && nfb == 2) {
        if (a.cylinder) {
            turnLines(circle, a, n, turn);
            for (int k = 0; k < 2; ++k) { linePair(turn[2 * k], turn[2 * k + 1], fb[0], fb[1]); }
        }
        if (b.cylinder) {
            turnLines(circle, b, -n, turn);
            for (int k = 0; k < 2; ++k) { linePair(fa[0], fa[1], turn[2 * k], turn[2 * k + 1]); }
        }
    }
    reduceManifold(pts, np, worldN, band, m, 0.5f * band, motion.fast);
}

// Two shapes in the world frame, at least one of them a cylinder (src/collide3d.cpp:1266-1274).
TF_HD void collideRound(const CollideCtx& cx, const DShape& sa, const Transform& xa, const DShape& sb,
                        const Transform& xb, float margin, const Motion& motion, Manifold& m) {
    const Solid a = solidOf(cx, sa, xa);
    const Solid b = solidOf(cx, sb, xb);
    Separation best;
    if (!separate(a, b, convexOf(cx, sa), xa, convexOf(cx, sb), xb, qid(), margin, cx.tol, best)) { return; }
    solidContact(cx.cap, a, b, best.normal, best.gap, Transform{ zero3(), qid() }, margin, cx.tol.linearSlop, motion, m);
}

// A cylinder and a sphere; the normal points from the cylinder to the sphere (src/collide3d.cpp:1277-1306).
TF_HD void collideSphereCylinder(const DShape& cyl, const Transform& xc, const Vec3& center, float r, float margin,
                                 Manifold& m) {
    const Vec3 c = applyInverse(xc, center);
    const float rho = sqrtf(c.x * c.x + c.y * c.y);
    Vec3 n, surface;
    float sep;
    if (rho <= cyl.radius && fabsf(c.z) <= cyl.halfHeight) {
        const float side = cyl.radius - rho, cap = cyl.halfHeight - fabsf(c.z);
        if (side < cap) {
            n = rho > 0.0f ? Vec3{ c.x / rho, c.y / rho, 0.0f } : Vec3{ 1, 0, 0 };
            surface = c + n * side;
            sep = -side - r;
        } else {
            n = Vec3{ 0.0f, 0.0f, c.z < 0.0f ? -1.0f : 1.0f };
            surface = c + n * cap;
            sep = -cap - r;
        }
    } else {
        const float scale = rho > cyl.radius ? cyl.radius / rho : 1.0f;
        surface = Vec3{ c.x * scale, c.y * scale, minf(maxf(c.z, -cyl.halfHeight), cyl.halfHeight) };
        const float dist = length(c - surface);
        if (dist <= 0.0f) { return; }
        n = (c - surface) / dist;
        sep = dist - r;
    }
    if (sep > margin) { return; }
    m.normal = rotate(xc.q, n);
    m.points[0] = MPoint{ apply(xc, (surface + c - n * r) * 0.5f), sep, 0.0f };
    m.count = 1;
}

}
