// The planar path (src/collide2d.cpp): two bodies locked to one plane collide as the 2D profiles their
// shapes cut in that plane, worked out in the first body's 2D frame, with at most two points and a normal
// that stays in the plane.
//
// The reference caches two things between steps. A body's pose in the plane keeps its key (the plane normal
// in the body's frame) and 2D axes until the normal drifts past kProfileDrift; that state is kept here in the
// body (DBody::pose*), placed at most once per round of collisions and stored once the round's pairs are done.
// A shape's profile is cached under the exact bits of that key; it is a pure function of the shape and the
// key, so here it is made afresh for each pair, with the same bits the cache would return.
#pragma once

#include "tf_collide.cuh"

namespace tfb {

// How close to the plane normal a box axis or prism axis must lie for its profile to be a polygon, and how
// closely two bodies' plane normals must agree (src/collide2d.cpp:8, src/world.cpp:737-750).
constexpr float kPlaneAligned = 0.9999f;
// How far the plane normal may turn in a body's frame before the pose is placed again (src/collide2d.cpp:11).
constexpr float kProfileDrift = 1e-5f;
// Profile points a thread holds; a prism with a longer outline on a planar body stops the step as unsupported.
constexpr int kMaxProfilePoints = 16;

enum ProfileKind : int { kProfileNone = 0, kProfilePolygon = 1, kProfileCircle = 2, kProfileHalfPlane = 3 };

// A body's pose in a plane (src/internal.h:141-148).
struct PlanePose {
    Vec3 normal, key, u, v, axisU, axisV;
    Vec2 position, turn;
    float depth;
};

// The profile of a shape in its body's frame (src/internal.h:125-139).
struct Profile {
    int kind, count;
    Vec2 center, extent;
    float radius;
    Vec2 normal;
    float offset, tilt;
    float zLo, zHi;
    Vec2 points[kMaxProfilePoints];
    Vec2 normals[kMaxProfilePoints];
};

TF_HD bool sameBits(const Vec3& a, const Vec3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

// Whether a pair is solved in a plane, and which (src/world.cpp:737-750): every dynamic body of the pair is
// locked to a plane, the planes agree, and there is at least one.
TF_HD bool usePlanar(const DBody& a, const DBody& b, Vec3& n) {
    const DBody* both[2] = { &a, &b };
    bool found = false;
    for (int k = 0; k < 2; ++k) {
        const DBody& x = *both[k];
        if (x.type != kDynamic) { continue; }
        if (!isPlanar(x)) { return false; }
        if (!found) {
            found = true;
            n = planeNormal(x);
        } else if (fabsf(dot(n, planeNormal(x))) < kPlaneAligned) {
            return false;
        }
    }
    return found;
}

// placeInPlane (src/collide2d.cpp:423-437), starting from the pose the body kept.
TF_HD PlanePose placeInPlane(const DBody& b, const Vec3& n) {
    PlanePose p;
    p.normal = b.poseNormal;
    p.key = b.poseKey;
    p.u = b.poseU;
    p.v = b.poseV;
    p.axisU = b.poseAxisU;
    p.axisV = b.poseAxisV;
    const Vec3 key = unrotate(b.xf.q, n);
    if (!sameBits(p.normal, n) || lengthSquared(key - p.key) > kProfileDrift * kProfileDrift) {
        p.normal = n;
        p.key = key;
        p.u = perpendicular(key);
        p.v = cross(key, p.u);
        p.axisU = perpendicular(n);
        p.axisV = cross(n, p.axisU);
    }
    const Vec3 u = rotate(b.xf.q, p.u);
    p.turn = normalize(Vec2{ dot(u, p.axisU), dot(u, p.axisV) });
    p.position = Vec2{ dot(b.xf.p, p.axisU), dot(b.xf.p, p.axisV) };
    p.depth = dot(b.xf.p, n);
    return p;
}

// Stores the lasting part of a placement in the body.
TF_HD void keepPose(DBody& b, const PlanePose& p) {
    b.poseNormal = p.normal;
    b.poseKey = p.key;
    b.poseU = p.u;
    b.poseV = p.v;
    b.poseAxisU = p.axisU;
    b.poseAxisV = p.axisV;
}

TF_HD Vec2 project2(const Vec3& p, const Vec3& u, const Vec3& v) { return Vec2{ dot(p, u), dot(p, v) }; }

TF_HD void setDepth(Profile& p, float center, float a, float b) {
    p.zLo = center + minf(a, b);
    p.zHi = center + maxf(a, b);
}

// The profile of shape s seen along n, with u and v the 2D axes around n, all in the body's frame
// (src/collide2d.cpp:47-96). Returns false for an outline longer than kMaxProfilePoints.
TF_HD bool makeProfile(const PolyTables& pt, const DShape& s, const Vec3& n, const Vec3& u, const Vec3& v, Profile& p) {
    const Transform& xf = s.local;
    const float c = dot(xf.p, n);
    p.kind = kProfileNone;
    p.count = 0;
    if (s.geometry == 1 /* TF_BOX */) {
        const Vec3 axes[3] = { rotate(xf.q, Vec3{ 1, 0, 0 }), rotate(xf.q, Vec3{ 0, 1, 0 }), rotate(xf.q, Vec3{ 0, 0, 1 }) };
        const float h[3] = { s.halfExtents.x, s.halfExtents.y, s.halfExtents.z };
        for (int i = 0; i < 3; ++i) {
            const float a = dot(axes[i], n);
            if (fabsf(a) < kPlaneAligned) { continue; }
            const int j = (i + 1) % 3, k = (i + 2) % 3;
            const Vec3 aj = axes[j] * h[j];
            const Vec3 ak = axes[k] * h[k];
            p.points[0] = project2(xf.p + aj + ak, u, v);
            p.points[1] = project2(xf.p - aj + ak, u, v);
            p.points[2] = project2(xf.p - aj - ak, u, v);
            p.points[3] = project2(xf.p + aj - ak, u, v);
            p.count = 4;
            setDepth(p, c, -h[i], h[i]);
            p.kind = kProfilePolygon;
            return true;
        }
        return true;
    }
    const Vec3 zw = rotate(xf.q, Vec3{ 0, 0, 1 });
    const float a = dot(zw, n);
    // A half-space standing on the plane cuts every depth along nearly the same line.
    if (s.kind == kHalfSpace) {
        if (a * a > 1.0f - kPlaneAligned * kPlaneAligned) { return true; }
        const Vec2 m = project2(zw, u, v);
        const float inv = 1.0f / length(m);
        p.normal = m * inv;
        p.offset = dot(zw, xf.p) * inv;
        p.tilt = a * inv;
        p.zLo = -FLT_MAX;
        p.zHi = FLT_MAX;
        p.kind = kProfileHalfPlane;
        return true;
    }
    if (fabsf(a) < kPlaneAligned) { return true; }
    if (s.kind == kCylinder) {
        p.center = project2(xf.p, u, v);
        p.radius = s.radius;
        setDepth(p, c, -s.halfHeight, s.halfHeight);
        p.kind = kProfileCircle;
        return true;
    }
    if (s.geometry == 3 /* TF_PRISM */ && s.poly >= 0) {
        // A prism's polyhedron starts with its outline at zMin, then the same outline at zMax.
        const DPoly& P = pt.polys[s.poly];
        const int n2 = P.vCount / 2;
        if (n2 < 3) { return true; }
        if (n2 > kMaxProfilePoints) { return false; }
        for (int i = 0; i < n2; ++i) {
            const Vec3 k = pt.verts[P.vFirst + i];
            p.points[i] = project2(apply(xf, Vec3{ k.x, k.y, 0.0f }), u, v);
        }
        p.count = n2;
        setDepth(p, c, a * pt.verts[P.vFirst].z, a * pt.verts[P.vFirst + n2].z);
        p.kind = kProfilePolygon;
    }
    return true;
}

// profileOf (src/collide2d.cpp:101-124): the profile for a pose key, its polygon wound counter-clockwise
// with edge normals and bounds.
TF_HD bool profileOf(const PolyTables& pt, const DShape& s, const PlanePose& pose, Profile& p) {
    if (!makeProfile(pt, s, pose.key, pose.u, pose.v, p)) { return false; }
    if (p.kind == kProfilePolygon) {
        const int n = p.count;
        float area = 0.0f;
        for (int i = 0; i < n; ++i) { area += cross(p.points[i], p.points[(i + 1) % n]); }
        if (area < 0.0f) {
            for (int i = 0, j = n - 1; i < j; ++i, --j) {
                const Vec2 t = p.points[i];
                p.points[i] = p.points[j];
                p.points[j] = t;
            }
        }
        Vec2 lo = p.points[0], hi = p.points[0];
        for (int i = 0; i < n; ++i) {
            const Vec2 e = p.points[(i + 1) % n] - p.points[i];
            p.normals[i] = normalize(Vec2{ e.y, -e.x });
            lo = Vec2{ minf(lo.x, p.points[i].x), minf(lo.y, p.points[i].y) };
            hi = Vec2{ maxf(hi.x, p.points[i].x), maxf(hi.y, p.points[i].y) };
        }
        p.center = (lo + hi) * 0.5f;
        p.extent = (hi - lo) * 0.5f;
    } else if (p.kind == kProfileCircle) {
        p.extent = Vec2{ p.radius, p.radius };
    }
    return true;
}

// A convex polygon: points counter-clockwise, normals[i] the outward normal of edge i -> i+1.
struct Polygon2 {
    const Vec2* points;
    const Vec2* normals;
    int count;
};

// The result of one 2D pair in the first profile's frame (src/collide2d.cpp:26-31).
struct Planar2 {
    Vec2 normal;
    Vec2 points[2];
    float separations[2];
    int count;
};

// std::clamp(x, 0, 1).
TF_HD float clamp01(float x) { return x < 0.0f ? 0.0f : (1.0f < x ? 1.0f : x); }

struct SegmentClosest {
    Vec2 a, b;
    float s, t;
};

// Closest points of two segments (src/collide2d.cpp:133-159).
TF_HD SegmentClosest closestOnSegments(const Vec2& p1, const Vec2& q1, const Vec2& p2, const Vec2& q2) {
    const Vec2 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    const float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    SegmentClosest c;
    c.s = 0.0f;
    c.t = 0.0f;
    if (a <= FLT_EPSILON && e > FLT_EPSILON) {
        c.t = clamp01(f / e);
    } else if (a > FLT_EPSILON) {
        const float k = dot(d1, r);
        if (e <= FLT_EPSILON) {
            c.s = clamp01(-k / a);
        } else {
            const float b = dot(d1, d2), denom = a * e - b * b;
            c.s = denom > 0.0f ? clamp01((b * f - k * e) / denom) : 0.0f;
            c.t = (b * c.s + f) / e;
            if (c.t < 0.0f) {
                c.t = 0.0f;
                c.s = clamp01(-k / a);
            } else if (c.t > 1.0f) {
                c.t = 1.0f;
                c.s = clamp01((b - k) / a);
            }
        }
    }
    c.a = p1 + d1 * c.s;
    c.b = p2 + d2 * c.t;
    return c;
}

// The edge of a with the largest separation from b, stopping once it is past margin
// (src/collide2d.cpp:162-180).
TF_HD float maxSeparation(const Polygon2& a, const Polygon2& b, float margin, int& edge) {
    float best = -FLT_MAX;
    edge = 0;
    for (int i = 0; i < a.count; ++i) {
        const Vec2 n = a.normals[i];
        float s = FLT_MAX;
        for (int k = 0; k < b.count; ++k) {
            const float d = dot(n, b.points[k] - a.points[i]);
            s = d < s ? d : s;
            if (s <= best) { break; }
        }
        if (s > best) {
            best = s;
            edge = i;
            if (best > margin) { break; }
        }
    }
    return best;
}

// Polygon against polygon: reference edge, incident edge clipped to it, or the two nearest vertices when the
// polygons are apart (src/collide2d.cpp:182-256).
TF_HD void collidePolygons(const Polygon2& a, const Polygon2& b, float margin, float slop, Planar2& out) {
    int edgeA = 0, edgeB = 0;
    const float sa = maxSeparation(a, b, margin, edgeA);
    if (sa > margin) { return; }
    const float sb = maxSeparation(b, a, margin, edgeB);
    if (sb > margin) { return; }

    const bool flip = sb > sa + 0.1f * slop;
    const Polygon2& ref = flip ? b : a;
    const Polygon2& inc = flip ? a : b;
    const int i1 = flip ? edgeB : edgeA;
    const Vec2 v11 = ref.points[i1];
    const Vec2 v12 = ref.points[(i1 + 1) % ref.count];
    const Vec2 normal = ref.normals[i1];

    int i2 = 0;
    float minDot = FLT_MAX;
    for (int i = 0; i < inc.count; ++i) {
        const float d = dot(normal, inc.normals[i]);
        if (d < minDot) {
            minDot = d;
            i2 = i;
        }
    }
    const Vec2 v21 = inc.points[i2];
    const Vec2 v22 = inc.points[(i2 + 1) % inc.count];

    if (maxf(sa, sb) > 0.1f * slop) {
        const SegmentClosest c = closestOnSegments(v11, v12, v21, v22);
        if ((c.s == 0.0f || c.s == 1.0f) && (c.t == 0.0f || c.t == 1.0f)) {
            const float dist = length(c.b - c.a);
            if (dist > margin || dist <= 0.0f) { return; }
            const Vec2 n = (c.b - c.a) * (1.0f / dist);
            out.normal = flip ? -n : n;
            out.points[0] = (c.a + c.b) * 0.5f;
            out.separations[0] = dist;
            out.count = 1;
            return;
        }
    }

    const Vec2 tangent = normalize(v12 - v11);
    const float lower1 = 0.0f;
    const float upper1 = dot(v12 - v11, tangent);
    const float upper2 = dot(v21 - v11, tangent);
    const float lower2 = dot(v22 - v11, tangent);
    const float span = upper2 - lower2;

    out.normal = flip ? -normal : normal;
    if (upper2 < lower1 || lower2 > upper1) {
        // The incident edge lies wholly past the reference edge: its deepest vertex stands in.
        int deepest = 0;
        float s = FLT_MAX;
        for (int i = 0; i < inc.count; ++i) {
            const float d = dot(inc.points[i] - v11, normal);
            if (d < s) {
                s = d;
                deepest = i;
            }
        }
        if (s > margin) { return; }
        out.points[0] = inc.points[deepest] - normal * (0.5f * s);
        out.separations[0] = s;
        out.count = 1;
        return;
    }

    Vec2 vLower = v22, vUpper = v21;
    if (span > FLT_EPSILON) {
        if (lower2 < lower1) { vLower = v22 + (v21 - v22) * ((lower1 - lower2) / span); }
        if (upper2 > upper1) { vUpper = v22 + (v21 - v22) * ((upper1 - lower2) / span); }
    }
    const Vec2 ends[2] = { vLower, vUpper };
    for (int k = 0; k < 2; ++k) {
        const float s = dot(ends[k] - v11, normal);
        if (s > margin) { continue; }
        out.points[out.count] = ends[k] - normal * (0.5f * s);
        out.separations[out.count] = s;
        ++out.count;
    }
}

// A polygon and a circle; the normal points from the polygon to the circle (src/collide2d.cpp:259-291).
TF_HD void collidePolygonCircle(const Polygon2& poly, const Vec2& c, float r, float margin, Planar2& out) {
    int edge = 0;
    float sep = -FLT_MAX;
    for (int i = 0; i < poly.count; ++i) {
        const float s = dot(poly.normals[i], c - poly.points[i]);
        if (s > sep) {
            sep = s;
            edge = i;
        }
    }
    if (sep - r > margin) { return; }
    const Vec2 v1 = poly.points[edge];
    const Vec2 v2 = poly.points[(edge + 1) % poly.count];
    Vec2 surface;
    if (sep > FLT_EPSILON && dot(c - v1, v2 - v1) < 0.0f) {
        surface = v1;
    } else if (sep > FLT_EPSILON && dot(c - v2, v1 - v2) < 0.0f) {
        surface = v2;
    } else {
        const Vec2 n = poly.normals[edge];
        out.normal = n;
        out.points[0] = ((c - n * sep) + (c - n * r)) * 0.5f;
        out.separations[0] = sep - r;
        out.count = 1;
        return;
    }
    const float dist = length(c - surface);
    const float s = dist - r;
    if (s > margin || dist <= 0.0f) { return; }
    const Vec2 n = (c - surface) * (1.0f / dist);
    out.normal = n;
    out.points[0] = (surface + (c - n * r)) * 0.5f;
    out.separations[0] = s;
    out.count = 1;
}

// src/collide2d.cpp:293-303.
TF_HD void collideCircles(const Vec2& ca, float ra, const Vec2& cb, float rb, float margin, Planar2& out) {
    const Vec2 d = cb - ca;
    const float dist = length(d);
    const float s = dist - ra - rb;
    if (s > margin) { return; }
    const Vec2 n = dist > 0.0f ? d * (1.0f / dist) : Vec2{ 1, 0 };
    out.normal = n;
    out.points[0] = ca + n * (ra + 0.5f * s);
    out.separations[0] = s;
    out.count = 1;
}

// A half-plane and a circle; the normal points out of the half-plane (src/collide2d.cpp:325-332).
TF_HD void collideHalfPlaneCircle(const Vec2& normal, float offset, const Vec2& c, float r, float margin, Planar2& out) {
    const float sep = dot(normal, c) - offset;
    if (sep - r > margin) { return; }
    out.normal = normal;
    out.points[0] = ((c - normal * sep) + (c - normal * r)) * 0.5f;
    out.separations[0] = sep - r;
    out.count = 1;
}

// A half-plane (normal out of it) against a polygon, which touches with the edge facing it most
// (src/collide2d.cpp:310-323).
TF_HD void collideHalfPlanePolygon(const Vec2& normal, float offset, const Polygon2& poly, float margin, Planar2& out) {
    int edge = 0;
    float minDot = FLT_MAX;
    for (int i = 0; i < poly.count; ++i) {
        const float d = dot(normal, poly.normals[i]);
        if (d < minDot) {
            minDot = d;
            edge = i;
        }
    }
    out.normal = normal;
    const Vec2 ends[2] = { poly.points[(edge + 1) % poly.count], poly.points[edge] };
    for (int k = 0; k < 2; ++k) {
        const float s = dot(normal, ends[k]) - offset;
        if (s > margin) { continue; }
        out.points[out.count] = ends[k] - normal * (0.5f * s);
        out.separations[out.count] = s;
        ++out.count;
    }
}

// collidePlanar (src/collide2d.cpp:335-421) on two shapes already placed: returns 1 when the planar path
// decided the pair (m.count may be 0), 0 when a profile is empty and the pair goes to the 3D path, and -1
// for a profile this build does not hold.
TF_HD int collidePlanar(const PolyTables& pt, const DShape& sa, const PlanePose& bodyA, const DShape& sb,
                        const PlanePose& bodyB, float margin, float slop, Manifold& m) {
    m.count = 0;
    Profile pa, pb;
    if (!profileOf(pt, sa, bodyA, pa) || !profileOf(pt, sb, bodyB, pb)) { return -1; }
    if (pa.kind == kProfileNone || pb.kind == kProfileNone) { return 0; }
    if (pa.kind == kProfileHalfPlane && pb.kind == kProfileHalfPlane) { return 0; }

    // b's profile comes into a's 2D frame by one turn and shift, and its depths by one lift.
    const Vec2 ta = bodyA.turn, tb = bodyB.turn;
    const Vec2 turn{ ta.x * tb.x + ta.y * tb.y, ta.x * tb.y - ta.y * tb.x };
    const Vec2 gap = bodyB.position - bodyA.position;
    const Vec2 shift{ ta.x * gap.x + ta.y * gap.y, ta.x * gap.y - ta.y * gap.x };
    const float lift = bodyB.depth - bodyA.depth;
    auto turned = [&](const Vec2& p) { return Vec2{ turn.x * p.x - turn.y * p.y, turn.y * p.x + turn.x * p.y }; };
    auto moved = [&](const Vec2& p) { return turned(p) + shift; };

    const bool halfB = pb.kind == kProfileHalfPlane;
    const float lo = maxf(pa.zLo, halfB ? -FLT_MAX : pb.zLo + lift);
    const float hi = minf(pa.zHi, halfB ? FLT_MAX : pb.zHi + lift);
    if (lo > hi) { return 1; }
    const float zMid = 0.5f * (lo + hi);
    // Profiles whose boxes are further apart than the margin cannot touch.
    if (pa.kind != kProfileHalfPlane && !halfB) {
        const Vec2 d = moved(pb.center) - pa.center;
        const float c = fabsf(turn.x), s = fabsf(turn.y);
        const Vec2 ea = pa.extent + Vec2{ margin, margin }, eb = pb.extent;
        if (fabsf(d.x) > ea.x + c * eb.x + s * eb.y || fabsf(d.y) > ea.y + s * eb.x + c * eb.y) { return 1; }
        const Vec2 db{ turn.x * d.x + turn.y * d.y, turn.x * d.y - turn.y * d.x };
        if (fabsf(db.x) > eb.x + c * ea.x + s * ea.y || fabsf(db.y) > eb.y + s * ea.x + c * ea.y) { return 1; }
    }

    // b's polygon in a's frame, in place: its profile is not used again.
    if (pb.kind == kProfilePolygon) {
        for (int i = 0; i < pb.count; ++i) {
            pb.points[i] = moved(pb.points[i]);
            pb.normals[i] = turned(pb.normals[i]);
        }
    }
    const Polygon2 polyA{ pa.points, pa.normals, pa.count };
    const Polygon2 polyB{ pb.points, pb.normals, pb.count };

    Planar2 out;
    out.count = 0;
    if (pa.kind == kProfileHalfPlane) {
        const float offset = pa.offset - pa.tilt * zMid;
        if (pb.kind == kProfileCircle) {
            collideHalfPlaneCircle(pa.normal, offset, moved(pb.center), pb.radius, margin, out);
        } else {
            collideHalfPlanePolygon(pa.normal, offset, polyB, margin, out);
        }
    } else if (halfB) {
        const Vec2 normal = turned(pb.normal);
        const float offset = pb.offset + dot(normal, shift) - pb.tilt * (zMid - lift);
        if (pa.kind == kProfileCircle) {
            collideHalfPlaneCircle(normal, offset, pa.center, pa.radius, margin, out);
        } else {
            collideHalfPlanePolygon(normal, offset, polyA, margin, out);
        }
        out.normal = -out.normal;
    } else if (pa.kind == kProfileCircle && pb.kind == kProfileCircle) {
        collideCircles(pa.center, pa.radius, moved(pb.center), pb.radius, margin, out);
    } else if (pa.kind == kProfileCircle) {
        collidePolygonCircle(polyB, pa.center, pa.radius, margin, out);
        out.normal = -out.normal;
    } else if (pb.kind == kProfileCircle) {
        collidePolygonCircle(polyA, moved(pb.center), pb.radius, margin, out);
    } else {
        collidePolygons(polyA, polyB, margin, slop, out);
    }
    if (out.count == 0) { return 1; }

    // The normal stays in the plane, so a contact never pushes layers apart in depth.
    auto toPlane = [&](const Vec2& p) { return Vec2{ ta.x * p.x - ta.y * p.y, ta.y * p.x + ta.x * p.y }; };
    const Vec2 normal = toPlane(out.normal);
    m.normal = bodyA.axisU * normal.x + bodyA.axisV * normal.y;
    const Vec3 lifted = bodyA.normal * (bodyA.depth + zMid);
    for (int i = 0; i < out.count; ++i) {
        const Vec2 p = toPlane(out.points[i]) + bodyA.position;
        m.points[i].position = bodyA.axisU * p.x + bodyA.axisV * p.y + lifted;
        m.points[i].separation = out.separations[i];
    }
    m.count = out.count;
    return 1;
}

// Distance from the centroid to the nearest face a planar body can move against, for the continuous test
// (src/world.cpp:1252-1266). The reference caches it under the plane normal in the shape's frame; which faces
// count changes only when a face normal crosses 0.9 against that normal, so the value is found afresh here.
TF_HD float innerExtent(const PolyTables& pt, const DShape& s, const DBody& b) {
    if ((s.kind != kConvex && s.kind != kCylinder) || !isPlanar(b)) { return s.minExtent; }
    const Vec3 n = unrotate(s.local.q, unrotate(b.xf.q, planeNormal(b)));
    if (s.kind == kCylinder) { return fabsf(n.z) > 0.9f ? s.radius : s.minExtent; }
    if (s.poly < 0) { return s.minExtent; }
    const DPoly& P = pt.polys[s.poly];
    float inner = FLT_MAX;
    for (int i = 0; i < P.fCount; ++i) {
        const Vec3 fn = pt.normals[P.fFirst + i];
        if (fabsf(dot(fn, n)) > 0.9f) { continue; }
        inner = minf(inner, pt.offsets[P.fFirst + i] - dot(fn, s.centroid));
    }
    return inner < FLT_MAX ? inner : s.minExtent;
}

}
