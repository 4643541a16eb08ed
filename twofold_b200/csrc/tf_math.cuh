// Vector, quaternion and matrix arithmetic shared by host and device code.
//
// Every operation evaluates the same IEEE single-precision operations in the same order as the
// reference's include/twofold/math.h, so that with contraction off (nvcc --fmad=false, host
// -ffp-contract=off) and IEEE division and square root, device results are bit-identical to the
// reference's CPU results. Operator forms are written out left to right where C++ would group them the
// same way (a + b + c is (a + b) + c).
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define TF_HD __host__ __device__ __forceinline__
#define TF_D __device__ __forceinline__
#else
#define TF_HD inline
#define TF_D inline
#endif

namespace tfb {

struct Vec2 {
    float x, y;
};

struct Vec3 {
    float x, y, z;
};

struct Quat {
    float x, y, z, w;
};

// Row-major, r[i] is row i.
struct Mat3 {
    Vec3 r[3];
};

struct Transform {
    Vec3 p;
    Quat q;
};

TF_HD Vec2 v2(float x, float y) { return { x, y }; }
TF_HD Vec3 v3(float x, float y, float z) { return { x, y, z }; }
TF_HD Vec3 zero3() { return { 0.0f, 0.0f, 0.0f }; }
TF_HD Quat qid() { return { 0.0f, 0.0f, 0.0f, 1.0f }; }

TF_HD Vec2 operator+(Vec2 a, Vec2 b) { return { a.x + b.x, a.y + b.y }; }
TF_HD Vec2 operator-(Vec2 a, Vec2 b) { return { a.x - b.x, a.y - b.y }; }
TF_HD Vec2 operator-(Vec2 a) { return { -a.x, -a.y }; }
TF_HD Vec2 operator*(Vec2 a, float s) { return { a.x * s, a.y * s }; }
TF_HD Vec2 operator*(float s, Vec2 a) { return a * s; }
TF_HD float dot(Vec2 a, Vec2 b) { return a.x * b.x + a.y * b.y; }
TF_HD float cross(Vec2 a, Vec2 b) { return a.x * b.y - a.y * b.x; }
TF_HD float length(Vec2 v) { return sqrtf(dot(v, v)); }
TF_HD Vec2 normalize(Vec2 v) {
    const float l = length(v);
    return l > 0 ? v * (1.0f / l) : Vec2{ 0.0f, 0.0f };
}

TF_HD Vec3 operator+(const Vec3& a, const Vec3& b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
TF_HD Vec3 operator-(const Vec3& a, const Vec3& b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
TF_HD Vec3 operator-(const Vec3& a) { return { -a.x, -a.y, -a.z }; }
TF_HD Vec3 operator*(const Vec3& a, float s) { return { a.x * s, a.y * s, a.z * s }; }
TF_HD Vec3 operator*(float s, const Vec3& a) { return a * s; }
TF_HD Vec3 operator/(const Vec3& a, float s) { return { a.x / s, a.y / s, a.z / s }; }
TF_HD Vec3& operator+=(Vec3& a, const Vec3& b) {
    a.x += b.x;
    a.y += b.y;
    a.z += b.z;
    return a;
}
TF_HD Vec3& operator-=(Vec3& a, const Vec3& b) {
    a.x -= b.x;
    a.y -= b.y;
    a.z -= b.z;
    return a;
}
TF_HD bool operator==(const Vec3& a, const Vec3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

TF_HD float comp(const Vec3& v, int i) { return i == 0 ? v.x : i == 1 ? v.y : v.z; }
TF_HD void setComp(Vec3& v, int i, float s) {
    if (i == 0) {
        v.x = s;
    } else if (i == 1) {
        v.y = s;
    } else {
        v.z = s;
    }
}

TF_HD float dot(const Vec3& a, const Vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
TF_HD Vec3 cross(const Vec3& a, const Vec3& b) {
    return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x };
}
TF_HD float lengthSquared(const Vec3& v) { return dot(v, v); }
TF_HD float length(const Vec3& v) { return sqrtf(dot(v, v)); }
TF_HD Vec3 normalize(const Vec3& v) {
    const float l = length(v);
    return l > 0 ? v * (1.0f / l) : Vec3{ 0.0f, 0.0f, 0.0f };
}
TF_HD Vec3 minVec(const Vec3& a, const Vec3& b) {
    return { a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z };
}
TF_HD Vec3 maxVec(const Vec3& a, const Vec3& b) {
    return { a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z };
}

// A unit vector orthogonal to n (math.h:70-73).
TF_HD Vec3 perpendicular(const Vec3& n) {
    if (fabsf(n.x) > 0.57735f) { return normalize(Vec3{ n.y, -n.x, 0.0f }); }
    return normalize(Vec3{ 0.0f, n.z, -n.y });
}

// std::fmax / std::fmin semantics, NaN and signed zeros included (src/internal.h:28-45).
TF_HD float maxf(float a, float b) {
    if (a == b || a != a || b != b) {
        if (a != a) { return b; }
        if (b != b) { return a; }
        return a == 0.0f ? a + b : a;
    }
    return a > b ? a : b;
}
TF_HD float minf(float a, float b) {
    if (a == b || a != a || b != b) {
        if (a != a) { return b; }
        if (b != b) { return a; }
        return a == 0.0f ? -(-a + -b) : a;
    }
    return a < b ? a : b;
}

TF_HD Mat3 mzero() { return { { { 0, 0, 0 }, { 0, 0, 0 }, { 0, 0, 0 } } }; }
TF_HD Mat3 mid() { return { { { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } } }; }
TF_HD Mat3 mdiag(const Vec3& d) {
    Mat3 m = mzero();
    m.r[0].x = d.x;
    m.r[1].y = d.y;
    m.r[2].z = d.z;
    return m;
}
TF_HD Mat3 outer(const Vec3& a, const Vec3& b) { return { { b * a.x, b * a.y, b * a.z } }; }
TF_HD Vec3 column(const Mat3& m, int i) { return { comp(m.r[0], i), comp(m.r[1], i), comp(m.r[2], i) }; }
TF_HD Vec3 operator*(const Mat3& m, const Vec3& v) { return { dot(m.r[0], v), dot(m.r[1], v), dot(m.r[2], v) }; }
TF_HD Mat3 operator*(const Mat3& a, const Mat3& b) {
    Mat3 m;
    const Vec3 c0 = column(b, 0), c1 = column(b, 1), c2 = column(b, 2);
    for (int i = 0; i < 3; ++i) { m.r[i] = { dot(a.r[i], c0), dot(a.r[i], c1), dot(a.r[i], c2) }; }
    return m;
}
TF_HD Mat3 operator+(const Mat3& a, const Mat3& b) { return { { a.r[0] + b.r[0], a.r[1] + b.r[1], a.r[2] + b.r[2] } }; }
TF_HD Mat3 operator-(const Mat3& a, const Mat3& b) { return { { a.r[0] - b.r[0], a.r[1] - b.r[1], a.r[2] - b.r[2] } }; }
TF_HD Mat3 operator*(const Mat3& a, float s) { return { { a.r[0] * s, a.r[1] * s, a.r[2] * s } }; }
TF_HD Mat3 transpose(const Mat3& m) { return { { column(m, 0), column(m, 1), column(m, 2) } }; }

TF_HD Mat3 inverse(const Mat3& m) {
    const Vec3 c0 = cross(m.r[1], m.r[2]);
    const Vec3 c1 = cross(m.r[2], m.r[0]);
    const Vec3 c2 = cross(m.r[0], m.r[1]);
    float det = dot(m.r[0], c0);
    if (det == 0.0f) { return mzero(); }
    det = 1.0f / det;
    Mat3 inv;
    inv.r[0] = Vec3{ c0.x, c1.x, c2.x } * det;
    inv.r[1] = Vec3{ c0.y, c1.y, c2.y } * det;
    inv.r[2] = Vec3{ c0.z, c1.z, c2.z } * det;
    return inv;
}

TF_HD Vec3 qvec(const Quat& q) { return { q.x, q.y, q.z }; }
TF_HD Quat operator*(const Quat& a, const Quat& b) {
    return { a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
             a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z };
}
TF_HD Quat operator-(const Quat& q) { return { -q.x, -q.y, -q.z, -q.w }; }
TF_HD Quat conjugate(const Quat& q) { return { -q.x, -q.y, -q.z, q.w }; }
TF_HD Vec3 rotate(const Quat& q, const Vec3& v) {
    const Vec3 u = qvec(q);
    const Vec3 t = cross(u, v) * 2.0f;
    return v + t * q.w + cross(u, t);
}
TF_HD Vec3 unrotate(const Quat& q, const Vec3& v) { return rotate(conjugate(q), v); }
TF_HD Mat3 toMat3(const Quat& q) {
    const float xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
    const float xy = q.x * q.y, xz = q.x * q.z, yz = q.y * q.z;
    const float wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
    Mat3 m;
    m.r[0] = { 1.0f - 2.0f * (yy + zz), 2.0f * (xy - wz), 2.0f * (xz + wy) };
    m.r[1] = { 2.0f * (xy + wz), 1.0f - 2.0f * (xx + zz), 2.0f * (yz - wx) };
    m.r[2] = { 2.0f * (xz - wy), 2.0f * (yz + wx), 1.0f - 2.0f * (xx + yy) };
    return m;
}
TF_HD float dot(const Quat& a, const Quat& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
TF_HD Quat normalize(const Quat& q) {
    const float l = sqrtf(dot(q, q));
    return l > 0 ? Quat{ q.x / l, q.y / l, q.z / l, q.w / l } : qid();
}

// q advanced by angular velocity w over h (math.h:227-230).
TF_HD Quat integrate(const Quat& q, const Vec3& w, float h) {
    const Quat dq = Quat{ w.x, w.y, w.z, 0.0f } * q;
    return normalize(Quat{ q.x + 0.5f * h * dq.x, q.y + 0.5f * h * dq.y, q.z + 0.5f * h * dq.z, q.w + 0.5f * h * dq.w });
}

TF_HD Vec3 apply(const Transform& t, const Vec3& v) { return t.p + rotate(t.q, v); }
TF_HD Vec3 applyInverse(const Transform& t, const Vec3& v) { return unrotate(t.q, v - t.p); }
TF_HD Transform operator*(const Transform& a, const Transform& b) { return { apply(a, b.p), a.q * b.q }; }

}
