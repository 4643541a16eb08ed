// The differentiable model of a recorded run and its hand-written adjoint, in float and in double.
//
// The model is the substepped soft solve with integration (src/world.cpp:1649-1684, src/solver.cpp:319-460 in
// the reference) with each step's contact set held fixed: the contacts, their anchors, frames, adjusted
// separations and warm-start impulses, the color lists and the awake flags come from the recorded step
// (tf_tape.h). What flows through it: the bodies' centers of mass, rotations and velocities, the masses
// (inverse mass, and local inverse inertia scaling with it) and the shapes' friction (a contact's friction is
// sqrt(friction A * friction B), src/world.cpp:39-40, 951-955). Contacts keep their step-start anchors for
// the whole step (no mid-step collision) and the speed limits are taken as inactive.
//
// Forward: one warp per world walks every step, writing the state at each step boundary (the checkpoints).
// Backward: for each step from the last, the warp runs the step again from its checkpoint, logging the
// inputs of every contact solve and integration, then walks the same operations in reverse, carrying
// adjoints of the state back to the step's start and adding up the adjoints of masses and frictions.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/twofold_b200.h"
#include "tf_tape.h"

namespace tfb {

int noteError(int code, const std::string& msg);

namespace adj {

// ---------------------------------------------------------------------------------------------------------
// Small vector algebra in T.

template <class T>
struct V3 {
    T x, y, z;
};
template <class T>
struct Q4 {
    T x, y, z, w;
};
template <class T>
struct M3 {
    V3<T> r[3];
};

template <class T> __device__ __forceinline__ V3<T> operator+(V3<T> a, V3<T> b) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
template <class T> __device__ __forceinline__ V3<T> operator-(V3<T> a, V3<T> b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
template <class T> __device__ __forceinline__ V3<T> operator*(V3<T> a, T s) { return { a.x * s, a.y * s, a.z * s }; }
template <class T> __device__ __forceinline__ T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> __device__ __forceinline__ V3<T> cross(V3<T> a, V3<T> b) {
    return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x };
}
template <class T> __device__ __forceinline__ V3<T> mul(const M3<T>& m, V3<T> v) { return { dot(m.r[0], v), dot(m.r[1], v), dot(m.r[2], v) }; }
template <class T> __device__ __forceinline__ void addOuter(M3<T>& m, V3<T> a, V3<T> b, T s) {
    m.r[0] = m.r[0] + b * (a.x * s);
    m.r[1] = m.r[1] + b * (a.y * s);
    m.r[2] = m.r[2] + b * (a.z * s);
}
template <class T> __device__ __forceinline__ M3<T> zeroM() { return { { { 0, 0, 0 }, { 0, 0, 0 }, { 0, 0, 0 } } }; }
template <class T> __device__ __forceinline__ V3<T> zeroV() { return { 0, 0, 0 }; }
template <class T> __device__ __forceinline__ M3<T> transposeM(const M3<T>& m) {
    return { { { m.r[0].x, m.r[1].x, m.r[2].x }, { m.r[0].y, m.r[1].y, m.r[2].y }, { m.r[0].z, m.r[1].z, m.r[2].z } } };
}
template <class T> __device__ __forceinline__ M3<T> mmul(const M3<T>& a, const M3<T>& b) {
    const M3<T> bt = transposeM(b);
    M3<T> o;
    for (int i = 0; i < 3; ++i) { o.r[i] = { dot(a.r[i], bt.r[0]), dot(a.r[i], bt.r[1]), dot(a.r[i], bt.r[2]) }; }
    return o;
}
template <class T> __device__ __forceinline__ M3<T> madd(const M3<T>& a, const M3<T>& b) {
    return { { a.r[0] + b.r[0], a.r[1] + b.r[1], a.r[2] + b.r[2] } };
}

// Hamilton product and its adjoints with respect to each factor.
template <class T> __device__ __forceinline__ Q4<T> qmul(Q4<T> a, Q4<T> b) {
    return { a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
             a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z };
}
template <class T> __device__ __forceinline__ Q4<T> qmulAdjA(Q4<T> g, Q4<T> b) {
    return { g.x * b.w - g.y * b.z + g.z * b.y - g.w * b.x, g.x * b.z + g.y * b.w - g.z * b.x - g.w * b.y,
             -g.x * b.y + g.y * b.x + g.z * b.w - g.w * b.z, g.x * b.x + g.y * b.y + g.z * b.z + g.w * b.w };
}
template <class T> __device__ __forceinline__ Q4<T> qmulAdjB(Q4<T> g, Q4<T> a) {
    return { g.x * a.w + g.y * a.z - g.z * a.y - g.w * a.x, -g.x * a.z + g.y * a.w + g.z * a.x - g.w * a.y,
             g.x * a.y - g.y * a.x + g.z * a.w - g.w * a.z, g.x * a.x + g.y * a.y + g.z * a.z + g.w * a.w };
}
template <class T> __device__ __forceinline__ Q4<T> conj(Q4<T> q) { return { -q.x, -q.y, -q.z, q.w }; }
template <class T> __device__ __forceinline__ Q4<T> qadd(Q4<T> a, Q4<T> b) { return { a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w }; }

// rotate(q, v) = v + w t + u x t with t = 2 u x v (u the vector part), as math.h writes it.
template <class T> __device__ __forceinline__ V3<T> rotate(Q4<T> q, V3<T> v) {
    const V3<T> u{ q.x, q.y, q.z };
    const V3<T> t = cross(u, v) * T(2);
    return v + t * q.w + cross(u, t);
}
// Adjoint of rotate: given g = d/d(result), adds d/dq to qg and returns d/dv.
template <class T> __device__ __forceinline__ V3<T> rotateAdj(Q4<T> q, V3<T> v, V3<T> g, Q4<T>& qg) {
    const V3<T> u{ q.x, q.y, q.z };
    const V3<T> t = cross(u, v) * T(2);
    const V3<T> tg = g * q.w + cross(g, u);
    const V3<T> ug = cross(t, g) + cross(v, tg) * T(2);
    qg.x += ug.x;
    qg.y += ug.y;
    qg.z += ug.z;
    qg.w += dot(g, t);
    return g + cross(tg, u) * T(2);
}

template <class T> __device__ __forceinline__ M3<T> toMat3(Q4<T> q) {
    const T xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z, xy = q.x * q.y, xz = q.x * q.z, yz = q.y * q.z;
    const T wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
    M3<T> m;
    m.r[0] = { 1 - 2 * (yy + zz), 2 * (xy - wz), 2 * (xz + wy) };
    m.r[1] = { 2 * (xy + wz), 1 - 2 * (xx + zz), 2 * (yz - wx) };
    m.r[2] = { 2 * (xz - wy), 2 * (yz + wx), 1 - 2 * (xx + yy) };
    return m;
}
template <class T> __device__ __forceinline__ Q4<T> toMat3Adj(Q4<T> q, const M3<T>& g) {
    const T x = q.x, y = q.y, z = q.z, w = q.w;
    const V3<T>* r = g.r;
    Q4<T> o;
    o.x = r[0].y * 2 * y + r[0].z * 2 * z + r[1].x * 2 * y - r[1].y * 4 * x - r[1].z * 2 * w + r[2].x * 2 * z +
          r[2].y * 2 * w - r[2].z * 4 * x;
    o.y = -r[0].x * 4 * y + r[0].y * 2 * x + r[0].z * 2 * w + r[1].x * 2 * x + r[1].z * 2 * z - r[2].x * 2 * w +
          r[2].y * 2 * z - r[2].z * 4 * y;
    o.z = -r[0].x * 4 * z - r[0].y * 2 * w + r[0].z * 2 * x + r[1].x * 2 * w - r[1].y * 4 * z + r[1].z * 2 * y +
          r[2].x * 2 * x + r[2].y * 2 * y;
    o.w = -r[0].y * 2 * z + r[0].z * 2 * y + r[1].x * 2 * z - r[1].z * 2 * x - r[2].x * 2 * y + r[2].y * 2 * x;
    return o;
}

template <class T> __device__ __forceinline__ T sqrtT(T x) { return sqrt(x); }

// integrate(q, w, h) = normalize(q + (h/2) (w, 0) q) (math.h:227-230).
template <class T> __device__ __forceinline__ Q4<T> integrateQ(Q4<T> q, V3<T> w, T h) {
    const Q4<T> d = qmul(Q4<T>{ w.x, w.y, w.z, T(0) }, q);
    const T c = T(0.5) * h;
    const Q4<T> u{ q.x + c * d.x, q.y + c * d.y, q.z + c * d.z, q.w + c * d.w };
    const T l = sqrtT(u.x * u.x + u.y * u.y + u.z * u.z + u.w * u.w);
    return l > T(0) ? Q4<T>{ u.x / l, u.y / l, u.z / l, u.w / l } : Q4<T>{ 0, 0, 0, 1 };
}
template <class T> __device__ __forceinline__ void integrateQAdj(Q4<T> q, V3<T> w, T h, Q4<T> g, Q4<T>& qg, V3<T>& wg) {
    const Q4<T> d = qmul(Q4<T>{ w.x, w.y, w.z, T(0) }, q);
    const T c = T(0.5) * h;
    const Q4<T> u{ q.x + c * d.x, q.y + c * d.y, q.z + c * d.z, q.w + c * d.w };
    const T l = sqrtT(u.x * u.x + u.y * u.y + u.z * u.z + u.w * u.w);
    if (!(l > T(0))) { return; }
    const Q4<T> n{ u.x / l, u.y / l, u.z / l, u.w / l };
    const T gn = g.x * n.x + g.y * n.y + g.z * n.z + g.w * n.w;
    const Q4<T> ug{ (g.x - n.x * gn) / l, (g.y - n.y * gn) / l, (g.z - n.z * gn) / l, (g.w - n.w * gn) / l };
    qg = qadd(qg, ug);
    const Q4<T> dg{ ug.x * c, ug.y * c, ug.z * c, ug.w * c };
    const Q4<T> wq = qmulAdjA(dg, q);
    wg.x += wq.x;
    wg.y += wq.y;
    wg.z += wq.z;
    qg = qadd(qg, qmulAdjB(dg, Q4<T>{ w.x, w.y, w.z, T(0) }));
}

template <class T> __device__ __forceinline__ void atomicAddT(T* p, T v) { atomicAdd(p, v); }

// ---------------------------------------------------------------------------------------------------------
// Model data.

template <class T>
struct Softness {
    T biasRate, massScale, impulseScale;
};

// Per-step state of one contact point while the step runs.
template <class T>
struct PointState {
    T n;      // normal impulse
    V3<T> t;  // tangent impulse
    T maxN;   // largest normal impulse added this step
};

template <class T>
struct Model {
    AdjointSetup S;
    T h, invH, dt;
    V3<T> gravity;
    Softness<T> contactSoft, staticSoft;
    T maxPushout, restThreshold;
    // Parameters in T.
    const T* mass;      // per body
    const T* friction;  // per shape
    const T* init;      // per body 13: com, q, v, w (the initial state)
    // Checkpoints: (nSteps + 1) x totalBodies x 13.
    T* states;
    // Per body working arrays of the current step.
    T* invM;    // 1
    T* invI;    // 9 world inverse inertia
    T* dp;      // 3
    T* dq;      // 4
    T* qBase;   // 4
    PointState<T>* points;  // contactSlots x 4
    // Backward only.
    T* stateAdj;   // totalBodies x 13
    T* dpAdj;      // 3
    T* dqAdj;      // 4
    T* qBaseAdj;   // 4
    T* invMAdj;    // 1
    T* invIAdj;    // 9
    PointState<T>* pointAdj;  // contactSlots x 4
    T* massAdj;      // per body (output, summed)
    T* frictionAdj;  // per shape (output, summed)
    T* log;          // per slot and world: logStride values
    uint64_t logStride;
    T* integLog;     // per slot, substep and body: q (4) and w (3) before the position update, dp (3) after it
    T* scratch;      // per slot: one state
    // Per world, the forward's branch signature (k_model_forward writes it when not null): a sum over every row
    // the run solved of a hash of (step, operation, row, which side of each non-smooth point the row took).
    unsigned long long* branches;
};


constexpr int kIntegWords = 10;

// The working arrays of one step's recomputation. The backward recomputes a chunk of steps at once, one warp
// per world and step, so each step of the chunk has its own slot; the forward uses slot 0.
template <class T>
struct Slot {
    T* invM;
    T* invI;
    T* dp;
    T* dq;
    T* qBase;
    PointState<T>* points;
    T* log;       // nWorlds x logStride
    T* integLog;  // substeps x totalBodies x kIntegWords
    T* scratch;   // totalBodies x kState: the recomputed step's end state
};

constexpr int kState = 13;

template <class T>
__device__ __forceinline__ Slot<T> slotOf(const Model<T>& M, uint32_t k) {
    const size_t nb = M.S.totalBodies;
    Slot<T> W;
    W.invM = M.invM + k * nb;
    W.invI = M.invI + k * 9 * nb;
    W.dp = M.dp + k * 3 * nb;
    W.dq = M.dq + k * 4 * nb;
    W.qBase = M.qBase + k * 4 * nb;
    W.points = M.points + k * (size_t)M.S.contactSlots * 4;
    W.log = M.log ? M.log + k * (size_t)M.S.nWorlds * M.logStride : nullptr;
    W.integLog = M.integLog ? M.integLog + k * (size_t)M.S.substeps * nb * kIntegWords : nullptr;
    W.scratch = M.scratch ? M.scratch + k * nb * kState : nullptr;
    return W;
}

template <class T> __device__ __forceinline__ V3<T> ld3(const T* p) { return { p[0], p[1], p[2] }; }
template <class T> __device__ __forceinline__ void st3(T* p, V3<T> v) { p[0] = v.x, p[1] = v.y, p[2] = v.z; }
template <class T> __device__ __forceinline__ Q4<T> ld4(const T* p) { return { p[0], p[1], p[2], p[3] }; }
template <class T> __device__ __forceinline__ void st4(T* p, Q4<T> q) { p[0] = q.x, p[1] = q.y, p[2] = q.z, p[3] = q.w; }
template <class T> __device__ __forceinline__ V3<T> fl3(const float* p) { return { T(p[0]), T(p[1]), T(p[2]) }; }
template <class T> __device__ __forceinline__ M3<T> ldM(const T* p) {
    return { { { p[0], p[1], p[2] }, { p[3], p[4], p[5] }, { p[6], p[7], p[8] } } };
}
template <class T> __device__ __forceinline__ void stM(T* p, const M3<T>& m) {
    for (int r = 0; r < 3; ++r) { p[3 * r] = m.r[r].x, p[3 * r + 1] = m.r[r].y, p[3 * r + 2] = m.r[r].z; }
}

// A body as a contact solve sees it.
template <class T>
struct SBody {
    V3<T> v, w, dp;
    Q4<T> dq;
    T im;
    M3<T> I;
    bool moves;
};

// One direction at a contact point: lever arms are constants (recorded anchors x direction).
template <class T>
struct Axis {
    V3<T> d, armA, armB, angA, angB;
    T dd, k, mass;
    bool on;
};

template <class T>
__device__ __forceinline__ Axis<T> makeAxis(const SBody<T>& a, const SBody<T>& b, V3<T> ra, V3<T> rb, V3<T> d) {
    Axis<T> x;
    x.d = d;
    x.armA = cross(ra, d);
    x.armB = cross(rb, d);
    x.angA = mul(a.I, x.armA);
    x.angB = mul(b.I, x.armB);
    x.dd = dot(d, d);
    x.k = a.im * x.dd + b.im * x.dd + dot(x.armA, x.angA) + dot(x.armB, x.angB);
    x.on = x.k > T(1e-6) * (a.im + b.im);
    x.mass = x.on ? T(1) / x.k : T(0);
    return x;
}

// Adjoint of the effective mass: mass = 1/k with k from both bodies' inverse mass and inertia.
template <class T>
__device__ __forceinline__ void axisMassAdj(const Axis<T>& x, T massAdj, T& imA, M3<T>& IA, T& imB, M3<T>& IB) {
    if (!x.on) { return; }
    const T kg = -massAdj * x.mass * x.mass;
    imA += kg * x.dd;
    imB += kg * x.dd;
    addOuter(IA, x.armA, x.armA, kg);
    addOuter(IB, x.armB, x.armB, kg);
}

template <class T>
__device__ __forceinline__ T speedAlong(const SBody<T>& a, const SBody<T>& b, const Axis<T>& x) {
    return dot(x.d, b.v - a.v) + dot(x.armB, b.w) - dot(x.armA, a.w);
}

template <class T>
__device__ __forceinline__ void push(SBody<T>& a, SBody<T>& b, const Axis<T>& x, T impulse) {
    if (a.moves) {
        a.v = a.v - x.d * (a.im * impulse);
        a.w = a.w - x.angA * impulse;
    }
    if (b.moves) {
        b.v = b.v + x.d * (b.im * impulse);
        b.w = b.w + x.angB * impulse;
    }
}

// Adjoints of one body during a contact's reverse pass.
template <class T>
struct BodyAdj {
    V3<T> v, w, dp;
    Q4<T> dq;
    T im;
    M3<T> I;
};

template <class T>
__device__ __forceinline__ T pushAdj(const SBody<T>& a, const SBody<T>& b, const Axis<T>& x, T impulse, BodyAdj<T>& ga,
                                     BodyAdj<T>& gb) {
    T g = 0;
    if (a.moves) {
        g -= a.im * dot(x.d, ga.v) + dot(x.angA, ga.w);
        ga.im -= impulse * dot(x.d, ga.v);
        addOuter(ga.I, ga.w, x.armA, -impulse);
    }
    if (b.moves) {
        g += b.im * dot(x.d, gb.v) + dot(x.angB, gb.w);
        gb.im += impulse * dot(x.d, gb.v);
        addOuter(gb.I, gb.w, x.armB, impulse);
    }
    return g;
}

template <class T>
__device__ __forceinline__ void speedAdj(const Axis<T>& x, T g, BodyAdj<T>& ga, BodyAdj<T>& gb) {
    ga.v = ga.v - x.d * g;
    gb.v = gb.v + x.d * g;
    ga.w = ga.w - x.armA * g;
    gb.w = gb.w + x.armB * g;
}

// The recorded contact in T.
template <class T>
struct CData {
    int count;
    V3<T> n, t1, t2;
    V3<T> ra[4], rb[4];
    T adjSep[4], relVel[4];
    T restitution;
};

template <class T>
__device__ __forceinline__ CData<T> loadContact(const TapeContact& c) {
    CData<T> d;
    d.count = c.count;
    d.n = fl3<T>(c.normal);
    d.t1 = fl3<T>(c.t1);
    d.t2 = fl3<T>(c.t2);
    for (int i = 0; i < 4; ++i) {
        d.ra[i] = fl3<T>(c.anchorA[i]);
        d.rb[i] = fl3<T>(c.anchorB[i]);
        d.adjSep[i] = T(c.adjSep[i]);
        d.relVel[i] = T(c.relVel[i]);
    }
    d.restitution = T(c.restitution);
    return d;
}

// One point of a recorded contact. The reverse walk reaches a point's values through selects over the four
// (pointOf, pick4, put4) so that the contact's arrays stay in registers: an array indexed at run time lives in
// local memory, whose loads stall the walk's dependent chain.
template <class T>
struct CPoint {
    V3<T> ra, rb;
    T adjSep, relVel;
};

template <class U>
__device__ __forceinline__ U pick4(const U (&v)[4], int i) {
    U r = v[0];
    if (i == 1) { r = v[1]; }
    if (i == 2) { r = v[2]; }
    if (i == 3) { r = v[3]; }
    return r;
}

template <class U>
__device__ __forceinline__ void put4(U (&v)[4], int i, const U& x) {
    if (i == 0) { v[0] = x; }
    if (i == 1) { v[1] = x; }
    if (i == 2) { v[2] = x; }
    if (i == 3) { v[3] = x; }
}

template <class T>
__device__ __forceinline__ CPoint<T> pointOf(const CData<T>& c, int i) {
    return { pick4(c.ra, i), pick4(c.rb, i), pick4(c.adjSep, i), pick4(c.relVel, i) };
}

// ---------------------------------------------------------------------------------------------------------
// Contact operations: forward, and reverse from the logged inputs.

enum Op : int { kWarm = 0, kBias = 1, kRelax = 2, kRestitute = 3 };

// The record a contact operation leaves for its reverse, kCallWords values: what the reverse cannot rebuild
// from the step's constants (axes, inverse masses and displacements are rebuilt).
//   [0, 20)  each point's state before the operation: normal impulse, tangent impulse (3), largest normal impulse
//   [20, 24) each normal row's (or restitution row's) approach speed along the normal, by point
//   [24, 36) each friction row's speeds along the two tangents and the normal impulse that bounds it, by row
// A color's records are consecutive, so the reverse walk copies a color's batch to shared memory in one go.
constexpr int kCallWords = 36;
constexpr int kSpeedAt = 20;
constexpr int kFrictionAt = 24;

template <class T>
__device__ __forceinline__ void writeCall(T* log, const PointState<T>* p) {
    for (int i = 0; i < 4; ++i) {
        log[5 * i] = p[i].n;
        st3(log + 5 * i + 1, p[i].t);
        log[5 * i + 4] = p[i].maxN;
    }
}

// The normal row of point i (src/solver.cpp:364-392). Returns the impulse added.
// The branches of one row that change the model's derivative, for the branch signature: bit 0 the axis has
// an effective mass, bits 1-2 the bias case, bit 3 the impulse clamp; friction: the axes, the cone clamp, a
// nonzero magnitude; restitution: whether the point restitutes and the clamp. (The largest impulse of a step,
// a running maximum, decides only whether a point restitutes, which the restitution bits hold.)
template <class T>
__device__ __forceinline__ T normalRow(const Model<T>& M, SBody<T>& a, SBody<T>& b, const CData<T>& c, int i,
                                       PointState<T>& p, bool useBias, const Softness<T>& soft, uint32_t* br = nullptr,
                                       T* speedOut = nullptr) {
    const Axis<T> x = makeAxis(a, b, c.ra[i], c.rb[i], c.n);
    const V3<T> d = b.dp - a.dp + rotate(b.dq, c.rb[i]) - rotate(a.dq, c.ra[i]);
    const T sep = dot(d, c.n) + c.adjSep[i];
    T bias = 0, ms = 1, is = 0;
    uint32_t biasKind = 0;
    if (sep > T(0)) {
        bias = sep * M.invH;
        biasKind = 1;
    } else if (useBias) {
        biasKind = soft.biasRate * sep > -M.maxPushout ? 2 : 3;
        bias = fmax(soft.biasRate * sep, -M.maxPushout);
        ms = soft.massScale;
        is = soft.impulseScale;
    }
    const T vn = speedAlong(a, b, x);
    if (speedOut) { *speedOut = vn; }
    const T imp = -x.mass * ms * (vn + bias) - is * p.n;
    const T total = fmax(p.n + imp, T(0));
    const T delta = total - p.n;
    if (br) { *br = (x.on ? 1u : 0u) | biasKind << 1 | (p.n + imp > T(0) ? 8u : 0u); }
    p.n = total;
    p.maxN = fmax(p.maxN, delta);
    push(a, b, x, delta);
    return delta;
}

template <class T>
__device__ __forceinline__ void normalRowAdj(const Model<T>& M, const SBody<T>& a, const SBody<T>& b, const CData<T>& c,
                                             const CPoint<T>& q, const PointState<T>& p0, T vn, bool useBias, const Softness<T>& soft,
                                             BodyAdj<T>& ga, BodyAdj<T>& gb, PointState<T>& gp) {
    const Axis<T> x = makeAxis(a, b, q.ra, q.rb, c.n);
    const V3<T> d = b.dp - a.dp + rotate(b.dq, q.rb) - rotate(a.dq, q.ra);
    const T sep = dot(d, c.n) + q.adjSep;
    T bias = 0, ms = 1, is = 0;
    int biasKind = 0;  // 0 none, 1 sep * invH, 2 biasRate * sep, 3 clamped at -maxPushout
    if (sep > T(0)) {
        bias = sep * M.invH;
        biasKind = 1;
    } else if (useBias) {
        const T b1 = soft.biasRate * sep;
        biasKind = b1 > -M.maxPushout ? 2 : 3;
        bias = fmax(b1, -M.maxPushout);
        ms = soft.massScale;
        is = soft.impulseScale;
    }
    const T imp = -x.mass * ms * (vn + bias) - is * p0.n;
    const T total = fmax(p0.n + imp, T(0));
    const T delta = total - p0.n;
    // Reverse: push, max, total, impulse.
    T deltaG = pushAdj(a, b, x, delta, ga, gb);
    if (delta > p0.maxN) {
        deltaG += gp.maxN;
        gp.maxN = 0;
    }
    T totalG = gp.n + deltaG;
    T nG = -deltaG;
    T impG = 0;
    if (p0.n + imp > T(0)) {
        nG += totalG;
        impG = totalG;
    }
    const T massG = -impG * ms * (vn + bias);
    const T vnG = -impG * x.mass * ms;
    const T biasG = vnG;
    nG += -impG * is;
    gp.n = nG;
    speedAdj(x, vnG, ga, gb);
    axisMassAdj(x, massG, ga.im, ga.I, gb.im, gb.I);
    T sepG = 0;
    if (biasKind == 1) { sepG = biasG * M.invH; }
    if (biasKind == 2) { sepG = biasG * soft.biasRate; }
    if (sepG != T(0)) {
        const V3<T> dg = c.n * sepG;
        gb.dp = gb.dp + dg;
        ga.dp = ga.dp - dg;
        rotateAdj(b.dq, q.rb, dg, gb.dq);
        rotateAdj(a.dq, q.ra, dg * T(-1), ga.dq);
    }
}

// The friction rows of point i (src/solver.cpp:393-418).
template <class T>
__device__ __forceinline__ void frictionRow(SBody<T>& a, SBody<T>& b, const CData<T>& c, int i, PointState<T>& p, T mu,
                                            uint32_t* br = nullptr, T* rowOut = nullptr) {
    const Axis<T> x1 = makeAxis(a, b, c.ra[i], c.rb[i], c.t1);
    const Axis<T> x2 = makeAxis(a, b, c.ra[i], c.rb[i], c.t2);
    const T old1 = dot(p.t, c.t1), old2 = dot(p.t, c.t2);
    const T s1 = speedAlong(a, b, x1), s2 = speedAlong(a, b, x2);
    if (rowOut) { rowOut[0] = s1, rowOut[1] = s2, rowOut[2] = p.n; }
    T f1 = old1 - x1.mass * s1;
    T f2 = old2 - x2.mass * s2;
    const T limit = mu * p.n;
    const T mag = sqrtT(f1 * f1 + f2 * f2);
    if (br) { *br = (x1.on ? 1u : 0u) | (x2.on ? 2u : 0u) | (mag > limit ? 4u : 0u) | (mag > T(0) ? 8u : 0u) | 32u; }
    if (mag > limit) {
        const T scale = mag > T(0) ? limit / mag : T(0);
        f1 *= scale;
        f2 *= scale;
    }
    p.t = c.t1 * f1 + c.t2 * f2;
    push(a, b, x1, f1 - old1);
    push(a, b, x2, f2 - old2);
}

// The reverse of the friction rows of point i: t0 is the point's tangent impulse before them, row[0..2] their
// logged speeds along the two tangents and the normal impulse that bounds them.
template <class T>
__device__ __forceinline__ void frictionRowAdj(const SBody<T>& a, const SBody<T>& b, const CData<T>& c,
                                               const CPoint<T>& q, V3<T> t0, const T* row, T mu, BodyAdj<T>& ga, BodyAdj<T>& gb,
                                               PointState<T>& gp, T& muG) {
    const Axis<T> x1 = makeAxis(a, b, q.ra, q.rb, c.t1);
    const Axis<T> x2 = makeAxis(a, b, q.ra, q.rb, c.t2);
    const T old1 = dot(t0, c.t1), old2 = dot(t0, c.t2);
    const T s1 = row[0], s2 = row[1], pn = row[2];
    const T f1 = old1 - x1.mass * s1, f2 = old2 - x2.mass * s2;
    const T limit = mu * pn;
    const T mag = sqrtT(f1 * f1 + f2 * f2);
    // With no friction allowed (limit 0) the row adds nothing whatever f is, also at f = 0 where the forward
    // takes the unclamped branch with the same result: the derivative is that of the clamp.
    const bool clamp = mag > limit || limit == T(0);
    const T scale = mag > limit ? (mag > T(0) ? limit / mag : T(0)) : (limit == T(0) ? T(0) : T(1));
    const T g1 = f1 * scale, g2 = f2 * scale;
    // Reverse the pushes (they commute), the stored tangent impulse, the cone, the rows.
    const T d1G = pushAdj(a, b, x1, g1 - old1, ga, gb);
    const T d2G = pushAdj(a, b, x2, g2 - old2, ga, gb);
    T g1G = d1G + dot(gp.t, c.t1);
    T g2G = d2G + dot(gp.t, c.t2);
    T old1G = -d1G, old2G = -d2G;
    T f1G = g1G, f2G = g2G;
    if (clamp && mag > T(0)) {
        const T scaleG = g1G * f1 + g2G * f2;
        f1G = g1G * scale;
        f2G = g2G * scale;
        const T limitG = scaleG / mag;
        const T magG = -scaleG * limit / (mag * mag);
        f1G += magG * f1 / mag;
        f2G += magG * f2 / mag;
        muG += limitG * pn;
        gp.n += limitG * mu;
    } else if (clamp) {
        f1G = 0;
        f2G = 0;
    }
    old1G += f1G;
    old2G += f2G;
    axisMassAdj(x1, -f1G * s1, ga.im, ga.I, gb.im, gb.I);
    axisMassAdj(x2, -f2G * s2, ga.im, ga.I, gb.im, gb.I);
    speedAdj(x1, -f1G * x1.mass, ga, gb);
    speedAdj(x2, -f2G * x2.mass, ga, gb);
    gp.t = c.t1 * old1G + c.t2 * old2G;
}

// The restitution row of point i (src/solver.cpp:423-460); does nothing when the point does not qualify.
template <class T>
__device__ __forceinline__ bool restitutes(const Model<T>& M, const CData<T>& c, int i, const PointState<T>& p) {
    return !(c.relVel[i] > -M.restThreshold || p.maxN == T(0));
}

template <class T>
__device__ __forceinline__ void restituteRow(const Model<T>& M, SBody<T>& a, SBody<T>& b, const CData<T>& c, int i,
                                             PointState<T>& p, uint32_t* br = nullptr, T* speedOut = nullptr) {
    const Axis<T> x = makeAxis(a, b, c.ra[i], c.rb[i], c.n);
    const T vn = speedAlong(a, b, x);
    if (speedOut) { *speedOut = vn; }
    const T imp = -x.mass * (vn + c.restitution * c.relVel[i]);
    const T total = fmax(p.n + imp, T(0));
    const T delta = total - p.n;
    if (br) { *br = (x.on ? 1u : 0u) | (p.n + imp > T(0) ? 2u : 0u) | 64u; }
    p.n = total;
    p.maxN = fmax(p.maxN, delta);
    push(a, b, x, delta);
}

template <class T>
__device__ __forceinline__ void restituteRowAdj(const Model<T>& M, const SBody<T>& a, const SBody<T>& b, const CData<T>& c,
                                                const CPoint<T>& q, const PointState<T>& p0, T vn, BodyAdj<T>& ga, BodyAdj<T>& gb,
                                                PointState<T>& gp) {
    const Axis<T> x = makeAxis(a, b, q.ra, q.rb, c.n);
    const T imp = -x.mass * (vn + c.restitution * q.relVel);
    const T total = fmax(p0.n + imp, T(0));
    const T delta = total - p0.n;
    T deltaG = pushAdj(a, b, x, delta, ga, gb);
    if (delta > p0.maxN) {
        deltaG += gp.maxN;
        gp.maxN = 0;
    }
    const T totalG = gp.n + deltaG;
    T nG = -deltaG;
    T impG = 0;
    if (p0.n + imp > T(0)) {
        nG += totalG;
        impG = totalG;
    }
    gp.n = nG;
    const T massG = -impG * (vn + c.restitution * q.relVel);
    speedAdj(x, -impG * x.mass, ga, gb);
    axisMassAdj(x, massG, ga.im, ga.I, gb.im, gb.I);
}

// One operation on one contact, forward. The points' state comes in and goes out through p.
// A 64-bit mix of one row's place in the run and its branches (the finaliser of splitmix64).
__device__ __forceinline__ unsigned long long branchHash(unsigned long long tag, uint32_t row, uint32_t bits) {
    unsigned long long z = tag * 0x9E3779B97F4A7C15ull + ((unsigned long long)row << 8 | bits);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// rec, when not null, is the operation's record (kCallWords values; the caller has written the points' state
// to it): the rows add their speeds.
template <class T>
__device__ void contactOp(const Model<T>& M, int op, SBody<T>& a, SBody<T>& b, const CData<T>& c, PointState<T>* p,
                          T mu, T* rec = nullptr, unsigned long long* sig = nullptr, unsigned long long tag = 0) {
    const Softness<T> soft = (!a.moves || !b.moves) ? M.staticSoft : M.contactSoft;
    const int n = c.count;
    uint32_t bits = 0;
    uint32_t* br = sig ? &bits : nullptr;
    if (op == kWarm) {
        for (int i = 0; i < n; ++i) {
            const Axis<T> xn = makeAxis(a, b, c.ra[i], c.rb[i], c.n);
            const Axis<T> x1 = makeAxis(a, b, c.ra[i], c.rb[i], c.t1);
            const Axis<T> x2 = makeAxis(a, b, c.ra[i], c.rb[i], c.t2);
            push(a, b, xn, p[i].n);
            push(a, b, x1, dot(p[i].t, c.t1));
            push(a, b, x2, dot(p[i].t, c.t2));
        }
        return;
    }
    if (op == kRestitute) {
        if (c.restitution == T(0)) { return; }
        for (int i = 0; i < n; ++i) {
            bits = 128u;
            if (restitutes(M, c, i, p[i])) { restituteRow(M, a, b, c, i, p[i], br, rec ? rec + kSpeedAt + i : nullptr); }
            if (sig) { *sig += branchHash(tag, (uint32_t)i, bits); }
        }
        return;
    }
    const bool useBias = op == kBias;
    for (int i = 0; i < n; ++i) {
        normalRow(M, a, b, c, i, p[i], useBias, soft, br, rec ? rec + kSpeedAt + i : nullptr);
        if (sig) { *sig += branchHash(tag, (uint32_t)i, bits); }
    }
    // Friction forward in the biased pass and backward in the relax pass; row n + j is the j-th friction row.
    for (int j = 0; j < n; ++j) {
        const int i = useBias ? j : n - 1 - j;
        frictionRow(a, b, c, i, p[i], mu, br, rec ? rec + kFrictionAt + 3 * j : nullptr);
        if (sig) { *sig += branchHash(tag, (uint32_t)(n + j), bits); }
    }
}

// The same operation in reverse, from its record: each row's input that the reverse needs is the points' state
// before the operation (a point's rows of one kind run once, so each row starts from it, the friction rows with
// the normal impulse logged beside them) and the logged speeds. ga, gb, gp hold the adjoints after the operation
// on entry and before it on return. Velocities of a and b are not read.
template <class T>
__device__ __forceinline__ void contactOpAdj(const Model<T>& M, int op, const SBody<T>& a, const SBody<T>& b,
                                             const CData<T>& c, T mu, BodyAdj<T>& ga, BodyAdj<T>& gb,
                                             PointState<T> (&gp)[4], T& muG, const T* rec) {
    // Point i's state before the operation, read from the record where it is needed.
    auto p0 = [&](int i) { return PointState<T>{ rec[5 * i], ld3(rec + 5 * i + 1), rec[5 * i + 4] }; };
    const Softness<T> soft = (!a.moves || !b.moves) ? M.staticSoft : M.contactSoft;
    const int n = c.count;
    if (op == kWarm) {
        for (int i = 0; i < n; ++i) {
            const CPoint<T> q = pointOf(c, i);
            const PointState<T> pi = p0(i);
            PointState<T> g = pick4(gp, i);
            const Axis<T> xn = makeAxis(a, b, q.ra, q.rb, c.n);
            const Axis<T> x1 = makeAxis(a, b, q.ra, q.rb, c.t1);
            const Axis<T> x2 = makeAxis(a, b, q.ra, q.rb, c.t2);
            const T l1 = dot(pi.t, c.t1), l2 = dot(pi.t, c.t2);
            g.n += pushAdj(a, b, xn, pi.n, ga, gb);
            const T g1 = pushAdj(a, b, x1, l1, ga, gb);
            const T g2 = pushAdj(a, b, x2, l2, ga, gb);
            g.t = g.t + c.t1 * g1 + c.t2 * g2;
            put4(gp, i, g);
        }
        return;
    }
    if (op == kRestitute) {
        if (c.restitution == T(0)) { return; }
        for (int i = n - 1; i >= 0; --i) {
            const CPoint<T> q = pointOf(c, i);
            const PointState<T> pi = p0(i);
            if (q.relVel > -M.restThreshold || pi.maxN == T(0)) { continue; }  // restitutes() false
            PointState<T> g = pick4(gp, i);
            restituteRowAdj(M, a, b, c, q, pi, rec[kSpeedAt + i], ga, gb, g);
            put4(gp, i, g);
        }
        return;
    }
    const bool useBias = op == kBias;
    for (int j = n - 1; j >= 0; --j) {
        const int i = useBias ? j : n - 1 - j;
        PointState<T> g = pick4(gp, i);
        frictionRowAdj(a, b, c, pointOf(c, i), ld3(rec + 5 * i + 1), rec + kFrictionAt + 3 * j, mu, ga, gb, g, muG);
        put4(gp, i, g);
    }
    for (int i = n - 1; i >= 0; --i) {
        PointState<T> g = pick4(gp, i);
        normalRowAdj(M, a, b, c, pointOf(c, i), p0(i), rec[kSpeedAt + i], useBias, soft, ga, gb, g);
        put4(gp, i, g);
    }
}

// Asks for the 128-byte lines of [from, to) in L1, spread over the warp's lanes.
template <class T>
__device__ __forceinline__ void prefetchRange(const T* from, const T* to, uint32_t lane) {
    const char* end = reinterpret_cast<const char*>(to);
    for (const char* p = reinterpret_cast<const char*>(from) + 128 * lane; p < end; p += 128 * 32) {
        asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
    }
}

// Records a stage buffer of the reverse walk holds: one color's batch (each warp has two buffers, one being
// filled while the other is read). In float, two buffers and the body arrays of a 65-body world take 27 KB, so
// that two CTAs of four warps share an SM.
template <class T>
__host__ __device__ constexpr int stageCalls() { return sizeof(T) == 4 ? 48 : 32; }

// Copies `words` values (whole 16-byte pieces, both addresses 16-byte aligned) from global to shared memory
// with asynchronous copies spread over the warp's lanes, as one commit group of each lane.
template <class T>
__device__ __forceinline__ void copyToShared(T* dst, const T* src, uint32_t words, uint32_t lane) {
    const uint32_t pieces = words * (uint32_t)sizeof(T) / 16u;
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    const char* from = reinterpret_cast<const char*>(src);
    for (uint32_t k = lane; k < pieces; k += 32) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d + 16u * k), "l"(from + 16u * k) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// ---------------------------------------------------------------------------------------------------------
// One world's step, forward (with optional logging) and in reverse. One warp per world.

struct WorldView {
    uint32_t bodyFirst, bodyCount, shapeFirst;
    const TapeWorld* tw;
    const TapeContact* contacts;
    const uint32_t* colored;
    const uint32_t* impactColored;
    const uint32_t* rest;
    const uint32_t* impactRest;
    const uint8_t* awake;
};

__device__ __forceinline__ WorldView viewOf(const AdjointSetup& S, int step, uint32_t w) {
    const TapeStep ts = S.steps[step];
    WorldView v;
    v.bodyFirst = S.bodyFirst[w];
    v.bodyCount = S.bodyCount[w];
    v.shapeFirst = S.shapeFirst[w];
    v.tw = ts.worlds + w;
    const uint32_t cf = v.tw->contactFirst;
    v.contacts = ts.contacts + cf;
    v.colored = ts.colored + cf;
    v.impactColored = ts.impactColored + cf;
    v.rest = ts.rest + cf;
    v.impactRest = ts.impactRest + cf;
    v.awake = ts.awake;
    return v;
}

template <class T>
__device__ __forceinline__ bool movesIn(const Model<T>& M, const WorldView& V, uint32_t g) {
    return M.S.dynamic[g] && V.awake[g];
}

template <class T>
__device__ __forceinline__ SBody<T> bodyOf(const Model<T>& M, const Slot<T>& W, const WorldView& V, uint32_t g, const T* state) {
    SBody<T> b;
    b.v = ld3(state + (size_t)g * kState + 7);
    b.w = ld3(state + (size_t)g * kState + 10);
    b.dp = ld3(W.dp + 3 * (size_t)g);
    b.dq = ld4(W.dq + 4 * (size_t)g);
    b.im = W.invM[g];
    b.I = ldM(W.invI + 9 * (size_t)g);
    b.moves = movesIn(M, V, g);
    return b;
}

template <class T>
__device__ __forceinline__ T contactFriction(const Model<T>& M, const WorldView& V, const TapeContact& tc) {
    return sqrtT(M.friction[V.shapeFirst + tc.shapeA] * M.friction[V.shapeFirst + tc.shapeB]);
}

// The list walks of one pass, in the order the step pipeline runs them.
struct PassList {
    const uint32_t* list;
    const uint32_t* start;  // color starts, or null for a one-at-a-time list
    uint32_t count;         // colors, or list length
};

__device__ __forceinline__ int passLists(const WorldView& V, int op, PassList* out) {
    const TapeWorld& tw = *V.tw;
    int n = 0;
    out[n++] = { V.colored, tw.colorStart, tw.colorCount };
    out[n++] = { V.rest, nullptr, tw.restCount };
    if (op != kWarm && op != kRestitute && tw.impactColorStart[tw.impactColorCount] + tw.impactRestCount > 0) {
        out[n++] = { V.impactColored, tw.impactColorStart, tw.impactColorCount };
        out[n++] = { V.impactRest, nullptr, tw.impactRestCount };
    }
    return n;
}

// Forward of one step of one world. state: in at `in`, out at `out` (may be the same). When log is non-null the
// inputs of every contact operation and position update are written there for the reverse pass.
template <class T>
__device__ void stepWorld(const Model<T>& M, const Slot<T>& W, int step, uint32_t w, const T* in, T* out, T* log,
                          T* integLog, unsigned long long* sig = nullptr) {
    const uint32_t lane = threadIdx.x & 31;
    const WorldView V = viewOf(M.S, step, w);
    const int n = M.S.substeps;
    // Step start: world inverse inertia at this pose, zero displacement, warm-start impulses.
    for (uint32_t i = lane; i < V.bodyCount; i += 32) {
        const uint32_t g = V.bodyFirst + i;
        const T* s = in + (size_t)g * kState;
        T* o = out + (size_t)g * kState;
        for (int k = 0; k < kState; ++k) { o[k] = s[k]; }
        const bool moves = movesIn(M, V, g);
        const Q4<T> q = ld4(s + 3);
        T im = 0;
        M3<T> I = zeroM<T>();
        if (moves) {
            const T scale = T(M.S.mass[g]) / M.mass[g];
            im = T(1) / M.mass[g];
            const M3<T> r = toMat3(q);
            M3<T> L;
            for (int a = 0; a < 3; ++a) {
                L.r[a] = { T(M.S.invInertiaLocal[9 * g + 3 * a]) * scale, T(M.S.invInertiaLocal[9 * g + 3 * a + 1]) * scale,
                           T(M.S.invInertiaLocal[9 * g + 3 * a + 2]) * scale };
            }
            I = mmul(r, mmul(L, transposeM(r)));
        }
        W.invM[g] = im;
        stM(W.invI + 9 * (size_t)g, I);
        st3(W.dp + 3 * (size_t)g, zeroV<T>());
        st4(W.dq + 4 * (size_t)g, Q4<T>{ 0, 0, 0, 1 });
        st4(W.qBase + 4 * (size_t)g, q);
    }
    const uint32_t cf = V.tw->contactFirst;
    for (uint32_t ci = lane; ci < V.tw->contactCount; ci += 32) {
        const TapeContact& tc = V.contacts[ci];
        for (int i = 0; i < 4; ++i) {
            PointState<T>& p = W.points[(size_t)(cf + ci) * 4 + i];
            p.n = T(tc.normalImpulse[i]);
            p.t = fl3<T>(tc.tangentImpulse[i]);
            p.maxN = 0;
        }
    }
    __syncwarp();
    uint64_t cursor = 0;  // log index of the next operation; every lane keeps the same count
    auto runOp = [&](int op, uint32_t ci, uint64_t at) {
        const TapeContact& tc = V.contacts[ci];
        const CData<T> c = loadContact<T>(tc);
        const uint32_t ga = V.bodyFirst + tc.a, gb = V.bodyFirst + tc.b;
        SBody<T> a = bodyOf(M, W, V, ga, out), b = bodyOf(M, W, V, gb, out);
        PointState<T>* p = W.points + (size_t)(cf + ci) * 4;
        PointState<T> ps[4];
        for (int i = 0; i < 4; ++i) { ps[i] = p[i]; }
        T* rec = log ? log + at * kCallWords : nullptr;
        if (rec) { writeCall(rec, ps); }
        contactOp(M, op, a, b, c, ps, contactFriction(M, V, tc), rec, sig,
                  (unsigned long long)step << 40 ^ at << 2 ^ (unsigned long long)op);
        for (int i = 0; i < 4; ++i) { p[i] = ps[i]; }
        if (a.moves) {
            st3(out + (size_t)ga * kState + 7, a.v);
            st3(out + (size_t)ga * kState + 10, a.w);
        }
        if (b.moves) {
            st3(out + (size_t)gb * kState + 7, b.v);
            st3(out + (size_t)gb * kState + 10, b.w);
        }
    };
    // One pass: colored lists color by color (a lane per contact), one-at-a-time lists on lane 0.
    auto pass = [&](int op) {
        PassList lists[4];
        const int nl = passLists(V, op, lists);
        for (int l = 0; l < nl; ++l) {
            const PassList& L = lists[l];
            if (L.start) {
                const uint32_t first = L.start[0];
                for (uint32_t k = 0; k < L.count; ++k) {
                    for (uint32_t x = L.start[k] + lane; x < L.start[k + 1]; x += 32) { runOp(op, L.list[x], cursor + (x - first)); }
                    __syncwarp();
                }
                cursor += L.start[L.count] - first;
            } else {
                if (lane == 0) {
                    for (uint32_t x = 0; x < L.count; ++x) { runOp(op, L.list[x], cursor + x); }
                }
                cursor += L.count;
                __syncwarp();
            }
        }
    };
    for (int sub = 0; sub < n; ++sub) {
        for (uint32_t i = lane; i < V.bodyCount; i += 32) {
            const uint32_t g = V.bodyFirst + i;
            if (!movesIn(M, V, g)) { continue; }
            T* o = out + (size_t)g * kState;
            const V3<T> v = ld3(o + 7), wv = ld3(o + 10);
            const T gs = T(M.S.gravityScale[g]);
            const V3<T> nv = (v + M.gravity * (gs * M.h)) * (T(1) / (T(1) + M.h * T(M.S.linearDamping[g])));
            const V3<T> nw = wv * (T(1) / (T(1) + M.h * T(M.S.angularDamping[g])));
            st3(o + 7, nv);
            st3(o + 10, nw);
        }
        __syncwarp();
        pass(kWarm);
        pass(kBias);
        for (uint32_t i = lane; i < V.bodyCount; i += 32) {
            const uint32_t g = V.bodyFirst + i;
            if (!movesIn(M, V, g)) { continue; }
            T* o = out + (size_t)g * kState;
            const V3<T> v = ld3(o + 7), wv = ld3(o + 10);
            const Q4<T> q = ld4(o + 3);
            st3(o, ld3(o) + v * M.h);
            const V3<T> ndp = ld3(W.dp + 3 * (size_t)g) + v * M.h;
            st3(W.dp + 3 * (size_t)g, ndp);
            if (integLog) {
                T* L = integLog + ((size_t)sub * M.S.totalBodies + g) * kIntegWords;
                st4(L, q);
                st3(L + 4, wv);
                st3(L + 7, ndp);
            }
            const Q4<T> nq = integrateQ(q, wv, M.h);
            st4(o + 3, nq);
            st4(W.dq + 4 * (size_t)g, qmul(nq, conj(ld4(W.qBase + 4 * (size_t)g))));
        }
        __syncwarp();
        pass(kRelax);
    }
    pass(kRestitute);
}

// The per-body arrays the reverse walk reads and writes, indexed by the body's place in its world. They are
// the warp's share of shared memory when the kernel has one for bodies (the adjoint state is copied in at the
// start of the walk and out at its end, the step's inverse masses and inertias at each step's start), else the
// global arrays offset to the world's first body.
template <class T>
struct BodyArrays {
    T* stateAdj;  // kState per body
    T* dpAdj;     // 3
    T* dqAdj;     // 4
    T* qBaseAdj;  // 4
    T* invMAdj;   // 1
    T* invIAdj;   // 9
    T* dp;        // 3: the body's displacement during the pass being reversed
    T* dq;        // 4
    T* invM;      // 1: the step's inverse mass and world inverse inertia
    T* invI;      // 9
};
constexpr int kBodyWords = kState + 3 + 4 + 4 + 1 + 9 + 3 + 4 + 1 + 9;

template <class T>
__device__ __forceinline__ BodyArrays<T> sharedBodies(T* area, uint32_t cap) {
    BodyArrays<T> B;
    T* p = area;
    B.stateAdj = p, p += kState * cap;
    B.dpAdj = p, p += 3 * cap;
    B.dqAdj = p, p += 4 * cap;
    B.qBaseAdj = p, p += 4 * cap;
    B.invMAdj = p, p += cap;
    B.invIAdj = p, p += 9 * cap;
    B.dp = p, p += 3 * cap;
    B.dq = p, p += 4 * cap;
    B.invM = p, p += cap;
    B.invI = p;
    return B;
}

template <class T>
__device__ __forceinline__ BodyArrays<T> globalBodies(const Model<T>& M, const Slot<T>& W, size_t first) {
    return { M.stateAdj + kState * first, M.dpAdj + 3 * first, M.dqAdj + 4 * first, M.qBaseAdj + 4 * first,
             M.invMAdj + first, M.invIAdj + 9 * first, W.dp + 3 * first, W.dq + 4 * first, W.invM + first,
             W.invI + 9 * first };
}

// Reverse of one world's step: adjoints of the state at the step's end in M.stateAdj become those at its start.
// Needs the log and integLog that stepWorld wrote for this step, and the bodies' dp/dq of every substep, which
// it recomputes by replaying the integration from the checkpoint as it goes back. stage: the warp's two
// shared-memory buffers of stageCalls<T>() records each, or null to read every record from the log. bodies:
// the warp's shared-memory body arrays (sharedBodies) holding the world's adjoint state, or null to use the
// global arrays.
template <class T>
__device__ void stepWorldAdj(const Model<T>& M, const Slot<T>& W, int step, uint32_t w, const T* in, const T* log,
                             const T* integLog, uint64_t calls, T* stage, T* bodies, uint32_t bodyCap) {
    constexpr int kStage = stageCalls<T>();
    const uint32_t lane = threadIdx.x & 31;
    const WorldView V = viewOf(M.S, step, w);
    const int n = M.S.substeps;
    const uint32_t cf = V.tw->contactFirst;
    const BodyArrays<T> B = bodies ? sharedBodies(bodies, bodyCap) : globalBodies(M, W, V.bodyFirst);
    // The step's adjoint accumulators start at zero; the inverse masses and inertias the recomputation found.
    for (uint32_t i = lane; i < V.bodyCount; i += 32) {
        st3(B.dpAdj + 3 * i, zeroV<T>());
        st4(B.dqAdj + 4 * i, Q4<T>{ 0, 0, 0, 0 });
        st4(B.qBaseAdj + 4 * i, Q4<T>{ 0, 0, 0, 0 });
        B.invMAdj[i] = 0;
        stM(B.invIAdj + 9 * i, zeroM<T>());
        if (bodies) {
            const uint32_t g = V.bodyFirst + i;
            B.invM[i] = W.invM[g];
            for (int k = 0; k < 9; ++k) { B.invI[9 * i + k] = W.invI[9 * (size_t)g + k]; }
        }
    }
    for (uint32_t ci = lane; ci < V.tw->contactCount; ci += 32) {
        for (int i = 0; i < 4; ++i) { M.pointAdj[(size_t)(cf + ci) * 4 + i] = PointState<T>{ 0, zeroV<T>(), 0 }; }
    }
    __syncwarp();
    // dp and dq a body had during substep `sub`'s passes: before its position update (warm start, biased
    // solve) or after it (relax, restitution), from the integration log of the recomputed step.
    auto setDisplacement = [&](int sub, bool afterUpdate) {
        for (uint32_t i = lane; i < V.bodyCount; i += 32) {
            const uint32_t g = V.bodyFirst + i;
            const int k = afterUpdate ? sub : sub - 1;  // the last position update before the pass
            if (!movesIn(M, V, g) || k < 0) {
                st3(B.dp + 3 * i, zeroV<T>());
                st4(B.dq + 4 * i, Q4<T>{ 0, 0, 0, 1 });
                continue;
            }
            const T* L = integLog + ((size_t)k * M.S.totalBodies + g) * kIntegWords;
            const Q4<T> qb = ld4(in + (size_t)g * kState + 3);
            st3(B.dp + 3 * i, ld3(L + 7));
            st4(B.dq + 4 * i, qmul(integrateQ(ld4(L), ld3(L + 4), M.h), conj(qb)));
        }
        __syncwarp();
    };
    uint64_t cursor = calls;  // one past the last call of the step
    auto opAdj = [&](int op, uint32_t ci, const T* rec) {
        const TapeContact& tc = V.contacts[ci];
        const CData<T> c = loadContact<T>(tc);
        const uint32_t ia = tc.a, ib = tc.b, ga = V.bodyFirst + ia, gb = V.bodyFirst + ib;
        SBody<T> a, b;
        a.v = a.w = b.v = b.w = zeroV<T>();  // the reverse reads no velocity
        a.dp = ld3(B.dp + 3 * ia), a.dq = ld4(B.dq + 4 * ia), a.im = B.invM[ia];
        a.I = ldM(B.invI + 9 * ia), a.moves = movesIn(M, V, ga);
        b.dp = ld3(B.dp + 3 * ib), b.dq = ld4(B.dq + 4 * ib), b.im = B.invM[ib];
        b.I = ldM(B.invI + 9 * ib), b.moves = movesIn(M, V, gb);
        T* sa = B.stateAdj + ia * kState;
        T* sb = B.stateAdj + ib * kState;
        BodyAdj<T> gA{ zeroV<T>(), zeroV<T>(), zeroV<T>(), Q4<T>{ 0, 0, 0, 0 }, 0, zeroM<T>() };
        BodyAdj<T> gB = gA;
        // Moving bodies belong to this contact alone within its color: their adjoints are read and written in
        // place. Anchored bodies are shared: their contributions are added atomically.
        if (a.moves) { gA.v = ld3(sa + 7), gA.w = ld3(sa + 10); }
        if (b.moves) { gB.v = ld3(sb + 7), gB.w = ld3(sb + 10); }
        PointState<T>* gp = M.pointAdj + (size_t)(cf + ci) * 4;
        PointState<T> g4[4];
        for (int i = 0; i < 4; ++i) { g4[i] = gp[i]; }
        T muG = 0;
        const T mu = contactFriction(M, V, tc);
        contactOpAdj(M, op, a, b, c, mu, gA, gB, g4, muG, rec);
        for (int i = 0; i < 4; ++i) { gp[i] = g4[i]; }
        auto put = [&](bool moves, uint32_t i, uint32_t g, T* s, const BodyAdj<T>& G) {
            if (moves) {
                st3(s + 7, G.v);
                st3(s + 10, G.w);
                st3(B.dpAdj + 3 * i, ld3(B.dpAdj + 3 * i) + G.dp);
                st4(B.dqAdj + 4 * i, qadd(ld4(B.dqAdj + 4 * i), G.dq));
                B.invMAdj[i] += G.im;
                T* I = B.invIAdj + 9 * i;
                for (int r = 0; r < 3; ++r) { I[3 * r] += G.I.r[r].x, I[3 * r + 1] += G.I.r[r].y, I[3 * r + 2] += G.I.r[r].z; }
            } else if (M.S.dynamic[g]) {
                // A sleeping dynamic body: its velocity carries back to steps where it moved. A static body's
                // never changes, so nothing is added for it.
                atomicAddT(s + 7, G.v.x), atomicAddT(s + 8, G.v.y), atomicAddT(s + 9, G.v.z);
                atomicAddT(s + 10, G.w.x), atomicAddT(s + 11, G.w.y), atomicAddT(s + 12, G.w.z);
            }
        };
        put(a.moves, ia, ga, sa, gA);
        put(b.moves, ib, gb, sb, gB);
        if (muG != T(0)) {
            // mu = sqrt(fa fb): d mu / d fa = fb / (2 mu).
            const T fa = M.friction[V.shapeFirst + tc.shapeA], fb = M.friction[V.shapeFirst + tc.shapeB];
            if (mu > T(0)) {
                atomicAddT(M.frictionAdj + V.shapeFirst + tc.shapeA, muG * fb / (T(2) * mu));
                atomicAddT(M.frictionAdj + V.shapeFirst + tc.shapeB, muG * fa / (T(2) * mu));
            }
        }
    };
    auto passAdj = [&](int op) {
        PassList lists[4];
        const int nl = passLists(V, op, lists);
        for (int l = nl - 1; l >= 0; --l) {
            const PassList& L = lists[l];
            if (L.start) {
                const uint32_t first = L.start[0];
                cursor -= L.start[L.count] - first;
                // Color k's records, consecutive in the log. A color that fits a stage buffer is copied to shared
                // memory while the color before it in the walk runs; a larger one is read where it lies.
                auto records = [&](int k) { return log + (cursor + (L.start[k] - first)) * kCallWords; };
                auto staged = [&](int k) { return stage != nullptr && L.start[k + 1] - L.start[k] <= (uint32_t)kStage; };
                auto fetch = [&](int k, int buffer) {
                    if (staged(k)) {
                        copyToShared(stage + buffer * kStage * kCallWords, records(k), (L.start[k + 1] - L.start[k]) * kCallWords, lane);
                    } else {
                        prefetchRange(records(k), records(k + 1), lane);
                    }
                    // Its contacts are read one per lane: ask for their lines too.
                    for (uint32_t x = L.start[k] + lane; x < L.start[k + 1]; x += 32) {
                        const char* tc = reinterpret_cast<const char*>(V.contacts + L.list[x]);
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(tc));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(tc + sizeof(TapeContact) - 1));
                    }
                };
                if (L.count > 0) { fetch((int)L.count - 1, 0); }
                for (int k = (int)L.count - 1; k >= 0; --k) {
                    const int buffer = ((int)L.count - 1 - k) & 1;
                    asm volatile("cp.async.wait_all;" ::: "memory");
                    __syncwarp();
                    if (k > 0) { fetch(k - 1, buffer ^ 1); }
                    const T* base = staged(k) ? stage + buffer * kStage * kCallWords : records(k);
                    for (uint32_t x = L.start[k] + lane; x < L.start[k + 1]; x += 32) {
                        opAdj(op, L.list[x], base + (x - L.start[k]) * kCallWords);
                    }
                    __syncwarp();
                }
            } else {
                cursor -= L.count;
                if (lane == 0) {
                    for (int x = (int)L.count - 1; x >= 0; --x) { opAdj(op, L.list[x], log + (cursor + (uint64_t)x) * kCallWords); }
                }
                __syncwarp();
            }
        }
    };
    setDisplacement(n - 1, true);
    passAdj(kRestitute);
    for (int sub = n - 1; sub >= 0; --sub) {
        setDisplacement(sub, true);
        passAdj(kRelax);
        // Position update in reverse.
        for (uint32_t i = lane; i < V.bodyCount; i += 32) {
            const uint32_t g = V.bodyFirst + i;
            if (!movesIn(M, V, g)) { continue; }
            T* s = B.stateAdj + i * kState;
            const T* L = integLog + ((size_t)sub * M.S.totalBodies + g) * kIntegWords;
            const Q4<T> q = ld4(L);
            const V3<T> wv = ld3(L + 4);
            const Q4<T> nq = integrateQ(q, wv, M.h);
            const Q4<T> qb = ld4(in + (size_t)g * kState + 3);
            // dq' = q' qBase*: its adjoint goes to q' and to qBase.
            const Q4<T> dqG = ld4(B.dqAdj + 4 * i);
            Q4<T> qG = qadd(ld4(s + 3), qmulAdjA(dqG, conj(qb)));
            const Q4<T> cG = qmulAdjB(dqG, nq);
            st4(B.qBaseAdj + 4 * i, qadd(ld4(B.qBaseAdj + 4 * i), Q4<T>{ -cG.x, -cG.y, -cG.z, cG.w }));
            st4(B.dqAdj + 4 * i, Q4<T>{ 0, 0, 0, 0 });
            Q4<T> qPrevG{ 0, 0, 0, 0 };
            V3<T> wG = ld3(s + 10);
            integrateQAdj(q, wv, M.h, qG, qPrevG, wG);
            st4(s + 3, qPrevG);
            st3(s + 10, wG);
            // com' = com + v h and dp' = dp + v h.
            const V3<T> vG = ld3(s + 7) + ld3(s) * M.h + ld3(B.dpAdj + 3 * i) * M.h;
            st3(s + 7, vG);
        }
        __syncwarp();
        setDisplacement(sub, false);
        passAdj(kBias);
        passAdj(kWarm);
        // Velocity update in reverse.
        for (uint32_t i = lane; i < V.bodyCount; i += 32) {
            const uint32_t g = V.bodyFirst + i;
            if (!movesIn(M, V, g)) { continue; }
            T* s = B.stateAdj + i * kState;
            st3(s + 7, ld3(s + 7) * (T(1) / (T(1) + M.h * T(M.S.linearDamping[g]))));
            st3(s + 10, ld3(s + 10) * (T(1) / (T(1) + M.h * T(M.S.angularDamping[g]))));
        }
        __syncwarp();
    }
    // Step start in reverse: qBase = q, the world inverse inertia r L r^T and the inverse mass 1/m.
    for (uint32_t i = lane; i < V.bodyCount; i += 32) {
        const uint32_t g = V.bodyFirst + i;
        T* s = B.stateAdj + i * kState;
        st4(s + 3, qadd(ld4(s + 3), ld4(B.qBaseAdj + 4 * i)));
        if (!movesIn(M, V, g)) { continue; }
        const Q4<T> q = ld4(in + (size_t)g * kState + 3);
        const T m = M.mass[g];
        const T scale = T(M.S.mass[g]) / m;
        M3<T> L;
        for (int a = 0; a < 3; ++a) {
            L.r[a] = { T(M.S.invInertiaLocal[9 * g + 3 * a]) * scale, T(M.S.invInertiaLocal[9 * g + 3 * a + 1]) * scale,
                       T(M.S.invInertiaLocal[9 * g + 3 * a + 2]) * scale };
        }
        const M3<T> r = toMat3(q);
        const M3<T> G = ldM(B.invIAdj + 9 * i);
        // I = r L r^T: dr = G r L^T + G^T r L, dL = r^T G r.
        const M3<T> rG = madd(mmul(G, mmul(r, transposeM(L))), mmul(transposeM(G), mmul(r, L)));
        const M3<T> LG = mmul(transposeM(r), mmul(G, r));
        T lG = 0;  // sum of dL_ij L_ij, for the mass
        for (int a = 0; a < 3; ++a) { lG += dot(LG.r[a], L.r[a]); }
        st4(s + 3, qadd(ld4(s + 3), toMat3Adj(q, rG)));
        // im = 1/m and L = L0 m0 / m: both scale as 1/m.
        M.massAdj[g] += -(B.invMAdj[i] / (m * m)) - lG / m;
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------------------------------------
// Kernels: one warp per world, every step of the run.

template <class T>
__global__ void __launch_bounds__(128) k_model_forward(const __grid_constant__ Model<T> M) {
    const uint32_t w = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    if (w >= (uint32_t)M.S.nWorlds) { return; }
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t b0 = M.S.bodyFirst[w], nb = M.S.bodyCount[w];
    for (uint32_t i = lane; i < nb; i += 32) {
        const uint32_t g = b0 + i;
        for (int k = 0; k < kState; ++k) { M.states[(size_t)g * kState + k] = M.init[(size_t)g * kState + k]; }
    }
    __syncwarp();
    const size_t stride = (size_t)M.S.totalBodies * kState;
    const Slot<T> W = slotOf(M, 0);
    unsigned long long sig = 0;
    for (int s = 0; s < M.S.nSteps; ++s) {
        stepWorld<T>(M, W, s, w, M.states + s * stride, M.states + (s + 1) * stride, nullptr, nullptr,
                     M.branches ? &sig : nullptr);
        __syncwarp();
    }
    if (M.branches) {
        for (int o = 16; o > 0; o >>= 1) { sig += __shfl_xor_sync(0xffffffffu, sig, o); }
        if (lane == 0) { M.branches[w] = sig; }
    }
}

// The backward runs chunk by chunk from the last step. Recomputing a step needs only its checkpoint, so a
// chunk's steps are recomputed all at once, one warp per world and step, each logging into its own slot; then
// one warp per world walks the chunk's steps in reverse from those logs, carrying the adjoints back.
template <class T>
__global__ void __launch_bounds__(128) k_model_recompute(const __grid_constant__ Model<T> M, int first, int count,
                                                         uint32_t slotBase) {
    const uint32_t warp = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const uint32_t nw = (uint32_t)M.S.nWorlds;
    const uint32_t k = warp / nw, w = warp % nw;
    if (k >= (uint32_t)count) { return; }
    const Slot<T> W = slotOf(M, slotBase + k);
    const int s = first + (int)k;
    const size_t stride = (size_t)M.S.totalBodies * kState;
    stepWorld(M, W, s, w, M.states + s * stride, W.scratch, W.log + (size_t)w * M.logStride, W.integLog);
}

template <class T>
__host__ __device__ constexpr size_t stageBytesPerWarp() { return 2 * (size_t)stageCalls<T>() * kCallWords * sizeof(T); }

template <class T>
__host__ __device__ constexpr size_t bodyBytesPerWarp(uint32_t cap) {
    return ((size_t)cap * kBodyWords * sizeof(T) + 15) / 16 * 16;
}

// The reverse walk of a chunk of steps, one warp per world, from the chunk's last step to its first. Each warp's
// share of the dynamic shared memory holds, when `staged`, its two stage buffers and, when bodyCap is not zero,
// body arrays for up to bodyCap bodies (no world has more).
template <class T>
__global__ void __launch_bounds__(128) k_model_reverse(const __grid_constant__ Model<T> M, int first, int count,
                                                       uint32_t slotBase, int staged, uint32_t bodyCap) {
    extern __shared__ __align__(16) unsigned char area[];
    const uint32_t w = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    if (w >= (uint32_t)M.S.nWorlds) { return; }
    const uint32_t lane = threadIdx.x & 31;
    const size_t stageBytes = staged ? stageBytesPerWarp<T>() : 0;
    unsigned char* mine = area + (threadIdx.x / 32) * (stageBytes + bodyBytesPerWarp<T>(bodyCap));
    T* stage = staged ? reinterpret_cast<T*>(mine) : nullptr;
    T* bodies = bodyCap ? reinterpret_cast<T*>(mine + stageBytes) : nullptr;
    const uint32_t b0 = M.S.bodyFirst[w], nb = M.S.bodyCount[w];
    if (bodies) {
        T* adj = sharedBodies(bodies, bodyCap).stateAdj;
        for (uint32_t k = lane; k < nb * kState; k += 32) { adj[k] = M.stateAdj[(size_t)b0 * kState + k]; }
        __syncwarp();
    }
    const size_t stride = (size_t)M.S.totalBodies * kState;
    for (int k = count - 1; k >= 0; --k) {
        const int s = first + k;
        const Slot<T> W = slotOf(M, slotBase + (uint32_t)k);
        // The number of contact operations the step logged: every pass walks its lists once.
        const WorldView V = viewOf(M.S, s, w);
        const TapeWorld& tw = *V.tw;
        const uint64_t colored = tw.colorStart[tw.colorCount] + tw.restCount;
        const uint64_t impact = tw.impactColorStart[tw.impactColorCount] + tw.impactRestCount;
        const uint64_t calls = (uint64_t)M.S.substeps * (3 * colored + 2 * impact) + colored;
        stepWorldAdj(M, W, s, w, M.states + s * stride, W.log + (size_t)w * M.logStride, W.integLog, calls, stage,
                     bodies, bodyCap);
        __syncwarp();
    }
    if (bodies) {
        const T* adj = sharedBodies(bodies, bodyCap).stateAdj;
        for (uint32_t k = lane; k < nb * kState; k += 32) { M.stateAdj[(size_t)b0 * kState + k] = adj[k]; }
    }
}

// ---------------------------------------------------------------------------------------------------------
// Host side: buffers of one differentiation run, in the precision it was started with.

struct Run {
    int precision = 0;
    size_t elem = 0;
    std::vector<void*> owned;
    void* mass = nullptr;
    void* friction = nullptr;
    void* init = nullptr;
    void* states = nullptr;
    void *invM = nullptr, *invI = nullptr, *dp = nullptr, *dq = nullptr, *qBase = nullptr, *points = nullptr;
    void *stateAdj = nullptr, *dpAdj = nullptr, *dqAdj = nullptr, *qBaseAdj = nullptr, *invMAdj = nullptr,
         *invIAdj = nullptr, *pointAdj = nullptr, *massAdj = nullptr, *frictionAdj = nullptr, *log = nullptr,
         *integLog = nullptr, *scratch = nullptr, *branches = nullptr;
    uint64_t logStride = 0;
    int slots = 0;  // steps the backward recomputes at once; two sets of slots alternate
    uint32_t maxBodies = 0;  // the most bodies of a world, read once
    bool forwardDone = false;
    float forwardMs = 0.0f, backwardMs = 0.0f;
    // The backward's two kinds of launch, each summed over its chunks (they overlap, so the sum can exceed the
    // backward's own time): recomputation and reverse walk.
    float recomputeMs = 0.0f, reverseMs = 0.0f;
    std::vector<cudaEvent_t> chunkEvents;  // per chunk: recompute start, end; reverse start, end
    // The recomputation runs on its own stream, one chunk ahead of the reverse walk. The walk, the backward's
    // critical path, runs on a stream of the highest priority, so that its CTAs take the SMs before the next
    // chunk's recomputation, which becomes ready at the same moment.
    cudaStream_t side = nullptr, walk = nullptr;
    cudaEvent_t ready = nullptr, recomputed[2] = {}, reversed[2] = {}, walked = nullptr;

    ~Run() {
        release();
        for (cudaEvent_t e : chunkEvents) { cudaEventDestroy(e); }
        for (cudaEvent_t e : { ready, recomputed[0], recomputed[1], reversed[0], reversed[1], walked }) {
            if (e) { cudaEventDestroy(e); }
        }
        if (side) { cudaStreamDestroy(side); }
        if (walk) { cudaStreamDestroy(walk); }
    }
    void release() {
        for (void* p : owned) { cudaFree(p); }
        owned.clear();
        for (void** p : { &mass, &friction, &init, &states, &invM, &invI, &dp, &dq, &qBase, &points, &stateAdj, &dpAdj,
                          &dqAdj, &qBaseAdj, &invMAdj, &invIAdj, &pointAdj, &massAdj, &frictionAdj, &log, &integLog,
                          &scratch, &branches }) {
            *p = nullptr;
        }
        forwardDone = false;
        slots = 0;
        maxBodies = 0;
    }
    int alloc(void** p, size_t bytes) {
        cudaError_t e = cudaMalloc(p, bytes < 16 ? 16 : bytes);
        if (e != cudaSuccess) { return noteError(TF_E_CUDA, std::string("adjoint: cudaMalloc: ") + cudaGetErrorString(e)); }
        owned.push_back(*p);
        return TF_OK;
    }
};

#define TF_ADJ_CUDA(call)                                                                                         \
    do {                                                                                                          \
        cudaError_t e_ = (call);                                                                                  \
        if (e_ != cudaSuccess) { return noteError(TF_E_CUDA, std::string("adjoint: " #call ": ") + cudaGetErrorString(e_)); } \
    } while (0)

template <class T>
Model<T> modelOf(const AdjointSetup& S, Run& r) {
    Model<T> M;
    M.S = S;
    M.dt = T(S.dt);
    M.h = T(S.dt) / T(S.substeps);
    M.invH = T(1) / M.h;
    M.gravity = { T(S.gravity[0]), T(S.gravity[1]), T(S.gravity[2]) };
    M.contactSoft = { T(S.contactSoft[0]), T(S.contactSoft[1]), T(S.contactSoft[2]) };
    M.staticSoft = { T(S.staticSoft[0]), T(S.staticSoft[1]), T(S.staticSoft[2]) };
    M.maxPushout = T(S.maxPushout);
    M.restThreshold = T(S.restitutionThreshold);
    M.mass = (const T*)r.mass;
    M.friction = (const T*)r.friction;
    M.init = (const T*)r.init;
    M.states = (T*)r.states;
    M.invM = (T*)r.invM;
    M.invI = (T*)r.invI;
    M.dp = (T*)r.dp;
    M.dq = (T*)r.dq;
    M.qBase = (T*)r.qBase;
    M.points = (PointState<T>*)r.points;
    M.stateAdj = (T*)r.stateAdj;
    M.dpAdj = (T*)r.dpAdj;
    M.dqAdj = (T*)r.dqAdj;
    M.qBaseAdj = (T*)r.qBaseAdj;
    M.invMAdj = (T*)r.invMAdj;
    M.invIAdj = (T*)r.invIAdj;
    M.pointAdj = (PointState<T>*)r.pointAdj;
    M.massAdj = (T*)r.massAdj;
    M.frictionAdj = (T*)r.frictionAdj;
    M.log = (T*)r.log;
    M.logStride = r.logStride;
    M.integLog = (T*)r.integLog;
    M.scratch = (T*)r.scratch;
    M.branches = (unsigned long long*)r.branches;
    return M;
}

// Host values in double to device values in T.
template <class T>
int upload(void* dst, const std::vector<double>& src, cudaStream_t stream) {
    std::vector<T> t(src.begin(), src.end());
    TF_ADJ_CUDA(cudaMemcpyAsync(dst, t.data(), t.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    TF_ADJ_CUDA(cudaStreamSynchronize(stream));
    return TF_OK;
}
template <class T>
int download(std::vector<double>& dst, const void* src, size_t n, cudaStream_t stream) {
    std::vector<T> t(n);
    TF_ADJ_CUDA(cudaMemcpyAsync(t.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, stream));
    TF_ADJ_CUDA(cudaStreamSynchronize(stream));
    dst.assign(t.begin(), t.end());
    return TF_OK;
}

template <class T>
int forwardT(Run& r, const AdjointSetup& S, cudaStream_t stream, const double* init, const double* mass,
             const double* friction, double* finalState) {
    const size_t nb = S.totalBodies, ns = S.totalShapes;
    r.release();
    r.elem = sizeof(T);
    int rc;
    const size_t stateBytes = nb * kState * sizeof(T);
    if ((rc = r.alloc(&r.mass, nb * sizeof(T))) || (rc = r.alloc(&r.friction, ns * sizeof(T))) ||
        (rc = r.alloc(&r.init, stateBytes)) || (rc = r.alloc(&r.states, stateBytes * (size_t)(S.nSteps + 2))) ||
        (rc = r.alloc(&r.invM, nb * sizeof(T))) || (rc = r.alloc(&r.invI, 9 * nb * sizeof(T))) ||
        (rc = r.alloc(&r.dp, 3 * nb * sizeof(T))) || (rc = r.alloc(&r.dq, 4 * nb * sizeof(T))) ||
        (rc = r.alloc(&r.qBase, 4 * nb * sizeof(T))) ||
        (rc = r.alloc(&r.points, (size_t)S.contactSlots * 4 * sizeof(PointState<T>))) ||
        (rc = r.alloc(&r.branches, (size_t)S.nWorlds * sizeof(unsigned long long)))) {
        return rc;
    }
    // Parameters: the caller's, else the recorded ones.
    std::vector<double> h(nb * kState);
    {
        std::vector<float> com(3 * nb), q(4 * nb), v(3 * nb), w(3 * nb);
        TF_ADJ_CUDA(cudaMemcpy(com.data(), S.com0, com.size() * 4, cudaMemcpyDeviceToHost));
        TF_ADJ_CUDA(cudaMemcpy(q.data(), S.q0, q.size() * 4, cudaMemcpyDeviceToHost));
        TF_ADJ_CUDA(cudaMemcpy(v.data(), S.v0, v.size() * 4, cudaMemcpyDeviceToHost));
        TF_ADJ_CUDA(cudaMemcpy(w.data(), S.w0, w.size() * 4, cudaMemcpyDeviceToHost));
        for (size_t g = 0; g < nb; ++g) {
            for (int k = 0; k < 3; ++k) { h[g * kState + k] = com[3 * g + k]; }
            for (int k = 0; k < 4; ++k) { h[g * kState + 3 + k] = q[4 * g + k]; }
            for (int k = 0; k < 3; ++k) { h[g * kState + 7 + k] = v[3 * g + k]; }
            for (int k = 0; k < 3; ++k) { h[g * kState + 10 + k] = w[3 * g + k]; }
        }
        if (init) { h.assign(init, init + nb * kState); }
    }
    if ((rc = upload<T>(r.init, h, stream)) != TF_OK) { return rc; }
    std::vector<double> m(nb), f(ns);
    {
        std::vector<float> mf(nb), ff(ns);
        TF_ADJ_CUDA(cudaMemcpy(mf.data(), S.mass, nb * 4, cudaMemcpyDeviceToHost));
        TF_ADJ_CUDA(cudaMemcpy(ff.data(), S.friction, ns * 4, cudaMemcpyDeviceToHost));
        for (size_t g = 0; g < nb; ++g) { m[g] = mass ? mass[g] : (double)mf[g]; }
        for (size_t k = 0; k < ns; ++k) { f[k] = friction ? friction[k] : (double)ff[k]; }
    }
    for (size_t g = 0; g < nb; ++g) {
        if (!(m[g] > 0.0)) { m[g] = 1.0; }  // bodies without mass (static ones) never use it
    }
    if ((rc = upload<T>(r.mass, m, stream)) != TF_OK || (rc = upload<T>(r.friction, f, stream)) != TF_OK) { return rc; }
    Model<T> M = modelOf<T>(S, r);
    cudaEvent_t e0, e1;
    TF_ADJ_CUDA(cudaEventCreate(&e0));
    TF_ADJ_CUDA(cudaEventCreate(&e1));
    cudaEventRecord(e0, stream);
    const int blocks = (S.nWorlds + 3) / 4;
    k_model_forward<T><<<blocks, 128, 0, stream>>>(M);
    cudaEventRecord(e1, stream);
    TF_ADJ_CUDA(cudaGetLastError());
    TF_ADJ_CUDA(cudaStreamSynchronize(stream));
    cudaEventElapsedTime(&r.forwardMs, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::vector<double> out;
    if ((rc = download<T>(out, (const char*)r.states + stateBytes * (size_t)S.nSteps, nb * kState, stream)) != TF_OK) { return rc; }
    if (finalState) { std::copy(out.begin(), out.end(), finalState); }
    r.forwardDone = true;
    return TF_OK;
}

// The largest number of contact operations one world logs in one step.
int maxCalls(const AdjointSetup& S, uint64_t* out) {
    std::vector<TapeStep> steps(S.nSteps);
    TF_ADJ_CUDA(cudaMemcpy(steps.data(), S.steps, steps.size() * sizeof(TapeStep), cudaMemcpyDeviceToHost));
    std::vector<TapeWorld> tw(S.nWorlds);
    uint64_t most = 1;
    for (const TapeStep& ts : steps) {
        TF_ADJ_CUDA(cudaMemcpy(tw.data(), ts.worlds, tw.size() * sizeof(TapeWorld), cudaMemcpyDeviceToHost));
        for (const TapeWorld& w : tw) {
            const uint64_t colored = w.colorStart[w.colorCount] + w.restCount;
            const uint64_t impact = w.impactColorStart[w.impactColorCount] + w.impactRestCount;
            most = std::max<uint64_t>(most, (uint64_t)S.substeps * (3 * colored + 2 * impact) + colored);
        }
    }
    *out = most;
    return TF_OK;
}

template <class T>
int backwardT(Run& r, const AdjointSetup& S, cudaStream_t stream, const double* gradFinal, double* gradInit,
              double* gradMass, double* gradFriction) {
    const size_t nb = S.totalBodies, ns = S.totalShapes;
    int rc;
    uint64_t calls = 0;
    if ((rc = maxCalls(S, &calls)) != TF_OK) { return rc; }
    r.logStride = calls * (uint64_t)kCallWords;
    if (!r.stateAdj) {
        // Steps recomputed at once: as many slots as fit in a share of the free memory, up to the whole run.
        const size_t perSlot = (size_t)S.nWorlds * r.logStride * sizeof(T) +
                               (size_t)S.substeps * nb * kIntegWords * sizeof(T) + nb * (kState + 21) * sizeof(T) +
                               (size_t)S.contactSlots * 4 * sizeof(PointState<T>);
        size_t freeBytes = 0, totalBytes = 0;
        TF_ADJ_CUDA(cudaMemGetInfo(&freeBytes, &totalBytes));
        const size_t budget = std::min<size_t>(freeBytes / 2, (size_t)32 << 30);
        r.slots = (int)std::max<size_t>(1, std::min<size_t>((size_t)S.nSteps, budget / 2 / std::max<size_t>(perSlot, 1)));
        const size_t k = 2 * (size_t)r.slots;
        // The forward's single-slot working arrays give way to one per slot.
        for (void** p : { &r.invM, &r.invI, &r.dp, &r.dq, &r.qBase, &r.points }) {
            auto it = std::find(r.owned.begin(), r.owned.end(), *p);
            if (it != r.owned.end()) {
                cudaFree(*p);
                r.owned.erase(it);
            }
            *p = nullptr;
        }
        if ((rc = r.alloc(&r.invM, k * nb * sizeof(T))) || (rc = r.alloc(&r.invI, k * 9 * nb * sizeof(T))) ||
            (rc = r.alloc(&r.dp, k * 3 * nb * sizeof(T))) || (rc = r.alloc(&r.dq, k * 4 * nb * sizeof(T))) ||
            (rc = r.alloc(&r.qBase, k * 4 * nb * sizeof(T))) ||
            (rc = r.alloc(&r.points, k * (size_t)S.contactSlots * 4 * sizeof(PointState<T>))) ||
            (rc = r.alloc(&r.scratch, k * nb * kState * sizeof(T))) ||
            (rc = r.alloc(&r.stateAdj, nb * kState * sizeof(T))) || (rc = r.alloc(&r.dpAdj, 3 * nb * sizeof(T))) ||
            (rc = r.alloc(&r.dqAdj, 4 * nb * sizeof(T))) || (rc = r.alloc(&r.qBaseAdj, 4 * nb * sizeof(T))) ||
            (rc = r.alloc(&r.invMAdj, nb * sizeof(T))) || (rc = r.alloc(&r.invIAdj, 9 * nb * sizeof(T))) ||
            (rc = r.alloc(&r.pointAdj, (size_t)S.contactSlots * 4 * sizeof(PointState<T>))) ||
            (rc = r.alloc(&r.massAdj, nb * sizeof(T))) || (rc = r.alloc(&r.frictionAdj, ns * sizeof(T))) ||
            (rc = r.alloc(&r.integLog, k * (size_t)S.substeps * nb * kIntegWords * sizeof(T))) ||
            (rc = r.alloc(&r.log, k * (size_t)S.nWorlds * r.logStride * sizeof(T)))) {
            return rc;
        }
    }
    std::vector<double> g(gradFinal, gradFinal + nb * kState);
    if ((rc = upload<T>(r.stateAdj, g, stream)) != TF_OK) { return rc; }
    TF_ADJ_CUDA(cudaMemsetAsync(r.massAdj, 0, nb * sizeof(T), stream));
    TF_ADJ_CUDA(cudaMemsetAsync(r.frictionAdj, 0, ns * sizeof(T), stream));
    Model<T> M = modelOf<T>(S, r);
    cudaEvent_t e0, e1;
    TF_ADJ_CUDA(cudaEventCreate(&e0));
    TF_ADJ_CUDA(cudaEventCreate(&e1));
    if (!r.side) {
        int least = 0, greatest = 0;
        TF_ADJ_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        TF_ADJ_CUDA(cudaStreamCreateWithFlags(&r.side, cudaStreamNonBlocking));
        TF_ADJ_CUDA(cudaStreamCreateWithPriority(&r.walk, cudaStreamNonBlocking, greatest));
        for (cudaEvent_t* e : { &r.ready, &r.recomputed[0], &r.recomputed[1], &r.reversed[0], &r.reversed[1], &r.walked }) {
            TF_ADJ_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        }
    }
    cudaEventRecord(e0, stream);
    cudaEventRecord(r.ready, stream);
    TF_ADJ_CUDA(cudaStreamWaitEvent(r.side, r.ready, 0));
    TF_ADJ_CUDA(cudaStreamWaitEvent(r.walk, r.ready, 0));
    const int blocks = (S.nWorlds + 3) / 4;
    // Each warp of the reverse walk stages color batches in shared memory when the device grants the space
    // (set on every call: the attribute belongs to the current device).
    // Each warp of the reverse walk stages color batches and its world's body arrays in shared memory when the
    // device grants the space and that leaves as many worlds resident at once as the walk can have at all (it
    // is one dependent chain per world: worlds beyond those wait for a second wave); else the body arrays, or
    // both, stay in global memory. The attribute is set on every call: it belongs to the current device.
    if (r.maxBodies == 0) {
        std::vector<uint32_t> counts(S.nWorlds);
        TF_ADJ_CUDA(cudaMemcpy(counts.data(), S.bodyCount, counts.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        r.maxBodies = std::max<uint32_t>(1, *std::max_element(counts.begin(), counts.end()));
    }
    int device = 0, sms = 0;
    TF_ADJ_CUDA(cudaGetDevice(&device));
    TF_ADJ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    auto walkBytes = [&](int option) {  // 0: records and bodies staged, 1: records only, 2: nothing
        return 4 * ((option < 2 ? stageBytesPerWarp<T>() : 0) + bodyBytesPerWarp<T>(option == 0 ? r.maxBodies : 0));
    };
    int perSm[3] = { 0, 0, 0 };
    for (int option = 0; option < 3; ++option) {
        const size_t bytes = walkBytes(option);
        if (cudaFuncSetAttribute(k_model_reverse<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm[option], k_model_reverse<T>, 128, bytes) != cudaSuccess) {
            cudaGetLastError();
            perSm[option] = 0;
        }
    }
    // CTAs per SM that hold every world at once, or as many as any option allows.
    const int wanted = std::min<int>((S.nWorlds + 4 * sms - 1) / (4 * sms), std::max({ perSm[0], perSm[1], perSm[2] }));
    int option = 2;
    while (option > 0 && perSm[option - 1] >= std::max(wanted, 1)) { --option; }  // less shared memory, more CTAs
    const int staged = option < 2 ? 1 : 0;
    const uint32_t bodyCap = option == 0 ? r.maxBodies : 0;
    const size_t walkShared = walkBytes(option);
    if (cudaFuncSetAttribute(k_model_reverse<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)walkShared) != cudaSuccess) {
        return noteError(TF_E_CUDA, "adjoint: the reverse walk's shared memory was not granted");
    }
    // Chunk c recomputes into slot set c % 2 on the side stream once the reverse walk of chunk c - 2 has left
    // that set, so that it runs beside the walk of chunk c - 1; the walk of chunk c waits for its recompute.
    const int chunks = (S.nSteps + r.slots - 1) / r.slots;
    while ((int)r.chunkEvents.size() < 4 * chunks) {
        cudaEvent_t e;
        TF_ADJ_CUDA(cudaEventCreate(&e));
        r.chunkEvents.push_back(e);
    }
    int c = 0;
    for (int end = S.nSteps; end > 0; ++c) {
        const int count = std::min(end, r.slots), first = end - count, set = c % 2;
        const uint32_t base = (uint32_t)(set * r.slots);
        const unsigned warps = (unsigned)count * (unsigned)S.nWorlds;
        cudaEvent_t* ev = r.chunkEvents.data() + 4 * c;
        if (c >= 2) { TF_ADJ_CUDA(cudaStreamWaitEvent(r.side, r.reversed[set], 0)); }
        cudaEventRecord(ev[0], r.side);
        k_model_recompute<T><<<(warps + 3) / 4, 128, 0, r.side>>>(M, first, count, base);
        cudaEventRecord(ev[1], r.side);
        cudaEventRecord(r.recomputed[set], r.side);
        TF_ADJ_CUDA(cudaStreamWaitEvent(r.walk, r.recomputed[set], 0));
        cudaEventRecord(ev[2], r.walk);
        k_model_reverse<T><<<blocks, 128, walkShared, r.walk>>>(M, first, count, base, staged, bodyCap);
        cudaEventRecord(ev[3], r.walk);
        cudaEventRecord(r.reversed[set], r.walk);
        end = first;
    }
    cudaEventRecord(r.walked, r.walk);
    TF_ADJ_CUDA(cudaStreamWaitEvent(stream, r.walked, 0));
    cudaEventRecord(e1, stream);
    TF_ADJ_CUDA(cudaGetLastError());
    TF_ADJ_CUDA(cudaStreamSynchronize(stream));
    cudaEventElapsedTime(&r.backwardMs, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    r.recomputeMs = r.reverseMs = 0.0f;
    for (int k = 0; k < c; ++k) {
        float a = 0.0f, b = 0.0f;
        cudaEventElapsedTime(&a, r.chunkEvents[4 * k], r.chunkEvents[4 * k + 1]);
        cudaEventElapsedTime(&b, r.chunkEvents[4 * k + 2], r.chunkEvents[4 * k + 3]);
        r.recomputeMs += a;
        r.reverseMs += b;
    }
    std::vector<double> out;
    if (gradInit) {
        if ((rc = download<T>(out, r.stateAdj, nb * kState, stream)) != TF_OK) { return rc; }
        std::copy(out.begin(), out.end(), gradInit);
    }
    if (gradMass) {
        if ((rc = download<T>(out, r.massAdj, nb, stream)) != TF_OK) { return rc; }
        std::copy(out.begin(), out.end(), gradMass);
    }
    if (gradFriction) {
        if ((rc = download<T>(out, r.frictionAdj, ns, stream)) != TF_OK) { return rc; }
        std::copy(out.begin(), out.end(), gradFriction);
    }
    return TF_OK;
}

}  // namespace adj

// Entry points for the C ABI (tf_engine.cu): one run per batch.
void* adjointCreate() { return new adj::Run(); }
void adjointDestroy(void* run) { delete static_cast<adj::Run*>(run); }

int adjointForward(void* run, const AdjointSetup& S, void* stream, int precision, const double* init, const double* mass,
                   const double* friction, double* finalState) {
    adj::Run& r = *static_cast<adj::Run*>(run);
    r.precision = precision;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == 64) { return adj::forwardT<double>(r, S, st, init, mass, friction, finalState); }
    if (precision == 32) { return adj::forwardT<float>(r, S, st, init, mass, friction, finalState); }
    return noteError(TF_E_INVALID, "adjoint: precision must be 32 or 64");
}

int adjointBackward(void* run, const AdjointSetup& S, void* stream, const double* gradFinal, double* gradInit,
                    double* gradMass, double* gradFriction) {
    adj::Run& r = *static_cast<adj::Run*>(run);
    if (!r.forwardDone) { return noteError(TF_E_INVALID, "adjoint: backward needs a forward run first"); }
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (r.precision == 64) { return adj::backwardT<double>(r, S, st, gradFinal, gradInit, gradMass, gradFriction); }
    return adj::backwardT<float>(r, S, st, gradFinal, gradInit, gradMass, gradFriction);
}

int adjointBranches(void* run, int nWorlds, uint64_t* out) {
    const adj::Run& r = *static_cast<adj::Run*>(run);
    if (!r.forwardDone || !r.branches) { return noteError(TF_E_INVALID, "adjoint: no forward run to read branches from"); }
    const cudaError_t e = cudaMemcpy(out, r.branches, (size_t)nWorlds * sizeof(uint64_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { return noteError(TF_E_CUDA, std::string("adjoint: branches: ") + cudaGetErrorString(e)); }
    return TF_OK;
}

void adjointTimes(void* run, float* ms) {
    const adj::Run& r = *static_cast<adj::Run*>(run);
    ms[0] = r.forwardMs;
    ms[1] = r.backwardMs;
    ms[2] = r.recomputeMs;
    ms[3] = r.reverseMs;
}

}  // namespace tfb
