// The step kernels. Each kernel processes whole worlds: CTA k takes worlds order[k], order[k + gridDim.x],
// ... (largest first), and within a world its threads split bodies, candidates or one color's contacts,
// with __syncthreads() between dependent phases. Work that the reference does in one sequential pass
// whose result depends on order (graph coloring, union-find islands, the wake flood and contacts solved
// one at a time) runs on the world's first thread, in the reference's order.
//
// Kernel sequence of one step (src/world.cpp:1564-1727):
//   k_broadphase   growth, body-pair and half-space candidates, sort + unique   (world.cpp:752-870)
//   k_narrowphase  reuse or collide each candidate, carry impulses, merge       (world.cpp:872-993)
//   k_wake         wake sleeping bodies touched by moving ones                  (world.cpp:705-735)
//   k_prepare      step state, active/fast/impact lists, prepare, coloring     (world.cpp:1589-1657)
//   k_substep x n  refresh, integrate, warm start, solve, integrate, relax      (world.cpp:1658-1681)
//   k_finish       restitution, limits, refit bounds, sweep test, sleep         (world.cpp:1682-1726)
#pragma once

#include "tf_batch.cuh"
#include "tf_solver.cuh"

namespace tfb {

constexpr int kMaxBlock = 512;
constexpr uint32_t kDevPairOverflow = 1u << 0, kDevContactOverflow = 1u << 1, kDevNonFinite = 1u << 2,
                   kDevUnsupported = 1u << 4, kDevSweepSkipped = 1u << 5, kDevListOverflow = 1u << 6;

// Exclusive prefix sum over the block. Every thread calls it; blockDim.x is a multiple of 32.
__device__ __forceinline__ uint32_t blockExclusiveScan(uint32_t v, uint32_t& total) {
    __shared__ uint32_t warpSums[kMaxBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) { x += y; }
    }
    if (lane == 31) { warpSums[warp] = x; }
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < nw ? warpSums[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) { s += y; }
        }
        if (lane < nw) { warpSums[lane] = s; }
    }
    __syncthreads();
    const uint32_t prefix = (warp > 0 ? warpSums[warp - 1] : 0u) + x - v;
    total = warpSums[nw - 1];
    __syncthreads();
    return prefix;
}

// Calls emit(i, position) for every i < n where pred(i) holds, positions dense and in index order. Ends with
// a block barrier, so everything emit wrote is visible to every thread on return.
template <class Pred, class Emit>
__device__ uint32_t blockCompact(uint32_t n, Pred pred, Emit emit) {
    uint32_t base = 0;
    for (uint32_t start = 0; start < n; start += blockDim.x) {
        const uint32_t i = start + threadIdx.x;
        const bool f = i < n && pred(i);
        uint32_t tot;
        const uint32_t pos = blockExclusiveScan(f ? 1u : 0u, tot);
        if (f) { emit(i, base + pos); }
        base += tot;
    }
    __syncthreads();
    return base;
}

__device__ __forceinline__ uint64_t pairKey(uint32_t a, uint32_t b) {
    return ((uint64_t)(a < b ? a : b) << 32) | (uint64_t)(a < b ? b : a);
}

__device__ __forceinline__ void emitCandidate(const Batch& B, const WorldInfo& wi, uint32_t* count, uint64_t key) {
    const uint32_t pos = atomicAdd(count, 1u);
    if (pos < wi.candCap) { B.cand[wi.candFirst + pos] = key; }
}

// ---------------------------------------------------------------------------------------------------------
// Broadphase (src/world.cpp:752-870).

// A half-space against one body's shapes (src/world.cpp:844-867).
__device__ void pairPlane(const Batch& B, const WorldInfo& wi, uint32_t gp, uint32_t gb, uint32_t* count) {
    const DShape& sp = B.shapes[gp];
    const DBody& pb = B.bodies[sp.body];
    const DBody& b = B.bodies[gb];
    const bool planeMoving = movingAwake(pb);
    if (!b.alive || gb == sp.body || (!planeMoving && !movingAwake(b))) { return; }
    const float gp_ = B.grow[sp.body];
    const Transform xp = pb.xf * sp.local;
    const Vec3 n = rotate(xp.q, Vec3{ 0, 0, 1 });
    const float offset = dot(n, xp.p);
    const float g = gp_ + B.grow[gb];
    auto reaches = [&](const Vec3& lo, const Vec3& hi) {
        const Vec3 c = (lo + hi) * 0.5f, e = (hi - lo) * 0.5f + Vec3{ g, g, g };
        return dot(c, n) - offset <= e.x * fabsf(n.x) + e.y * fabsf(n.y) + e.z * fabsf(n.z);
    };
    if (b.hasBounds && !reaches(b.lo, b.hi)) { return; }
    for (uint32_t x = 0; x < b.shapeCount; ++x) {
        const uint32_t gs = B.shapeList[b.shapeFirst + x];
        const DShape& s = B.shapes[gs];
        if (s.kind != kHalfSpace && !reaches(s.lo, s.hi)) { continue; }
        // pairable(sp, s): neither a sensor, different bodies, one of them dynamic.
        if (sp.sensor || s.sensor || sp.body == s.body) { continue; }
        if (pb.type != kDynamic && b.type != kDynamic) { continue; }
        // test(pi, si) (src/world.cpp:798-808).
        const float ga = B.grow[sp.body], gbb = B.grow[s.body];
        const Vec3 g3a{ ga, ga, ga }, g3b{ gbb, gbb, gbb };
        if (!boxesOverlap(sp.lo - g3a, sp.hi + g3a, s.lo - g3b, s.hi + g3b)) { continue; }
        if (!(sp.category & s.mask) || !(s.category & sp.mask)) { continue; }
        emitCandidate(B, wi, count, pairKey(sp.index, s.index));
    }
}

// Sorts keys[0, n) ascending in shared memory and removes repeats; returns the unique count written back to
// out[0, unique).
__device__ uint32_t sortUnique(uint64_t* s, uint32_t n, uint64_t* out) {
    uint32_t p = 1;
    while (p < n) { p <<= 1; }
    for (uint32_t i = n + threadIdx.x; i < p; i += blockDim.x) { s[i] = ~0ull; }
    __syncthreads();
    for (uint32_t k = 2; k <= p; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < p; i += blockDim.x) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const uint64_t a = s[i], b = s[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        s[i] = b;
                        s[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    const uint32_t unique = blockCompact(
        n, [&](uint32_t i) { return i == 0 || s[i] != s[i - 1]; }, [&](uint32_t i, uint32_t pos) { out[pos] = s[i]; });
    __syncthreads();
    return unique;
}

// Reads the abort word once per CTA: true when an earlier step of this launch sequence overflowed a list,
// or this step did in an earlier kernel.
__device__ __forceinline__ bool stepAborted(const Batch& B, int serial) {
    __shared__ int s_skip;
    if (threadIdx.x == 0) { s_skip = *(volatile uint32_t*)B.abortStep <= (uint32_t)serial; }
    __syncthreads();
    const bool skip = s_skip != 0;
    __syncthreads();
    return skip;
}

// The shapes of two bodies whose grown bounds overlap, paired by their own grown bounds
// (src/world.cpp:819-842).
__device__ void pairShapes(const Batch& B, const WorldInfo& wi, const DBody& ba, const DBody& bb, float gA, float gB,
                           const Vec3& loA, const Vec3& hiA, const Vec3& loB, const Vec3& hiB, const Vec3& reach,
                           uint32_t* count) {
    const Vec3 nearLoA = loB - reach, nearHiA = hiB + reach;
    const Vec3 nearLoB = loA - reach, nearHiB = hiA + reach;
    const Vec3 grownA{ gA, gA, gA }, grownB{ gB, gB, gB };
    for (uint32_t x = 0; x < ba.shapeCount; ++x) {
        const DShape& s = B.shapes[B.shapeList[ba.shapeFirst + x]];
        if (s.kind == kHalfSpace || s.sensor || !boxesOverlap(s.lo, s.hi, nearLoA, nearHiA)) { continue; }
        const Vec3 xlo = s.lo - grownA, xhi = s.hi + grownA;
        for (uint32_t y = 0; y < bb.shapeCount; ++y) {
            const DShape& t = B.shapes[B.shapeList[bb.shapeFirst + y]];
            if (t.kind == kHalfSpace || t.sensor || !boxesOverlap(t.lo, t.hi, nearLoB, nearHiB)) { continue; }
            if (!boxesOverlap(xlo, xhi, t.lo - grownB, t.hi + grownB)) { continue; }
            if (!(s.category & t.mask) || !(t.category & s.mask)) { continue; }
            emitCandidate(B, wi, count, pairKey(s.index, t.index));
        }
    }
}

constexpr uint32_t kBodyLive = 1u, kBodyDynamic = 2u, kBodyMoving = 4u;
// Largest worlds whose bodies the broadphase and the substep stage in shared memory.
constexpr uint32_t kBroadStage = 2048;
constexpr uint32_t kSolveStage = 1400;

// A body as the pair test sees it: bounds, growth and the three flags above.
struct PairBody {
    Vec3 lo, hi;
    float grow;
    uint32_t flags;
};

__device__ __forceinline__ PairBody pairBodyOf(const Batch& B, uint32_t g) {
    const DBody& b = B.bodies[g];
    PairBody p;
    p.lo = b.lo;
    p.hi = b.hi;
    p.grow = B.grow[g];
    p.flags = ((b.alive && b.hasBounds) ? kBodyLive : 0u) | (b.type == kDynamic ? kBodyDynamic : 0u) |
              (movingAwake(b) ? kBodyMoving : 0u);
    return p;
}

// Body pairs whose grown bounds overlap, then their shapes (src/world.cpp:788-842), and half-space pairs
// (:844-867); the keys are sorted and made unique (:868-869). Bodies and growths are staged in shared
// memory for worlds of up to stageN bodies; a warp takes one body and its lanes the bodies after it.
__global__ void __launch_bounds__(kMaxBlock) k_broadphase(Batch B, StepParams P, uint32_t sortCap, uint32_t stageN,
                                                          int serial) {
    extern __shared__ __align__(16) uint64_t s_keys[];
    __shared__ uint32_t s_count;
    PairBody* staged = reinterpret_cast<PairBody*>(s_keys + sortCap);
    if (stepAborted(B, serial)) { return; }
    for (int o = blockIdx.x; o < B.nWorlds; o += gridDim.x) {
        const uint32_t w = B.order[o];
        const WorldInfo wi = B.info[w];
        WorldCounts& wc = B.counts[w];
        const uint32_t n = wi.bodyCount;
        const bool useStage = n <= stageN;
        if (threadIdx.x == 0) { s_count = 0; }
        // Growth by the speculative distance and the travel over the step (src/world.cpp:754-765).
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const DBody& b = B.bodies[wi.bodyFirst + i];
            float g = P.tol.speculative;
            if (b.alive && b.type != kStatic && !(lengthSquared(b.v) == 0.0f && lengthSquared(b.w) == 0.0f)) {
                g += (length(b.v) + length(b.w) * b.extent) * P.dt;
            }
            B.grow[wi.bodyFirst + i] = g;
            if (useStage) {
                PairBody p;
                p.lo = b.lo;
                p.hi = b.hi;
                p.grow = g;
                p.flags = ((b.alive && b.hasBounds) ? kBodyLive : 0u) | (b.type == kDynamic ? kBodyDynamic : 0u) |
                          (movingAwake(b) ? kBodyMoving : 0u);
                staged[i] = p;
            }
        }
        __syncthreads();
        const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
        for (uint32_t a = warp; a + 1 < n; a += warps) {
            const PairBody A = useStage ? staged[a] : pairBodyOf(B, wi.bodyFirst + a);
            if (!(A.flags & kBodyLive)) { continue; }
            for (uint32_t b = a + 1 + lane; b < n; b += 32) {
                const PairBody Bb = useStage ? staged[b] : pairBodyOf(B, wi.bodyFirst + b);
                if (!(Bb.flags & kBodyLive)) { continue; }
                if (!((A.flags | Bb.flags) & kBodyDynamic)) { continue; }
                if (!((A.flags | Bb.flags) & kBodyMoving)) { continue; }
                const float g = A.grow + Bb.grow;
                const Vec3 reach{ g, g, g };
                if (!boxesOverlap(A.lo - reach, A.hi + reach, Bb.lo, Bb.hi)) { continue; }
                pairShapes(B, wi, B.bodies[wi.bodyFirst + a], B.bodies[wi.bodyFirst + b], A.grow, Bb.grow, A.lo, A.hi,
                           Bb.lo, Bb.hi, reach, &s_count);
            }
        }
        for (uint32_t pl = 0; pl < wi.planeCount; ++pl) {
            const uint32_t gp = B.planeList[wi.planeFirst + pl];
            for (uint32_t b = threadIdx.x; b < n; b += blockDim.x) { pairPlane(B, wi, gp, wi.bodyFirst + b, &s_count); }
        }
        __syncthreads();
        const uint32_t count = s_count;
        if (count > wi.candCap || count > sortCap) {
            // The list did not fit: this step stops here and the host grows the world's lists.
            if (threadIdx.x == 0) {
                wc.flags |= count > wi.candCap ? kDevPairOverflow : kDevUnsupported;
                wc.candNeeded = max(wc.candNeeded, count);
                atomicMin(B.abortStep, (uint32_t)serial);
            }
            __syncthreads();
            continue;
        }
        for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) { s_keys[i] = B.cand[wi.candFirst + i]; }
        __syncthreads();
        const uint32_t unique = sortUnique(s_keys, count, B.cand + wi.candFirst);
        if (threadIdx.x == 0) {
            wc.candCount = unique;
            wc.candNeeded = max(wc.candNeeded, count);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------------------
// Narrowphase and contact bookkeeping (src/world.cpp:872-1025).

__device__ __forceinline__ Vec3 lift(const DBody& a, const DBody& b, const Vec3& normal, float separation, float spec) {
    if (isPlanar(a) || isPlanar(b)) { return zero3(); }
    return separation > spec ? normal * (0.5f * separation) : zero3();
}

// src/world.cpp:1002-1009.
__device__ __forceinline__ bool stillFits(const DContact& c, const DBody& a, const DBody& b, const StepParams& P) {
    if (!(c.flags & kCReusable)) { return false; }
    const float reach = P.reuseDistance;
    if (lengthSquared(unrotate(a.xf.q, b.com - a.com) - c.baseOffset) > reach * reach) { return false; }
    const Quat turn = conjugate(a.xf.q) * b.xf.q;
    return fabsf(dot(turn, c.baseTurn)) >= P.reuseCos;
}

// src/world.cpp:1012-1025.
__device__ void measureAgain(const DBody& a, const DBody& b, DContact& c, const StepParams& P) {
    c.normal = rotate(a.xf.q, c.localNormal);
    c.tangent1 = perpendicular(c.normal);
    c.tangent2 = cross(c.normal, c.tangent1);
    for (int i = 0; i < c.count; ++i) {
        DPoint& p = c.points[i];
        const Vec3 pa = apply(a.xf, p.surfaceA), pb = apply(b.xf, p.surfaceB);
        const Vec3 mid = (pa + pb) * 0.5f;
        p.separation = dot(pb - pa, c.normal);
        const Vec3 up = lift(a, b, c.normal, p.separation, P.tol.speculative);
        p.anchorA = mid - up - a.com;
        p.anchorB = mid + up - b.com;
        p.tangentImpulse = p.tangentImpulse - c.normal * dot(c.normal, p.tangentImpulse);
    }
}

// Each new point continues the nearest old point in reach; an old point continued by several new points
// splits its impulse among them (src/world.cpp:102-124).
__device__ void carryImpulses(const DContact& old, DContact& c, float matchSq) {
    int from[4], claims[4] = { 0, 0, 0, 0 };
    for (int i = 0; i < c.count; ++i) {
        from[i] = -1;
        float bestSq = matchSq;
        for (int k = 0; k < old.count; ++k) {
            const float d = lengthSquared(old.points[k].localA - c.points[i].localA);
            if (d <= bestSq) {
                from[i] = k;
                bestSq = d;
            }
        }
        if (from[i] >= 0) { ++claims[from[i]]; }
    }
    for (int i = 0; i < c.count; ++i) {
        if (from[i] < 0) { continue; }
        const DPoint& o = old.points[from[i]];
        const float share = 1.0f / (float)claims[from[i]];
        c.points[i].normalImpulse = o.normalImpulse * share;
        c.points[i].tangentImpulse = (o.tangentImpulse - c.normal * dot(c.normal, o.tangentImpulse)) * share;
    }
    c.rollingImpulse = old.rollingImpulse;
}

__device__ __forceinline__ int nearestPoint(const DContact& old, const Vec3& localA) {
    int best = -1;
    float bestSq = FLT_MAX;
    for (int k = 0; k < old.count; ++k) {
        const float d = lengthSquared(old.points[k].localA - localA);
        if (d < bestSq) {
            best = k;
            bestSq = d;
        }
    }
    return best;
}

// Collides one shape pair over dt as Impl::collidePair does for non-mesh, non-planar pairs
// (src/world.cpp:505-533). Returns false for a pair this build cannot collide.
__device__ bool collidePair(const Batch& B, const StepParams& P, const DShape& sa, const DShape& sb, float dt,
                            Manifold& m, int reuseKind, int reuseA, int reuseB) {
    if (!TF_OK_INDEX(B, (sa.poly < 0 || (uint32_t)sa.poly < B.nPolys) && (sb.poly < 0 || (uint32_t)sb.poly < B.nPolys) &&
                            sa.body < B.totalBodies && sb.body < B.totalBodies,
                     30, sa.body, sb.body)) {
        m.count = 0;
        return true;
    }
    const DBody& ba = B.bodies[sa.body];
    const DBody& bb = B.bodies[sb.body];
    const float travel = relativeTravel(ba, bb, dt);
    const float margin = P.tol.speculative + travel;
    const Transform xa = ba.xf * sa.local;
    const Transform xb = bb.xf * sb.local;
    const Motion mo{ ba.v, ba.w, ba.com, bb.v, bb.w, bb.com, dt, travel > P.tol.speculative };
    return collideShapes(B.cx, sa, xa, sb, xb, margin, mo, m, reuseKind, reuseA, reuseB);
}

// First index in [0, n) whose key is not below key.
__device__ __forceinline__ uint32_t lowerKey(const DContact* c, uint32_t n, uint64_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (c[mid].key < key) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// One candidate: keep and measure the old contact when the pair barely moved, else collide it and carry the
// old impulses over (src/world.cpp:883-959).
__device__ void narrowOne(const Batch& B, const StepParams& P, const WorldInfo& wi, WorldCounts& wc, uint32_t i,
                          const DContact* old, uint32_t oldCount) {
    const uint64_t key = B.cand[wi.candFirst + i];
    const uint32_t ia = (uint32_t)(key >> 32), ib = (uint32_t)(key & 0xffffffffu);
    if (!TF_OK_INDEX(B, ia < wi.shapeCount && ib < wi.shapeCount, 1, wi.bodyFirst, ia)) {
        B.stageUsed[wi.candFirst + i] = 0;
        return;
    }
    const uint32_t gsa = wi.shapeFirst + ia, gsb = wi.shapeFirst + ib;
    const DShape sa = B.shapes[gsa];
    const DShape sb = B.shapes[gsb];
    if (!TF_OK_INDEX(B, sa.body - wi.bodyFirst < wi.bodyCount && sb.body - wi.bodyFirst < wi.bodyCount, 2,
                     wi.bodyFirst, sa.body)) {
        B.stageUsed[wi.candFirst + i] = 0;
        return;
    }
    if (!TF_OK_INDEX(B, oldCount <= wi.contactCap, 3, wi.bodyFirst, oldCount)) {
        B.stageUsed[wi.candFirst + i] = 0;
        return;
    }
    const DBody& ba = B.bodies[sa.body];
    const DBody& bb = B.bodies[sb.body];
    const uint32_t lo = lowerKey(old, oldCount, key);
    uint32_t hi = lo;
    while (hi < oldCount && old[hi].key == key) { ++hi; }
    const bool hasOld = lo < hi;
    bool keep = hasOld;
    for (uint32_t it = lo; it < hi && keep; ++it) { keep = stillFits(old[it], ba, bb, P); }
    const bool touched = hasOld && (old[lo].flags & kCTouched);
    DContact& out = B.stage[wi.candFirst + i];
    uint8_t used = 0;
    if (keep) {
        if (hi - lo > 1) { atomicOr(&wc.flags, kDevUnsupported); }
        out = old[lo];
        measureAgain(ba, bb, out, P);
        used = 1;
    } else {
        if (isPlanar(ba) || isPlanar(bb)) { atomicOr(&wc.flags, kDevUnsupported); }
        Manifold m;
        if (!collidePair(B, P, sa, sb, P.dt, m, kFeatNone, -1, -1)) { atomicOr(&wc.flags, kDevUnsupported); }
        if (m.count > 0) {
            DContact c{};
            c.key = key;
            c.part = 0;
            c.shapeA = gsa;
            c.shapeB = gsb;
            c.bodyA = sa.body;
            c.bodyB = sb.body;
            c.flags = touched ? kCTouched : 0u;
            c.featKind = m.featKind;
            c.featA = m.featA;
            c.featB = m.featB;
            c.normal = m.normal;
            c.tangent1 = perpendicular(m.normal);
            c.tangent2 = cross(m.normal, c.tangent1);
            c.count = m.count;
            for (int k = 0; k < m.count; ++k) {
                DPoint& p = c.points[k];
                const Vec3 pos = m.points[k].position;
                const float sep = m.points[k].separation;
                const Vec3 half = m.normal * (0.5f * sep);
                p.surfaceA = applyInverse(ba.xf, pos - half);
                p.surfaceB = applyInverse(bb.xf, pos + half);
                p.localA = applyInverse(ba.xf, pos);
                p.separation = sep;
                const Vec3 up = lift(ba, bb, m.normal, sep, P.tol.speculative);
                p.anchorA = pos - up - ba.com;
                p.anchorB = pos + up - bb.com;
            }
            // remember (src/world.cpp:995-1000).
            c.localNormal = unrotate(ba.xf.q, c.normal);
            c.baseOffset = unrotate(ba.xf.q, bb.com - ba.com);
            c.baseTurn = conjugate(ba.xf.q) * bb.xf.q;
            c.flags |= kCReusable;
            // The old contact of the pair whose normal is closest (src/world.cpp:543-549).
            int best = -1;
            for (uint32_t it = lo; it < hi; ++it) {
                if (old[it].count > 0 && (best < 0 || dot(old[it].normal, c.normal) > dot(old[best].normal, c.normal))) {
                    best = (int)it;
                }
            }
            if (best >= 0) { carryImpulses(old[best], c, P.tol.speculative * P.tol.speculative); }
            out = c;
            used = 1;
        }
    }
    if (used) {
        out.friction = sqrtf(sa.friction * sb.friction);
        out.restitution = maxf(sa.restitution, sb.restitution);
        out.rollingResistance = maxf(sa.rollingResistance, sb.rollingResistance);
        if (ba.type == kDynamic && !ba.awake && movingAwake(bb)) {
            B.wakeMark[sa.body] = 1;
            wc.wakePending = 1;
        }
        if (bb.type == kDynamic && !bb.awake && movingAwake(ba)) {
            B.wakeMark[sb.body] = 1;
            wc.wakePending = 1;
        }
    }
    B.stageUsed[wi.candFirst + i] = used;
}

__device__ __forceinline__ bool keyLess(uint64_t ka, uint32_t pa, uint64_t kb, uint32_t pb) {
    return ka != kb ? ka < kb : pa < pb;
}

__global__ void __launch_bounds__(kMaxBlock) k_narrowphase(Batch B, StepParams P, int serial) {
    if (stepAborted(B, serial)) { return; }
    for (int o = blockIdx.x; o < B.nWorlds; o += gridDim.x) {
        const uint32_t w = B.order[o];
        const WorldInfo wi = B.info[w];
        WorldCounts& wc = B.counts[w];
        const uint32_t nc = wc.candCount;
        const uint32_t oldCount = wc.contactCount;
        const DContact* old = B.previous + wi.contactFirst;
        for (uint32_t i = threadIdx.x; i < nc; i += blockDim.x) { narrowOne(B, P, wi, wc, i, old, oldCount); }
        __syncthreads();
        const uint32_t cf = wi.contactFirst;
        const uint32_t nC = blockCompact(
            nc, [&](uint32_t i) { return B.stageUsed[wi.candFirst + i] != 0; },
            [&](uint32_t i, uint32_t pos) {
                const DContact& c = B.stage[wi.candFirst + i];
                B.mergeKeyA[cf + pos] = c.key;
                B.mergePartA[cf + pos] = c.part;
                B.mergeIdxA[cf + pos] = i;
            });
        // Contacts of pairs where nothing moves and one body is dynamic (asleep) stay as they were
        // (src/world.cpp:961-988).
        const uint32_t nK = blockCompact(
            oldCount,
            [&](uint32_t j) {
                const DContact& c = old[j];
                if (!TF_OK_INDEX(B, c.bodyA - wi.bodyFirst < wi.bodyCount && c.bodyB - wi.bodyFirst < wi.bodyCount, 4,
                                 wi.bodyFirst, j)) {
                    return false;
                }
                const DBody& a = B.bodies[c.bodyA];
                const DBody& b = B.bodies[c.bodyB];
                if ((c.flags & kCRemoved) || movingAwake(a) || movingAwake(b)) { return false; }
                return !(a.type != kDynamic && b.type != kDynamic);
            },
            [&](uint32_t j, uint32_t pos) {
                B.mergeKeyB[cf + pos] = old[j].key;
                B.mergePartB[cf + pos] = old[j].part;
                B.mergeIdxB[cf + pos] = j;
            });
        __syncthreads();
        const uint32_t total = nC + nK;
        if (total > wi.contactCap) {
            if (threadIdx.x == 0) {
                wc.flags |= kDevContactOverflow;
                wc.contactNeeded = max(wc.contactNeeded, total);
                atomicMin(B.abortStep, (uint32_t)serial);
            }
            __syncthreads();
            continue;
        }
        // Stable merge by (key, part): collided contacts first among equals, as std::inplace_merge keeps them.
        for (uint32_t x = threadIdx.x; x < nC; x += blockDim.x) {
            const uint64_t k = B.mergeKeyA[cf + x];
            const uint32_t p = B.mergePartA[cf + x];
            uint32_t l = 0, h = nK;
            while (l < h) {
                const uint32_t mid = (l + h) >> 1;
                if (keyLess(B.mergeKeyB[cf + mid], B.mergePartB[cf + mid], k, p)) {
                    l = mid + 1;
                } else {
                    h = mid;
                }
            }
            B.contacts[cf + x + l] = B.stage[wi.candFirst + B.mergeIdxA[cf + x]];
        }
        for (uint32_t y = threadIdx.x; y < nK; y += blockDim.x) {
            const uint64_t k = B.mergeKeyB[cf + y];
            const uint32_t p = B.mergePartB[cf + y];
            uint32_t l = 0, h = nC;
            while (l < h) {
                const uint32_t mid = (l + h) >> 1;
                if (!keyLess(k, p, B.mergeKeyA[cf + mid], B.mergePartA[cf + mid])) {
                    l = mid + 1;
                } else {
                    h = mid;
                }
            }
            B.contacts[cf + y + l] = old[B.mergeIdxB[cf + y]];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            wc.nextContactCount = total;
            wc.contactNeeded = max(wc.contactNeeded, total);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------------------
// Waking (src/world.cpp:705-735): sleeping bodies a moving body reached wake, and so does everything linked
// to them by a contact with points. Runs on the world's first thread; it is rare.

__global__ void k_wake(Batch B, int serial) {
    if (stepAborted(B, serial)) { return; }
    if (threadIdx.x != 0) { return; }
    for (int o = blockIdx.x; o < B.nWorlds; o += gridDim.x) {
        const uint32_t w = B.order[o];
        const WorldInfo wi = B.info[w];
        WorldCounts& wc = B.counts[w];
        if (!wc.wakePending) { continue; }
        wc.wakePending = 0;
        uint32_t* stack = B.unionParent + wi.bodyFirst;
        uint32_t top = 0;
        for (uint32_t i = 0; i < wi.bodyCount; ++i) {
            const uint32_t g = wi.bodyFirst + i;
            if (!B.wakeMark[g]) { continue; }
            const DBody& b = B.bodies[g];
            if (b.alive && b.type == kDynamic && !b.awake && top < wi.bodyCount) {
                stack[top++] = g;
            } else {
                B.wakeMark[g] = 0;
            }
        }
        const DContact* cs = B.contacts + wi.contactFirst;
        const uint32_t nc = wc.nextContactCount;
        while (top > 0) {
            const uint32_t g = stack[--top];
            DBody& b = B.bodies[g];
            B.wakeMark[g] = 0;
            if (b.awake) { continue; }
            b.awake = 1;
            b.sleepTime = 0.0f;
            updateInverseMass(b);
            for (uint32_t ci = 0; ci < nc; ++ci) {
                const DContact& c = cs[ci];
                if (c.bodyA != g && c.bodyB != g) { continue; }
                if (ci > 0 && cs[ci - 1].key == c.key) { continue; }  // one link per pair
                const uint32_t other = c.bodyA == g ? c.bodyB : c.bodyA;
                const DBody& ob = B.bodies[other];
                if (ob.type != kDynamic || ob.awake || B.wakeMark[other]) { continue; }
                bool linked = false;
                for (uint32_t k = ci; k < nc && cs[k].key == c.key; ++k) { linked = linked || cs[k].count > 0; }
                if (linked && top < wi.bodyCount) {
                    B.wakeMark[other] = 1;
                    stack[top++] = other;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------------------
// Step state, lists, preparation and coloring (src/world.cpp:1589-1657, src/lanes.cpp:356-407).

// Shared-memory staging of a world's coloring and islands, sized per batch by the host (at most these).
// Larger worlds run the same code on global scratch.
constexpr uint32_t kStageBodies = 4096;
constexpr uint32_t kStageContacts = 8192;
constexpr uint32_t kNone = 0xffffffffu;

// Greedy lowest free color of 32 over the moving bodies, in list order (src/lanes.cpp:356-374). endA/endB
// hold each contact's moving bodies (kNone for one that does not move) or kNone in both with colorable 0.
__device__ void colorSequential(uint32_t n, const uint32_t* endA, const uint32_t* endB, const uint8_t* colorable,
                                uint32_t* masks, uint8_t* color) {
    for (uint32_t x = 0; x < n; ++x) {
        uint8_t k = kNoColor;
        if (colorable[x]) {
            const uint32_t a = endA[x], b = endB[x];
            const uint32_t taken = (a != kNone ? masks[a] : 0u) | (b != kNone ? masks[b] : 0u);
            if (taken != 0xffffffffu) {
                const int f = __ffs(~taken) - 1;
                if (a != kNone) { masks[a] |= 1u << f; }
                if (b != kNone) { masks[b] |= 1u << f; }
                k = (uint8_t)f;
            }
        }
        color[x] = k;
    }
}

// Groups a contact list by color: every color's contacts (any order within a color, which solves the same)
// into colored, colors in ascending order, the uncolored ones into rest in list order.
__device__ void bucketByColor(uint32_t n, const uint32_t* list, const uint8_t* colorOf, uint32_t* colored,
                              uint32_t* rest, uint32_t* startOut, uint32_t& colorsUsed, uint32_t& restCount) {
    __shared__ uint32_t s_size[kColors + 1];
    __shared__ uint32_t s_fill[kColors + 1];
    for (uint32_t k = threadIdx.x; k <= kColors; k += blockDim.x) { s_size[k] = 0; }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < n; x += blockDim.x) { atomicAdd(&s_size[colorOf[list[x]]], 1u); }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t sum = 0, used = 0;
        for (int k = 0; k <= kColors; ++k) {
            startOut[k] = sum;
            s_fill[k] = sum;
            sum += s_size[k];
            if (k < kColors && s_size[k] > 0) { used = (uint32_t)k + 1; }
        }
        colorsUsed = used;
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < n; x += blockDim.x) {
        const uint8_t k = colorOf[list[x]];
        if (k != kNoColor) {
            const uint32_t at = atomicAdd(&s_fill[k], 1u);
#if defined(TF_DEVICE_CHECKS)
            if (at >= n) { continue; }
#endif
            colored[at] = list[x];
        }
    }
    const uint32_t r = blockCompact(n, [&](uint32_t x) { return colorOf[list[x]] == kNoColor; },
                                    [&](uint32_t x, uint32_t pos) { rest[pos] = list[x]; });
    if (threadIdx.x == 0) { restCount = r; }
    __syncthreads();
}

__global__ void __launch_bounds__(kMaxBlock) k_prepare(Batch B, StepParams P, uint32_t stageBodies,
                                                       uint32_t stageContacts, int serial) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    __shared__ uint32_t s_fast, s_fastSolid;
    if (stepAborted(B, serial)) { return; }
    for (int o = blockIdx.x; o < B.nWorlds; o += gridDim.x) {
        const uint32_t w = B.order[o];
        const WorldInfo wi = B.info[w];
        WorldCounts& wc = B.counts[w];
        uint32_t nc = wc.nextContactCount;
        if (!TF_OK_INDEX(B, nc <= wi.contactCap, 6, w, nc)) { nc = 0; }
        if (threadIdx.x == 0) {
            wc.contactCount = nc;
            s_fast = 0;
            s_fastSolid = 0;
        }
        for (uint32_t i = threadIdx.x; i < wi.bodyCount; i += blockDim.x) {
            const uint32_t g = wi.bodyFirst + i;
            DBody& b = B.bodies[g];
            B.struck[g] = 0;
            if (!b.alive) { continue; }
            b.q0 = b.xf.q;
            b.qBase = b.xf.q;
            b.com0 = b.com;
            b.expectedTravel = (length(b.v) + length(b.w) * b.extent) * P.dt;
            b.dp = zero3();
            b.dq = qid();
            updateInverseMass(b);
        }
        __syncthreads();
        const uint32_t cf = wi.contactFirst;
        DContact* cs = B.contacts + cf;
        const uint32_t nActive = blockCompact(
            nc,
            [&](uint32_t i) {
                if (!TF_OK_INDEX(B, cs[i].bodyA - wi.bodyFirst < wi.bodyCount && cs[i].bodyB - wi.bodyFirst < wi.bodyCount &&
                                    cs[i].count >= 0 && cs[i].count <= 4, 5, wi.bodyFirst, i)) {
                    B.cflags[cf + i] = 0;
                    return false;
                }
                const DBody& a = B.bodies[cs[i].bodyA];
                const DBody& b = B.bodies[cs[i].bodyB];
                const bool on = (a.type == kDynamic && a.awake) || (b.type == kDynamic && b.awake);
                uint8_t f = 0;
                if (on && relativeTravel(a, b, P.dt) > P.tol.speculative) {
                    f |= kFlagFast;
                    atomicAdd(&s_fast, 1u);
                    if (!isPlanar(a) && !isPlanar(b)) {
                        f |= kFlagFastSolid;
                        atomicAdd(&s_fastSolid, 1u);
                    }
                }
                B.cflags[cf + i] = f | (on ? kFlagActive : 0);
                return on;
            },
            [&](uint32_t i, uint32_t pos) { B.active[cf + pos] = i; });
        const uint32_t* act = B.active + cf;
        // Staging for the coloring: shared memory when the world fits, else the world's global scratch.
        const bool staged = wi.bodyCount <= stageBodies && nActive <= stageContacts;
        uint32_t* masks = staged ? reinterpret_cast<uint32_t*>(s_raw) : B.bodyColors + wi.bodyFirst;
        uint32_t* endA = staged ? masks + stageBodies : B.mergeIdxA + cf;
        uint32_t* endB = staged ? endA + stageContacts : B.mergeIdxB + cf;
        uint8_t* colorable = staged ? reinterpret_cast<uint8_t*>(endB + stageContacts) : B.cflags + cf;
        // Colors by active position; moved to contact order below. The merge scratch is free by now.
        uint8_t* colorTmp = reinterpret_cast<uint8_t*>(B.mergePartA + cf);
        for (uint32_t i = threadIdx.x; i < wi.bodyCount; i += blockDim.x) { masks[i] = 0; }
        for (uint32_t x = threadIdx.x; x < nActive; x += blockDim.x) {
            if (!TF_OK_INDEX(B, act[x] < nc, 7, w, x)) { continue; }
            DContact& c = cs[act[x]];
            const DBody& a = B.bodies[c.bodyA];
            const DBody& b = B.bodies[c.bodyB];
            prepareContact(a, b, c);
            makeContactAxes(a, b, c, B.axes + (size_t)(cf + act[x]) * kAxesPerContact);
            c.flags &= ~kCLaned;
            const bool can = !(c.flags & kCPlanar) && !(c.rollingResistance > 0.0f);
            endA[x] = movingBody(a) ? c.bodyA - wi.bodyFirst : kNone;
            endB[x] = movingBody(b) ? c.bodyB - wi.bodyFirst : kNone;
            if (staged) { colorable[x] = can ? 1 : 0; }
        }
        __syncthreads();
        if (!staged) {
            // The global form reuses cflags for colorable, so keep the fast flags in the upper bits.
            for (uint32_t x = threadIdx.x; x < nActive; x += blockDim.x) {
                const DContact& c = cs[act[x]];
                const bool can = !(c.flags & kCPlanar) && !(c.rollingResistance > 0.0f);
                B.cflags[cf + act[x]] = (B.cflags[cf + act[x]] & ~8) | (can ? 8 : 0);
            }
            __syncthreads();
        }
        // Bodies of pairs closing faster than the restitution threshold are struck (src/world.cpp:1029-1049).
        for (uint32_t x = threadIdx.x; x < nActive; x += blockDim.x) {
            const DContact& c = cs[act[x]];
            for (int i = 0; i < c.count; ++i) {
                if (c.points[i].relativeVelocity >= -P.restitutionThreshold) { continue; }
                if (B.bodies[c.bodyA].type == kDynamic) { B.struck[c.bodyA] = 1; }
                if (B.bodies[c.bodyB].type == kDynamic) { B.struck[c.bodyB] = 1; }
                break;
            }
        }
        if (threadIdx.x == 0) {
            if (staged) {
                colorSequential(nActive, endA, endB, colorable, masks, colorTmp);
            } else {
                for (uint32_t x = 0; x < nActive; ++x) {
                    uint8_t k = kNoColor;
                    if (B.cflags[cf + act[x]] & 8) {
                        const uint32_t a = endA[x], b = endB[x];
                        const uint32_t taken = (a != kNone ? masks[a] : 0u) | (b != kNone ? masks[b] : 0u);
                        if (taken != 0xffffffffu) {
                            const int f = __ffs(~taken) - 1;
                            if (a != kNone) { masks[a] |= 1u << f; }
                            if (b != kNone) { masks[b] |= 1u << f; }
                            k = (uint8_t)f;
                        }
                    }
                    colorTmp[x] = k;
                }
            }
        }
        __syncthreads();
        uint8_t* colorOf = B.color + cf;
        for (uint32_t x = threadIdx.x; x < nActive; x += blockDim.x) {
            const uint8_t k = colorTmp[x];
            colorOf[act[x]] = k;
            if (k != kNoColor) { cs[act[x]].flags |= kCLaned; }
        }
        __syncthreads();
        const uint32_t nImpact = blockCompact(
            nActive,
            [&](uint32_t x) {
                const DContact& c = cs[act[x]];
                return B.struck[c.bodyA] || B.struck[c.bodyB];
            },
            [&](uint32_t x, uint32_t pos) { B.impact[cf + pos] = act[x]; });
        bucketByColor(nActive, act, colorOf, B.colored + cf, B.rest + cf, wc.colorStart, wc.colorCount, wc.restCount);
        bucketByColor(nImpact, B.impact + cf, colorOf, B.impactColored + cf, B.impactRest + cf, wc.impactColorStart,
                      wc.impactColorCount, wc.impactRestCount);
        {
            __shared__ uint32_t s_points;
            if (threadIdx.x == 0) { s_points = 0; }
            __syncthreads();
            uint32_t mine = 0;
            for (uint32_t x = threadIdx.x; x < nActive; x += blockDim.x) { mine += (uint32_t)cs[act[x]].count; }
            atomicAdd(&s_points, mine);
            __syncthreads();
            if (threadIdx.x == 0) { wc.activePoints = s_points; }
        }
        if (threadIdx.x == 0) {
            wc.activeCount = nActive;
            wc.impactCount = nImpact;
            wc.fastCount = s_fast;
            wc.fastSolidCount = s_fastSolid;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------------------
// The substep (src/world.cpp:1658-1681).

// Calls f(contact index) for every contact of each color in turn, the colors apart by a block barrier.
template <class F>
__device__ void forEachColor(const uint32_t* list, const uint32_t* start, uint32_t colors, F f) {
    for (uint32_t k = 0; k < colors; ++k) {
        const uint32_t end = start[k + 1];
        for (uint32_t x = start[k] + threadIdx.x; x < end; x += blockDim.x) { f(list[x]); }
        __syncthreads();
    }
}

// In checked builds, whether contact ci of a world can be read: in the list, with bodies in the world.
__device__ __forceinline__ bool contactOk(const Batch& B, const WorldInfo& wi, const WorldCounts& wc,
                                          uint32_t ci, int code) {
#if defined(TF_DEVICE_CHECKS)
    if (!TF_OK_INDEX(B, ci < wc.contactCount, code, wi.bodyFirst, ci)) { return false; }
    const DContact& c = B.contacts[wi.contactFirst + ci];
    return TF_OK_INDEX(B, c.bodyA - wi.bodyFirst < wi.bodyCount && c.bodyB - wi.bodyFirst < wi.bodyCount &&
                              c.shapeA - wi.shapeFirst < wi.shapeCount && c.shapeB - wi.shapeFirst < wi.shapeCount &&
                              c.count >= 0 && c.count <= 4,
                       code + 1, wi.bodyFirst, ci);
#else
    return true;
#endif
}

// A fast pair collided again with the remaining time (src/world.cpp:1074-1138).
__device__ void refreshContact(const Batch& B, const StepParams& P, DContact& c, float remaining) {
    const DBody& a = B.bodies[c.bodyA];
    const DBody& b = B.bodies[c.bodyB];
    const DShape sa = B.shapes[c.shapeA];
    const DShape sb = B.shapes[c.shapeB];
    // Polyhedra that turned little against each other keep the edge pair they met on (src/world.cpp:1051-1055).
    const Quat now = conjugate(a.xf.q) * b.xf.q, then = conjugate(a.q0) * b.q0;
    const bool little = fabsf(dot(now, then)) >= P.featureTurnCos;
    Manifold m;
    collidePair(B, P, sa, sb, remaining, m, little ? c.featKind : kFeatNone, c.featA, c.featB);
    if (m.count == 0) {
        c.count = 0;
        return;
    }
    const DContact old = c;
    c.flags &= ~kCReusable;
    c.featKind = m.featKind;
    c.featA = m.featA;
    c.featB = m.featB;
    c.normal = m.normal;
    c.tangent1 = perpendicular(m.normal);
    c.tangent2 = cross(m.normal, c.tangent1);
    c.count = m.count;
    for (int i = 0; i < m.count; ++i) {
        DPoint& p = c.points[i];
        p = DPoint{};
        p.localA = applyInverse(a.xf, m.points[i].position);
        p.separation = m.points[i].separation;
        const Vec3 up = lift(a, b, m.normal, p.separation, P.tol.speculative);
        p.anchorA = m.points[i].position - up - a.com;
        p.anchorB = m.points[i].position + up - b.com;
    }
    prepareContact(a, b, c);
    for (int i = 0; i < c.count; ++i) {
        DPoint& p = c.points[i];
        const int k = nearestPoint(old, p.localA);
        if (k < 0) { continue; }
        p.relativeVelocity = old.points[k].relativeVelocity;
        p.maxNormalImpulse = old.points[k].maxNormalImpulse;
    }
    carryImpulses(old, c, P.tol.speculative * P.tol.speculative);
}

// The solver state of one body, as the substep keeps it in registers: what warm start, solve and
// restitution read and write. Field names match DBody so the same solver templates run on either.
struct SBody {
    Vec3 v, w, dp;
    Quat dq;
    Mat3 invMassWorld, invInertiaWorld;
    float invMass;
    uint32_t type, awake;
};

// What integrateVelocity reads and writes (src/world.cpp:1141-1151).
struct VelBody {
    uint32_t alive, type, awake;
    Vec3 v, w, force, torque;
    float gravityScale, invMass, linearDamping, angularDamping, kept;
    Mat3 linearProj, angularProj, invInertiaWorld;
};

// What integratePosition reads and writes (src/world.cpp:1161-1172).
struct PosBody {
    uint32_t alive, type, awake;
    Vec3 v, w, com, dp, localCenter;
    Quat dq, qBase;
    Transform xf;
    float kept;
};

constexpr int kSBodyWords = 33;

// Where one world's solver state lives during a substep: shared memory (structure of arrays, stride words
// apart) for worlds that fit, else the bodies in global memory.
struct SolverStore {
    float* s;
    uint32_t stride;
    bool staged;
    DBody* g;

    __device__ __forceinline__ float& at(int word, uint32_t i) const { return s[word * stride + i]; }

    __device__ SBody load(uint32_t i) const {
        SBody b;
        if (!staged) {
            const DBody& d = g[i];
            b.v = d.v;
            b.w = d.w;
            b.dp = d.dp;
            b.dq = d.dq;
            b.invMassWorld = d.invMassWorld;
            b.invInertiaWorld = d.invInertiaWorld;
            b.invMass = d.invMass;
            b.type = d.type;
            b.awake = d.awake;
            return b;
        }
        b.v = { at(0, i), at(1, i), at(2, i) };
        b.w = { at(3, i), at(4, i), at(5, i) };
        b.dp = { at(6, i), at(7, i), at(8, i) };
        b.dq = { at(9, i), at(10, i), at(11, i), at(12, i) };
        for (int r = 0; r < 3; ++r) {
            b.invMassWorld.r[r] = { at(13 + 3 * r, i), at(14 + 3 * r, i), at(15 + 3 * r, i) };
            b.invInertiaWorld.r[r] = { at(22 + 3 * r, i), at(23 + 3 * r, i), at(24 + 3 * r, i) };
        }
        b.invMass = at(31, i);
        const uint32_t f = __float_as_uint(at(32, i));
        b.type = f & 0xffu;
        b.awake = f >> 8;
        return b;
    }

    __device__ void storeVW(uint32_t i, const SBody& b) const {
        if (!staged) {
            g[i].v = b.v;
            g[i].w = b.w;
            return;
        }
        at(0, i) = b.v.x;
        at(1, i) = b.v.y;
        at(2, i) = b.v.z;
        at(3, i) = b.w.x;
        at(4, i) = b.w.y;
        at(5, i) = b.w.z;
    }

    // Copies a body's solver fields from global memory into the store.
    __device__ void stage(uint32_t i) const {
        const DBody& d = g[i];
        at(0, i) = d.v.x, at(1, i) = d.v.y, at(2, i) = d.v.z;
        at(3, i) = d.w.x, at(4, i) = d.w.y, at(5, i) = d.w.z;
        at(6, i) = d.dp.x, at(7, i) = d.dp.y, at(8, i) = d.dp.z;
        at(9, i) = d.dq.x, at(10, i) = d.dq.y, at(11, i) = d.dq.z, at(12, i) = d.dq.w;
        for (int r = 0; r < 3; ++r) {
            at(13 + 3 * r, i) = d.invMassWorld.r[r].x;
            at(14 + 3 * r, i) = d.invMassWorld.r[r].y;
            at(15 + 3 * r, i) = d.invMassWorld.r[r].z;
            at(22 + 3 * r, i) = d.invInertiaWorld.r[r].x;
            at(23 + 3 * r, i) = d.invInertiaWorld.r[r].y;
            at(24 + 3 * r, i) = d.invInertiaWorld.r[r].z;
        }
        at(31, i) = d.invMass;
        at(32, i) = __uint_as_float(d.type | (d.awake << 8));
    }

    // Writes the fields a substep changes back to global memory.
    __device__ void unstage(uint32_t i) const {
        DBody& d = g[i];
        d.v = { at(0, i), at(1, i), at(2, i) };
        d.w = { at(3, i), at(4, i), at(5, i) };
        d.dp = { at(6, i), at(7, i), at(8, i) };
        d.dq = { at(9, i), at(10, i), at(11, i), at(12, i) };
    }

    __device__ void integrateVelocityAt(uint32_t i, const StepParams& P) const {
        DBody& d = g[i];
        if (!d.alive || d.type != kDynamic || !d.awake) { return; }
        if (!staged) {
            integrateVelocity(d, P);
            return;
        }
        VelBody b;
        b.alive = d.alive;
        b.type = d.type;
        b.awake = d.awake;
        b.v = { at(0, i), at(1, i), at(2, i) };
        b.w = { at(3, i), at(4, i), at(5, i) };
        b.force = d.force;
        b.torque = d.torque;
        b.gravityScale = d.gravityScale;
        b.invMass = d.invMass;
        b.linearDamping = d.linearDamping;
        b.angularDamping = d.angularDamping;
        b.kept = d.kept;
        b.linearProj = d.linearProj;
        b.angularProj = d.angularProj;
        for (int r = 0; r < 3; ++r) {
            b.invInertiaWorld.r[r] = { at(22 + 3 * r, i), at(23 + 3 * r, i), at(24 + 3 * r, i) };
        }
        integrateVelocity(b, P);
        at(0, i) = b.v.x, at(1, i) = b.v.y, at(2, i) = b.v.z;
        at(3, i) = b.w.x, at(4, i) = b.w.y, at(5, i) = b.w.z;
        d.kept = b.kept;
    }

    __device__ void integratePositionAt(uint32_t i, const StepParams& P) const {
        DBody& d = g[i];
        if (!staged) {
            integratePosition(d, P);
            return;
        }
        PosBody b;
        b.alive = d.alive;
        b.type = d.type;
        b.awake = d.awake;
        b.v = { at(0, i), at(1, i), at(2, i) };
        b.w = { at(3, i), at(4, i), at(5, i) };
        b.dp = { at(6, i), at(7, i), at(8, i) };
        b.dq = { at(9, i), at(10, i), at(11, i), at(12, i) };
        b.com = d.com;
        b.localCenter = d.localCenter;
        b.qBase = d.qBase;
        b.xf = d.xf;
        b.kept = d.kept;
        integratePosition(b, P);
        at(0, i) = b.v.x, at(1, i) = b.v.y, at(2, i) = b.v.z;
        at(3, i) = b.w.x, at(4, i) = b.w.y, at(5, i) = b.w.z;
        at(6, i) = b.dp.x, at(7, i) = b.dp.y, at(8, i) = b.dp.z;
        at(9, i) = b.dq.x, at(10, i) = b.dq.y, at(11, i) = b.dq.z, at(12, i) = b.dq.w;
        d.com = b.com;
        d.xf = b.xf;
        d.kept = b.kept;
    }
};

// Fast pairs collided again before a substep (src/world.cpp:1658-1668): inverse mass refreshed, other
// contacts rebased, dp and dq reset, fast contacts collided with the time left. Does nothing in worlds
// without such pairs, so it can sit in a recorded graph before every substep but the first.
__global__ void __launch_bounds__(kMaxBlock) k_refresh(Batch B, StepParams P, int sub, int serial) {
    if (stepAborted(B, serial)) { return; }
    for (int o = blockIdx.x; o < B.nWorlds; o += gridDim.x) {
        const uint32_t w = B.order[o];
        const WorldInfo wi = B.info[w];
        WorldCounts& wc = B.counts[w];
        const int n = P.substeps;
        const uint8_t againFlag = sub == n / 2 ? kFlagFast : kFlagFastSolid;
        const uint32_t againCount = sub == n / 2 ? wc.fastCount : wc.fastSolidCount;
        if (!(sub > 0 && againCount > 0)) { continue; }
        const uint32_t cf = wi.contactFirst;
        DContact* cs = B.contacts + cf;
        const uint32_t nActive = wc.activeCount;
        const uint32_t* act = B.active + cf;
        for (uint32_t i = threadIdx.x; i < wi.bodyCount; i += blockDim.x) {
            DBody& b = B.bodies[wi.bodyFirst + i];
            if (b.alive && b.type == kDynamic && b.awake) { updateInverseMass(b); }
        }
        __syncthreads();
        for (uint32_t x = threadIdx.x; x < nActive; x += blockDim.x) {
            const uint32_t ci = act[x];
            if (B.cflags[cf + ci] & againFlag) { continue; }
            if (!contactOk(B, wi, wc, ci, 16)) { continue; }
            DContact& c = cs[ci];
            rebaseContact(B.bodies[c.bodyA], B.bodies[c.bodyB], c);
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < wi.bodyCount; i += blockDim.x) {
            DBody& b = B.bodies[wi.bodyFirst + i];
            b.dp = zero3();
            b.dq = qid();
            b.qBase = b.xf.q;
        }
        __syncthreads();
        const float remaining = (float)(n - sub) * P.h;
        for (uint32_t x = threadIdx.x; x < nActive; x += blockDim.x) {
            const uint32_t ci = act[x];
            if (!(B.cflags[cf + ci] & againFlag)) { continue; }
            if (!contactOk(B, wi, wc, ci, 14)) { continue; }
            refreshContact(B, P, cs[ci], remaining);
        }
        __syncthreads();
        // Every active contact's axes again, from the refreshed inertia and the new anchors.
        for (uint32_t x = threadIdx.x; x < nActive; x += blockDim.x) {
            const uint32_t ci = act[x];
            if (!contactOk(B, wi, wc, ci, 26)) { continue; }
            const DContact& c = cs[ci];
            makeContactAxes(B.bodies[c.bodyA], B.bodies[c.bodyB], c, B.axes + (size_t)(cf + ci) * kAxesPerContact);
        }
        __syncthreads();
    }
}

// Integrate velocities, warm start, biased solve, integrate positions, relax (src/world.cpp:1669-1680), with
// the world's bodies staged in shared memory when they fit (stageBodies of them).
__global__ void __launch_bounds__(kMaxBlock) k_substep(Batch B, StepParams P, uint32_t stageBodies, int serial) {
    extern __shared__ __align__(16) float s_bodies[];
    if (stepAborted(B, serial)) { return; }
    for (int o = blockIdx.x; o < B.nWorlds; o += gridDim.x) {
        const uint32_t w = B.order[o];
        const WorldInfo wi = B.info[w];
        const WorldCounts& wc = B.counts[w];
        const uint32_t cf = wi.contactFirst;
        DContact* cs = B.contacts + cf;
        const uint32_t nb = wi.bodyCount;
        const SolverStore st{ s_bodies, stageBodies, nb <= stageBodies, B.bodies + wi.bodyFirst };
        if (st.staged) {
            for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) { st.stage(i); }
            __syncthreads();
        }
        for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) { st.integrateVelocityAt(i, P); }
        __syncthreads();
        const uint32_t base = wi.bodyFirst;
        // A laned contact's bodies are stored only where they move, so a static body shared by a color's
        // contacts is never written concurrently; a contact solved on its own stores both, as the reference does.
        auto warm = [&](uint32_t ci, bool laned) {
            if (!contactOk(B, wi, wc, ci, 10)) { return; }
            const DContact& c = cs[ci];
            const uint32_t ia = c.bodyA - base, ib = c.bodyB - base;
            SBody a = st.load(ia), b = st.load(ib);
            warmStartContact(a, b, c, laned, B.axes + (size_t)(cf + ci) * kAxesPerContact);
            if (!laned || !anchored(a)) { st.storeVW(ia, a); }
            if (!laned || !anchored(b)) { st.storeVW(ib, b); }
        };
        auto solve = [&](uint32_t ci, bool bias, bool laned) {
            if (!contactOk(B, wi, wc, ci, 12)) { return; }
            DContact& c = cs[ci];
            const uint32_t ia = c.bodyA - base, ib = c.bodyB - base;
            SBody a = st.load(ia), b = st.load(ib);
            solveContact(a, b, c, P, bias, B.axes + (size_t)(cf + ci) * kAxesPerContact);
            if (!laned || !anchored(a)) { st.storeVW(ia, a); }
            if (!laned || !anchored(b)) { st.storeVW(ib, b); }
        };
        const uint32_t* colored = B.colored + cf;
        const uint32_t* rest = B.rest + cf;
        const uint32_t* icolored = B.impactColored + cf;
        const uint32_t* irest = B.impactRest + cf;
        forEachColor(colored, wc.colorStart, wc.colorCount, [&](uint32_t ci) { warm(ci, true); });
        if (threadIdx.x == 0) {
            for (uint32_t x = 0; x < wc.restCount; ++x) { warm(rest[x], false); }
        }
        __syncthreads();
        for (int pass = 0; pass < 2; ++pass) {
            const bool bias = pass == 0;
            forEachColor(colored, wc.colorStart, wc.colorCount, [&](uint32_t ci) { solve(ci, bias, true); });
            if (threadIdx.x == 0) {
                for (uint32_t x = 0; x < wc.restCount; ++x) { solve(rest[x], bias, false); }
            }
            __syncthreads();
            if (wc.impactCount > 0) {
                forEachColor(icolored, wc.impactColorStart, wc.impactColorCount,
                             [&](uint32_t ci) { solve(ci, bias, true); });
                if (threadIdx.x == 0) {
                    for (uint32_t x = 0; x < wc.impactRestCount; ++x) { solve(irest[x], bias, false); }
                }
                __syncthreads();
            }
            if (bias) {
                for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) { st.integratePositionAt(i, P); }
                __syncthreads();
            }
        }
        if (st.staged) {
            for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) { st.unstage(i); }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------------------------
// After the substeps (src/world.cpp:1682-1726).

__device__ __forceinline__ uint32_t findRoot(uint32_t* parent, uint32_t x) {
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x = parent[x];
    }
    return x;
}

__device__ __forceinline__ uint32_t rootOf(const uint32_t* parent, uint32_t x) {
    while (parent[x] != x) { x = parent[x]; }
    return x;
}

__global__ void __launch_bounds__(kMaxBlock) k_finish(Batch B, StepParams P, uint32_t stageBodies,
                                                      uint32_t stageContacts, int serial) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    __shared__ uint32_t s_awake, s_islands, s_sweep;
    if (stepAborted(B, serial)) { return; }
    for (int o = blockIdx.x; o < B.nWorlds; o += gridDim.x) {
        const uint32_t w = B.order[o];
        const WorldInfo wi = B.info[w];
        WorldCounts& wc = B.counts[w];
        const uint32_t cf = wi.contactFirst;
        DContact* cs = B.contacts + cf;
        if (threadIdx.x == 0) {
            s_awake = 0;
            s_islands = 0;
            s_sweep = 0;
        }
        // Restitution: colored contacts by color, then the rest in active order.
        forEachColor(B.colored + cf, wc.colorStart, wc.colorCount, [&](uint32_t ci) {
            if (!contactOk(B, wi, wc, ci, 18)) { return; }
            DContact& c = cs[ci];
            restituteContact(B.bodies[c.bodyA], B.bodies[c.bodyB], c, P, true, B.axes + (size_t)(cf + ci) * kAxesPerContact);
        });
        if (threadIdx.x == 0) {
            for (uint32_t x = 0; x < wc.restCount; ++x) {
                if (!contactOk(B, wi, wc, B.rest[cf + x], 20)) { continue; }
                DContact& c = cs[B.rest[cf + x]];
                restituteContact(B.bodies[c.bodyA], B.bodies[c.bodyB], c, P, false,
                                 B.axes + (size_t)(cf + B.rest[cf + x]) * kAxesPerContact);
            }
        }
        __syncthreads();
        const uint32_t nc = wc.contactCount;
        const bool staged = wi.bodyCount <= stageBodies && nc <= stageContacts;
        uint32_t* parent = staged ? reinterpret_cast<uint32_t*>(s_raw) : B.unionParent + wi.bodyFirst;
        uint32_t* islandTime = staged ? parent + stageBodies : reinterpret_cast<uint32_t*>(B.islandTime + wi.bodyFirst);
        uint32_t* uA = staged ? islandTime + stageBodies : B.mergeIdxA + cf;
        uint32_t* uB = staged ? uA + stageContacts : B.mergeIdxB + cf;
        const float threshold = P.sleepThreshold;
        for (uint32_t i = threadIdx.x; i < wi.bodyCount; i += blockDim.x) {
            const uint32_t g = wi.bodyFirst + i;
            DBody& b = B.bodies[g];
            parent[i] = i;
            islandTime[i] = __float_as_uint(FLT_MAX);
            if (!b.alive) { continue; }
            limitSpeed(b, P.maxLinearSpeed, P.maxAngularSpeed);
            b.force = zero3();
            b.torque = zero3();
            if (b.hasTarget) {
                b.xf = b.target;
                b.com = apply(b.xf, b.localCenter);
                b.hasTarget = 0;
            }
            if (b.type != kStatic && !(b.type == kDynamic && !b.awake)) {
                // Leaf refit over the new pose (src/world.cpp:1713-1718): shape bounds and the body's union.
                bool any = false;
                for (uint32_t x = 0; x < b.shapeCount; ++x) {
                    DShape& s = B.shapes[B.shapeList[b.shapeFirst + x]];
                    Vec3 lo, hi;
                    shapeBounds(s, B.cx.pt, b.xf * s.local, lo, hi);
                    s.lo = lo;
                    s.hi = hi;
                    if (s.kind == kHalfSpace) { continue; }
                    b.lo = any ? minVec(b.lo, lo) : lo;
                    b.hi = any ? maxVec(b.hi, hi) : hi;
                    any = true;
                }
                // Shapes that moved well past what the speculative contacts covered would be swept against
                // their surroundings (src/world.cpp:1260-1278). They are counted; the sweep is not run here.
                if (P.continuous && b.type == kDynamic && b.awake) {
                    const float moved = length(b.com - b.com0);
                    Quat d = normalize(b.xf.q * conjugate(b.q0));
                    if (d.w < 0.0f) { d = -d; }
                    const float sine = length(qvec(d));
                    const float angle = sine > 1.0e-7f ? 2.0f * atan2f(sine, d.w) : 0.0f;
                    for (uint32_t x = 0; x < b.shapeCount; ++x) {
                        const DShape& s = B.shapes[B.shapeList[b.shapeFirst + x]];
                        if (s.kind == kMesh || s.sensor) { continue; }
                        const float reach = length(s.local.p - b.localCenter) + s.extent;
                        const float travel = moved + angle * reach;
                        if (travel > b.expectedTravel && travel > b.expectedTravel + 0.5f * s.minExtent) {
                            atomicAdd(&s_sweep, 1u);
                        }
                    }
                }
            }
            // Sleep timers (src/world.cpp:1176-1185).
            if (b.type != kDynamic || !b.awake) { continue; }
            const float speed = maxf(length(b.v), length(b.w) * b.extent);
            if (!b.canSleep || speed > threshold) {
                b.sleepTime = 0.0f;
            } else {
                b.sleepTime += P.dt;
            }
            if (!(isfinite(b.v.x) && isfinite(b.v.y) && isfinite(b.v.z) && isfinite(b.xf.p.x) && isfinite(b.xf.p.y) &&
                  isfinite(b.xf.p.z))) {
                atomicOr(&wc.flags, kDevNonFinite);
            }
        }
        __syncthreads();
        // Islands over contacts with points (src/world.cpp:1187-1233). The roots are each component's lowest
        // body whatever order the unions run in, so only the unions themselves run on one thread.
        const uint32_t nu = blockCompact(
            nc,
            [&](uint32_t ci) {
                if (!contactOk(B, wi, wc, ci, 22)) { return false; }
                const DContact& c = cs[ci];
                if (c.count == 0) { return false; }
                DBody& a = B.bodies[c.bodyA];
                DBody& b = B.bodies[c.bodyB];
                const bool da = a.type == kDynamic && a.awake;
                const bool db = b.type == kDynamic && b.awake;
                if (da && db) { return true; }
                if (da && b.type == kKinematic && movingAwake(b)) {
                    a.sleepTime = 0.0f;
                } else if (db && a.type == kKinematic && movingAwake(a)) {
                    b.sleepTime = 0.0f;
                }
                return false;
            },
            [&](uint32_t ci, uint32_t pos) {
                uA[pos] = cs[ci].bodyA - wi.bodyFirst;
                uB[pos] = cs[ci].bodyB - wi.bodyFirst;
            });
        if (threadIdx.x == 0) {
            for (uint32_t x = 0; x < nu; ++x) {
                if (!TF_OK_INDEX(B, uA[x] < wi.bodyCount && uB[x] < wi.bodyCount, 24, w, x)) { continue; }
                const uint32_t ra = findRoot(parent, uA[x]), rb = findRoot(parent, uB[x]);
                if (ra != rb) { parent[ra > rb ? ra : rb] = ra < rb ? ra : rb; }
            }
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < wi.bodyCount; i += blockDim.x) {
            DBody& b = B.bodies[wi.bodyFirst + i];
            if (!b.alive || b.type != kDynamic || !b.awake) { continue; }
            const uint32_t r = rootOf(parent, i);
            b.island = r;
            atomicAdd(&s_awake, 1u);
            if (r == i) { atomicAdd(&s_islands, 1u); }
            atomicMin(&islandTime[r], __float_as_uint(b.sleepTime));
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < wi.bodyCount; i += blockDim.x) {
            DBody& b = B.bodies[wi.bodyFirst + i];
            if (!b.alive || b.type != kDynamic || !b.awake) { continue; }
            if (__uint_as_float(islandTime[rootOf(parent, i)]) < P.timeToSleep) { continue; }
            b.awake = 0;
            b.v = zero3();
            b.w = zero3();
            updateInverseMass(b);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            wc.awakeBodies = s_awake;
            wc.awakeIslands = s_islands;
            wc.bodySteps += s_awake;
            if (s_sweep > 0) {
                wc.sweepShapes += s_sweep;
                wc.flags |= kDevSweepSkipped;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------------------
// Host traffic of a running batch: per-step forces in, poses out.

// World::addForce / addTorque with wake = false on every body (src/world.cpp:2118-2142).
__global__ void k_add_forces(DBody* bodies, uint32_t n, const float* __restrict__ f, const float* __restrict__ t) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) { return; }
    DBody& b = bodies[i];
    if (!b.alive || b.type != kDynamic || !b.awake) { return; }
    if (f) { b.force += Vec3{ f[3 * i], f[3 * i + 1], f[3 * i + 2] }; }
    if (t) { b.torque += Vec3{ t[3 * i], t[3 * i + 1], t[3 * i + 2] }; }
}

__global__ void k_pack_poses(const DBody* bodies, uint32_t n, float* __restrict__ p, float* __restrict__ q) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) { return; }
    const Transform xf = bodies[i].xf;
    p[3 * i] = xf.p.x;
    p[3 * i + 1] = xf.p.y;
    p[3 * i + 2] = xf.p.z;
    q[4 * i] = xf.q.x;
    q[4 * i + 1] = xf.q.y;
    q[4 * i + 2] = xf.q.z;
    q[4 * i + 3] = xf.q.w;
}

}
