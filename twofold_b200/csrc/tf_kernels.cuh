// The step kernels. Each kernel walks whole worlds with thread groups: a group (one warp, or 64 to 512
// threads) steps one world at a time, and groups take worlds in largest-first order from a per-launch
// counter, so small worlds pack many to an SM and large ones get whole CTAs. Within a world a group's threads
// split bodies, candidates or one color's contacts, with a group barrier between dependent phases. Work that
// the reference does in one sequential pass whose result depends on order (graph coloring, union-find unions,
// the wake flood and contacts solved one at a time) runs on the group's first thread, in the reference's
// order, over shared memory when the world fits the group's slice and over L1/L2-cached scratch otherwise.
//
// Kernel sequence of one step (src/world.cpp:1564-1727):
//   k_broadphase   growth, body-pair and half-space candidates, sorted unique keys (world.cpp:752-870)
//   k_narrowphase  reuse or collide each candidate, carry impulses, merge       (world.cpp:872-993)
//   k_wake         wake sleeping bodies touched by moving ones                  (world.cpp:705-735)
//   k_prepare      step state, active/fast/impact lists, prepare, axes, colors   (world.cpp:1589-1657)
//   k_refresh      fast pairs collided again before substeps 2..n               (world.cpp:1658-1668)
//   k_substep      integrate, warm start, solve, integrate, relax               (world.cpp:1669-1680)
//   k_finish       restitution, limits, refit bounds, sweep test, sleep         (world.cpp:1682-1726)
#pragma once

#include "tf_batch.cuh"
#include "tf_continuous.cuh"
#include "tf_joint.cuh"
#include "tf_planar.cuh"
#include "tf_solver.cuh"
#include "tf_tape.h"

namespace tfb {

constexpr int kMaxBlock = 512;
constexpr int kMaxGroups = kMaxBlock / 32;
constexpr uint32_t kDevPairOverflow = 1u << 0, kDevContactOverflow = 1u << 1, kDevNonFinite = 1u << 2,
                   kDevTimeout = 1u << 3, kDevUnsupported = 1u << 4, kDevListOverflow = 1u << 6;

// Where each launch of a step takes its worlds from (one counter each, zeroed when the step starts).
// Up to kMaxSubsteps substeps per step.
constexpr int kMaxSubsteps = 32;
enum WorkSlot : int {
    kSlotBroad = 0, kSlotNarrow = 1, kSlotWake = 2, kSlotPrepare = 3,
    kSlotRefresh = 4,                            // + substep index
    kSlotSubstep = kSlotRefresh + kMaxSubsteps,  // + substep index
    kSlotFinish = kSlotSubstep + kMaxSubsteps,
    kSlotBroadFinish = kSlotFinish + 1,                  // the big worlds' half of the broadphase
    kSlotCandItems = kSlotBroadFinish + 1,               // + pair class: candidate items of that class
    kSlotFastItems = kSlotCandItems + kPairClasses,       // + pair class: fast contacts of that class; + kPairClasses:
                                                          // the other active contacts of refreshed worlds
    kSlotTape = kSlotFastItems + kPairClasses + 1,      // the recording kernel's world counter
    // The flat solve of batches of many worlds (k_substep_flat): each color's contacts over every world, the
    // impact colors' likewise, the most colors, impact colors and levels of one-at-a-time contacts any world
    // has, and the grid barrier.
    kSlotFlatColor = kSlotTape + 1,                    // + color: contacts of that color in all worlds
    kSlotFlatImpact = kSlotFlatColor + kColors,        // + color
    kSlotFlatMaxColors = kSlotFlatImpact + kColors,
    kSlotFlatMaxImpact = kSlotFlatMaxColors + 1,
    kSlotFlatMaxRestLevels = kSlotFlatMaxImpact + 1,
    kSlotFlatMaxImpactRestLevels = kSlotFlatMaxRestLevels + 1,
    kSlotFlatBarrier = kSlotFlatMaxImpactRestLevels + 1,  // arrivals, then barriers passed
    kSlotCount = kSlotFlatBarrier + 2
};

// A group of threads that steps one world at a time: one warp, several warps, or the whole CTA.
struct Group {
    uint32_t tid, size, id, count, lane, warp, warps;

    __device__ __forceinline__ void sync() const {
        if (count == 1) {
            __syncthreads();
        } else if (size == 32) {
            __syncwarp();
        } else {
            asm volatile("bar.sync %0, %1;" ::"r"(id + 1), "r"(size) : "memory");
        }
    }
    // A barrier (as sync) that also tells every thread whether p held on any thread of the group.
    __device__ __forceinline__ bool any(bool p) const {
        if (count == 1) { return __syncthreads_or(p) != 0; }
        if (size == 32) {
            __syncwarp();
            return __any_sync(0xffffffffu, p);
        }
        uint32_t r;
        asm volatile(
            "{\n\t.reg .pred in, out;\n\tsetp.ne.u32 in, %1, 0;\n\tbar.red.or.pred out, %2, %3, in;\n\t"
            "selp.u32 %0, 1, 0, out;\n\t}"
            : "=r"(r)
            : "r"((uint32_t)p), "r"(id + 1), "r"(size)
            : "memory");
        return r != 0;
    }
};

// blockDim.x is a multiple of size, size a multiple of 32, at most kMaxGroups groups.
__device__ __forceinline__ Group makeGroup(uint32_t size) {
    Group g;
    g.size = size;
    g.count = blockDim.x / size;
    g.id = threadIdx.x / size;
    g.tid = threadIdx.x % size;
    g.lane = threadIdx.x & 31;
    g.warp = g.tid >> 5;
    g.warps = size >> 5;
    return g;
}

// How a launch hands out worlds. A CTA takes worlds in largest-first order (B.order) and steps a world with
// more than bigBodies bodies with all its threads; once it draws a world at or under that size every later
// world is too, and its warps go on alone, a world each. Each mode has its own shared-memory staging
// capacity: the whole dynamic allocation for a CTA-sized group, an equal share per warp otherwise.
struct StageSizes {
    uint32_t bodies, contacts;
};
struct Split {
    uint32_t bigBodies;
    StageSizes big, small;
    uint32_t smemBytes;
};

__device__ __forceinline__ uint32_t grabWarp(uint32_t* counter) {
    uint32_t v = 0;
    if ((threadIdx.x & 31) == 0) { v = atomicAdd(counter, 1u); }
    return __shfl_sync(0xffffffffu, v, 0);
}

// Calls body(group, world, slice, stage sizes) for every world of the batch, each exactly once. The body has
// one call site, so it is inlined and reads the kernel's parameters in place.
template <class Body>
__device__ __forceinline__ void forWorlds(const Batch& B, int slotIndex, const Split& sp, unsigned char* smem,
                                          Body&& body) {
    __shared__ uint32_t s_world, s_big;
    const uint32_t nw = (uint32_t)B.nWorlds;
    uint32_t* counter = B.work + slotIndex;
    bool warpMode = false;
    for (;;) {
        uint32_t o;
        if (!warpMode) {
            if (threadIdx.x == 0) {
                const uint32_t t = atomicAdd(counter, 1u);
                s_world = t;
                s_big = (t < nw && B.info[B.order[t]].bodyCount > sp.bigBodies) ? 1u : 0u;
            }
            __syncthreads();
            o = s_world;
            const uint32_t big = s_big;
            __syncthreads();
            if (o >= nw) { return; }
            if (!big) {
                // Every later world is small too: from here on each warp takes worlds on its own.
                warpMode = true;
                if ((threadIdx.x >> 5) != 0) { o = grabWarp(counter); }
            }
        } else {
            o = grabWarp(counter);
        }
        if (o >= nw) { return; }
        const Group g = makeGroup(warpMode ? 32u : blockDim.x);
        unsigned char* slice = warpMode && smem ? smem + (size_t)g.id * (sp.smemBytes / g.count) : smem;
        body(g, B.order[o], slice, warpMode ? sp.small : sp.big);
    }
}

// Exclusive prefix sum over the group; every thread of the group calls it.
__device__ __forceinline__ uint32_t groupScan(const Group& g, uint32_t v, uint32_t& total) {
    __shared__ uint32_t sums[kMaxGroups][kMaxBlock / 32];
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if ((int)g.lane >= o) { x += y; }
    }
    if (g.warps == 1) {
        total = __shfl_sync(0xffffffffu, x, 31);
        return x - v;
    }
    if (g.lane == 31) { sums[g.id][g.warp] = x; }
    g.sync();
    if (g.warp == 0) {
        uint32_t s = g.lane < g.warps ? sums[g.id][g.lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if ((int)g.lane >= o) { s += y; }
        }
        if (g.lane < g.warps) { sums[g.id][g.lane] = s; }
    }
    g.sync();
    const uint32_t prefix = (g.warp > 0 ? sums[g.id][g.warp - 1] : 0u) + x - v;
    total = sums[g.id][g.warps - 1];
    g.sync();
    return prefix;
}

// Calls emit(i, position) for every i < n where pred(i) holds, positions dense and in index order. Ends with
// a group barrier, so everything emit wrote is visible to the whole group on return.
template <class Pred, class Emit>
__device__ uint32_t groupCompact(const Group& g, uint32_t n, Pred pred, Emit emit) {
    uint32_t base = 0;
    for (uint32_t start = 0; start < n; start += g.size) {
        const uint32_t i = start + g.tid;
        const bool f = i < n && pred(i);
        uint32_t tot;
        const uint32_t pos = groupScan(g, f ? 1u : 0u, tot);
        if (f) { emit(i, base + pos); }
        base += tot;
    }
    g.sync();
    return base;
}

// Calls emit(i, position, k) for k < count(i) of every i < n, positions dense and in (i, k) order. Ends with a
// group barrier.
template <class Count, class Emit>
__device__ uint32_t groupExpand(const Group& g, uint32_t n, Count count, Emit emit) {
    uint32_t base = 0;
    for (uint32_t start = 0; start < n; start += g.size) {
        const uint32_t i = start + g.tid;
        const uint32_t c = i < n ? count(i) : 0u;
        uint32_t tot;
        const uint32_t pos = groupScan(g, c, tot);
        for (uint32_t k = 0; k < c; ++k) { emit(i, base + pos + k, k); }
        base += tot;
    }
    g.sync();
    return base;
}

// Reads the abort word once per CTA at a kernel's start: true when an earlier step of this launch sequence
// overflowed a list, or this step did in an earlier kernel.
__device__ __forceinline__ bool stepAborted(const Batch& B, int serial) {
    __shared__ int s_skip;
    if (threadIdx.x == 0) { s_skip = *(volatile uint32_t*)B.abortStep <= (uint32_t)serial; }
    __syncthreads();
    const bool skip = s_skip != 0;
    __syncthreads();
    return skip;
}

// The flat list a pair of shapes (global indices) is collided from: the planar class when its bodies are
// solved in a plane (src/world.cpp:514), else the class of its shape kinds.
__device__ __forceinline__ int pairClassOf(const Batch& B, uint32_t a, uint32_t b) {
    const DShape& sa = B.shapes[a];
    const DShape& sb = B.shapes[b];
    if (sa.kind == kMesh || sb.kind == kMesh) { return kClassMesh; }
    Vec3 n;
    if (usePlanar(B.bodies[sa.body], B.bodies[sb.body], n)) { return kClassPlanar; }
    return pairClass(sa.kind, sb.kind);
}

__device__ __forceinline__ uint64_t pairKey(uint32_t a, uint32_t b) {
    return ((uint64_t)(a < b ? a : b) << 32) | (uint64_t)(a < b ? b : a);
}

__device__ __forceinline__ void emitCandidate(const Batch& B, const WorldInfo& wi, uint32_t* count, uint64_t key) {
    const uint32_t pos = atomicAdd(count, 1u);
    if (pos < wi.candCap) { B.cand[wi.candFirst + pos] = key; }
}

// ---------------------------------------------------------------------------------------------------------
// Joints outside the solve: the pairs they keep from colliding and the links they add for waking.

// Whether a joint that does not collide its bodies holds bodies ga and gb (src/world.cpp:375-388).
__device__ __forceinline__ bool joinedBodies(const Batch& B, const WorldInfo& wi, uint32_t ga, uint32_t gb) {
    if (wi.joinedCount == 0) { return false; }
    const uint32_t a = ga - wi.bodyFirst, b = gb - wi.bodyFirst;
    const uint64_t key = ((uint64_t)(a < b ? a : b) << 32) | (uint64_t)(a < b ? b : a);
    const uint64_t* keys = B.joined + wi.jointFirst;
    uint32_t l = 0, h = wi.joinedCount;
    while (l < h) {
        const uint32_t mid = (l + h) >> 1;
        if (keys[mid] < key) {
            l = mid + 1;
        } else {
            h = mid;
        }
    }
    return l < wi.joinedCount && keys[l] == key;
}

// Pushes onto a wake stack the sleeping dynamic bodies linked to body gb: by a pair whose contacts have points,
// or by a joint that holds and is not joined to the world (src/world.cpp:655-700). Marks what it pushes.
static __device__ void pushLinked(const Batch& B, const WorldInfo& wi, uint32_t gb, const DContact* cs, uint32_t nc,
                           uint32_t* stack, uint32_t& top) {
    for (uint32_t ci = 0; ci < nc; ++ci) {
        const DContact& c = cs[ci];
        if (c.bodyA != gb && c.bodyB != gb) { continue; }
        if (ci > 0 && cs[ci - 1].key == c.key) { continue; }  // one link per pair
        const uint32_t other = c.bodyA == gb ? c.bodyB : c.bodyA;
        const DBody& ob = B.bodies[other];
        if (ob.type != kDynamic || ob.awake || B.wakeMark[other]) { continue; }
        bool linked = false;
        for (uint32_t k = ci; k < nc && cs[k].key == c.key; ++k) { linked = linked || cs[k].count > 0; }
        if (linked && top < wi.bodyCount) {
            B.wakeMark[other] = 1;
            stack[top++] = other;
        }
    }
    const DJoint* js = B.joints + wi.jointFirst;
    for (uint32_t x = 0; x < wi.jointCount; ++x) {
        const DJoint& j = js[x];
        if (!j.alive || j.broken || j.bodyA == kWorldEnd || (j.bodyA != gb && j.bodyB != gb)) { continue; }
        const uint32_t other = j.bodyA == gb ? j.bodyB : j.bodyA;
        const DBody& ob = B.bodies[other];
        if (ob.type != kDynamic || ob.awake || B.wakeMark[other]) { continue; }
        if (top < wi.bodyCount) {
            B.wakeMark[other] = 1;
            stack[top++] = other;
        }
    }
}

// Wakes what a wake stack holds and everything linked to it (src/world.cpp:703-735).
static __device__ void wakeStack(const Batch& B, const WorldInfo& wi, const DContact* cs, uint32_t nc, uint32_t* stack,
                          uint32_t top) {
    while (top > 0) {
        const uint32_t gb = stack[--top];
        DBody& b = B.bodies[gb];
        B.wakeMark[gb] = 0;
        if (b.awake) { continue; }
        b.awake = 1;
        b.sleepTime = 0.0f;
        updateInverseMass(b);
        pushLinked(B, wi, gb, cs, nc, stack, top);
    }
}

// At the start of a step a joint pulls its sleeping dynamic end awake when the other end moves
// (src/world.cpp:1578-1585); runs on one thread, over the last step's contacts.
static __device__ void wakeJointPulled(const Batch& B, const WorldInfo& wi, const WorldCounts& wc) {
    uint32_t* stack = B.unionParent + wi.bodyFirst;
    uint32_t top = 0;
    const DJoint* js = B.joints + wi.jointFirst;
    auto moving = [&](uint32_t g) { return g != kWorldEnd && movingAwake(B.bodies[g]); };
    auto pull = [&](uint32_t g) {
        if (g == kWorldEnd) { return; }
        const DBody& b = B.bodies[g];
        if (b.alive && b.type == kDynamic && !b.awake && !B.wakeMark[g] && top < wi.bodyCount) {
            B.wakeMark[g] = 1;
            stack[top++] = g;
        }
    };
    for (uint32_t x = 0; x < wi.jointCount; ++x) {
        const DJoint& j = js[x];
        if (!j.alive || j.broken) { continue; }
        if (moving(j.bodyB)) { pull(j.bodyA); }
        if (moving(j.bodyA)) { pull(j.bodyB); }
    }
    wakeStack(B, wi, B.previous + wi.contactFirst, min(wc.contactCount, wi.contactCap), stack, top);
}

// ---------------------------------------------------------------------------------------------------------
// Broadphase (src/world.cpp:752-870).
// A half-space against one body's shapes (src/world.cpp:844-867).
static __device__ void pairPlane(const Batch& B, const WorldInfo& wi, uint32_t gp, uint32_t gb, uint32_t* count) {
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
        if (joinedBodies(B, wi, sp.body, s.body)) { continue; }
        emitCandidate(B, wi, count, pairKey(sp.index, s.index));
    }
}

// The shapes of two bodies whose grown bounds overlap, paired by their own grown bounds
// (src/world.cpp:819-842).
static __device__ void pairShapes(const Batch& B, const WorldInfo& wi, const DBody& ba, const DBody& bb, float gA, float gB,
                           const Vec3& loA, const Vec3& hiA, const Vec3& loB, const Vec3& hiB, const Vec3& reach,
                           uint32_t* count) {
    if (joinedBodies(B, wi, (uint32_t)(&ba - B.bodies), (uint32_t)(&bb - B.bodies))) { return; }
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

// Worlds with more bodies than this find their body pairs with a sweep along x over the whole grid instead of
// testing every pair on one group.
constexpr uint32_t kSweepBodies = 1024;

// Floats as unsigned keys in the same order, for atomicMin and atomicMax.
__device__ __forceinline__ uint32_t orderedKey(float f) {
    const uint32_t b = __float_as_uint(f);
    return b ^ ((b >> 31) ? 0xffffffffu : 0x80000000u);
}
__device__ __forceinline__ float fromOrderedKey(uint32_t k) {
    return __uint_as_float((k >> 31) ? (k ^ 0x80000000u) : ~k);
}

// How far a body's interval along x is widened beyond its grown bounds, so that two bodies the pair test
// accepts always have overlapping intervals whatever the rounding of the test's sums: a millimetre plus a
// millionth of the coordinate.
__device__ __forceinline__ float sweepSlack(float x) { return 1e-3f + 1e-6f * fabsf(x); }

// Buckets along x: a quarter as many as bodies, evenly over the range the intervals cover.
struct SweepGrid {
    float lo, scale;
    uint32_t buckets;
};

__device__ __forceinline__ SweepGrid sweepGrid(const WorldInfo& wi, const WorldCounts& wc) {
    SweepGrid s;
    s.buckets = wi.bodyCount / 4 + 1;
    s.lo = fromOrderedKey(wc.sweepMinKey);
    const float hi = fromOrderedKey(wc.sweepMaxKey);
    s.scale = hi > s.lo ? (float)s.buckets / (hi - s.lo) : 0.0f;
    return s;
}

__device__ __forceinline__ uint32_t sweepBucket(const SweepGrid& s, float x) {
    const float f = (x - s.lo) * s.scale;
    if (!(f > 0.0f)) { return 0u; }
    return f >= (float)(s.buckets - 1) ? s.buckets - 1 : (uint32_t)f;
}

// The first half of a big world's broadphase, after the growth: each live body's interval along x, their
// range, and the bodies counted into buckets by where their intervals start. Bucket b then holds
// sweepOrder[start[b - 1] .. start[b]), start[-1] being 0.
static __device__ void prepareSweep(const Batch& B, const Group& g, const WorldInfo& wi, WorldCounts& wc, uint32_t w) {
    const uint32_t n = wi.bodyCount;
    if (g.tid == 0) {
        wc.sweepMinKey = 0xffffffffu;
        wc.sweepMaxKey = 0u;
        wc.candRaw = 0;
    }
    g.sync();
    for (uint32_t i = g.tid; i < n; i += g.size) {
        const uint32_t gb = wi.bodyFirst + i;
        const DBody& b = B.bodies[gb];
        float lo = FLT_MAX, hi = -FLT_MAX;
        if (b.alive && b.hasBounds) {
            const float gr = B.grow[gb];
            lo = b.lo.x - gr - sweepSlack(b.lo.x);
            hi = b.hi.x + gr + sweepSlack(b.hi.x);
            atomicMin(&wc.sweepMinKey, orderedKey(lo));
            atomicMax(&wc.sweepMaxKey, orderedKey(hi));
        }
        B.sweepLo[gb] = lo;
        B.sweepHi[gb] = hi;
    }
    g.sync();
    const SweepGrid grid = sweepGrid(wi, wc);
    uint32_t* start = B.sweepStart + wi.bodyFirst + w;
    for (uint32_t k = g.tid; k < grid.buckets; k += g.size) { start[k] = 0; }
    g.sync();
    for (uint32_t i = g.tid; i < n; i += g.size) { atomicAdd(&start[sweepBucket(grid, B.sweepLo[wi.bodyFirst + i])], 1u); }
    g.sync();
    uint32_t base = 0;
    for (uint32_t first = 0; first < grid.buckets; first += g.size) {
        const uint32_t k = first + g.tid;
        const uint32_t v = k < grid.buckets ? start[k] : 0u;
        uint32_t tot;
        const uint32_t pre = groupScan(g, v, tot);
        if (k < grid.buckets) { start[k] = base + pre; }
        base += tot;
    }
    g.sync();
    // Scattering advances each bucket's start to its end.
    for (uint32_t i = g.tid; i < n; i += g.size) {
        const uint32_t k = sweepBucket(grid, B.sweepLo[wi.bodyFirst + i]);
        B.sweepOrder[wi.bodyFirst + atomicAdd(&start[k], 1u)] = i;
    }
    g.sync();
    // The records in bucket order, so a scan over neighbouring buckets reads one contiguous run.
    for (uint32_t q = g.tid; q < n; q += g.size) {
        const uint32_t i = B.sweepOrder[wi.bodyFirst + q];
        const PairBody p = pairBodyOf(B, wi.bodyFirst + i);
        B.sweepRecs[wi.bodyFirst + q] = SweepRec{ p.lo, p.hi, p.grow, p.flags, B.sweepLo[wi.bodyFirst + i], i };
    }
    g.sync();
}

// Sorts the world's count keys (minShape << 32 | maxShape, at B.cand) ascending and removes repeats: a
// counting sort by the first shape, then each row sorted on its own (rows are short), then compaction back
// into B.cand. Returns the unique count.
constexpr uint32_t kShortRow = 48;  // rows of keys at most this long are sorted by one thread

static __device__ uint32_t sortKeys(const Group& g, const Batch& B, const WorldInfo& wi, uint32_t count) {
    uint32_t* row = B.rowScratch + wi.shapeFirst;
    uint64_t* tmp = B.mergeKeyA + wi.contactFirst;
    uint64_t* keys = B.cand + wi.candFirst;
    const uint32_t rows = wi.shapeCount;
    for (uint32_t r = g.tid; r < rows; r += g.size) { row[r] = 0; }
    g.sync();
    for (uint32_t i = g.tid; i < count; i += g.size) { atomicAdd(&row[(uint32_t)(keys[i] >> 32)], 1u); }
    g.sync();
    uint32_t base = 0;
    for (uint32_t start = 0; start < rows; start += g.size) {
        const uint32_t r = start + g.tid;
        const uint32_t v = r < rows ? row[r] : 0u;
        uint32_t tot;
        const uint32_t pre = groupScan(g, v, tot);
        if (r < rows) { row[r] = base + pre; }
        base += tot;
    }
    g.sync();
    // Scattering advances each row's start to its end.
    for (uint32_t i = g.tid; i < count; i += g.size) {
        const uint64_t k = keys[i];
        tmp[atomicAdd(&row[(uint32_t)(k >> 32)], 1u)] = k;
    }
    g.sync();
    // Short rows: one thread each, by insertion.
    for (uint32_t r = g.tid; r < rows; r += g.size) {
        const uint32_t s = r > 0 ? row[r - 1] : 0u, e = row[r];
        if (e - s > kShortRow) { continue; }
        for (uint32_t i = s + 1; i < e; ++i) {
            const uint64_t k = tmp[i];
            uint32_t j = i;
            while (j > s && tmp[j - 1] > k) {
                tmp[j] = tmp[j - 1];
                --j;
            }
            tmp[j] = k;
        }
    }
    // Long rows (a half-space's or a mesh's pairs): one at a time by the whole group, counted by the second
    // shape. Equal keys may land in any order among themselves, which leaves the same sequence.
    uint32_t* longRows = B.rowLong + wi.shapeFirst;
    const uint32_t nLong = groupCompact(
        g, rows, [&](uint32_t r) { return row[r] - (r > 0 ? row[r - 1] : 0u) > kShortRow; },
        [&](uint32_t r, uint32_t pos) { longRows[pos] = r; });
    uint32_t* hist = B.rowCount + wi.shapeFirst;
    for (uint32_t x = 0; x < nLong; ++x) {
        const uint32_t r = longRows[x];
        const uint32_t s = r > 0 ? row[r - 1] : 0u, e = row[r];
        for (uint32_t c = g.tid; c < rows; c += g.size) { hist[c] = 0; }
        g.sync();
        for (uint32_t i = s + g.tid; i < e; i += g.size) { atomicAdd(&hist[(uint32_t)tmp[i]], 1u); }
        g.sync();
        uint32_t base = s;
        for (uint32_t first = 0; first < rows; first += g.size) {
            const uint32_t c = first + g.tid;
            const uint32_t v = c < rows ? hist[c] : 0u;
            uint32_t tot;
            const uint32_t pre = groupScan(g, v, tot);
            if (c < rows) { hist[c] = base + pre; }
            base += tot;
        }
        g.sync();
        for (uint32_t i = s + g.tid; i < e; i += g.size) {
            const uint64_t k = tmp[i];
            keys[atomicAdd(&hist[(uint32_t)k], 1u)] = k;
        }
        g.sync();
        for (uint32_t i = s + g.tid; i < e; i += g.size) { tmp[i] = keys[i]; }
        g.sync();
    }
    g.sync();
    return groupCompact(
        g, count, [&](uint32_t i) { return i == 0 || tmp[i] != tmp[i - 1]; }, [&](uint32_t i, uint32_t pos) { keys[pos] = tmp[i]; });
}

// Body pairs whose grown bounds overlap, then their shapes (src/world.cpp:788-842), and half-space pairs
// (:844-867); the keys are sorted and made unique (:868-869). A warp of the group takes one body and its
// lanes the bodies after it. Bodies are staged in the group's shared slice when at most stageN of them.
static __device__ void finishCandidates(const Batch& B, const Group& g, const WorldInfo& wi, WorldCounts& wc, uint32_t w,
                                 uint32_t total, int serial, uint32_t* cls, uint32_t* classBase);

template <int Unused = 0>
__global__ void __launch_bounds__(kMaxBlock) k_broadphase(const __grid_constant__ Batch B, const __grid_constant__ StepParams P, const __grid_constant__ Split sp, int serial) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    __shared__ uint32_t s_count[kMaxGroups];
    __shared__ uint32_t s_class[kMaxGroups][kPairClasses], s_classBase[kMaxGroups][kPairClasses];
    if (stepAborted(B, serial)) { return; }
    forWorlds(B, kSlotBroad, sp, s_raw, [&](const Group& g, uint32_t w, unsigned char* slice, const StageSizes& ss) {
        PairBody* staged = reinterpret_cast<PairBody*>(slice);
        const uint32_t stageN = ss.bodies;
        const WorldInfo wi = B.info[w];
        WorldCounts& wc = B.counts[w];
        const uint32_t n = wi.bodyCount;
        const bool useStage = n <= stageN;
        if (wi.jointCount > 0) {
            if (g.tid == 0) { wakeJointPulled(B, wi, wc); }
            g.sync();
        }
        if (g.tid == 0) { s_count[g.id] = 0; }
        // Growth by the speculative distance and the travel over the step (src/world.cpp:754-765).
        for (uint32_t i = g.tid; i < n; i += g.size) {
            const DBody& b = B.bodies[wi.bodyFirst + i];
            float gr = P.tol.speculative;
            if (b.alive && b.type != kStatic && !(lengthSquared(b.v) == 0.0f && lengthSquared(b.w) == 0.0f)) {
                gr += (length(b.v) + length(b.w) * b.extent) * P.dt;
            }
            B.grow[wi.bodyFirst + i] = gr;
            if (useStage) {
                PairBody p;
                p.lo = b.lo;
                p.hi = b.hi;
                p.grow = gr;
                p.flags = ((b.alive && b.hasBounds) ? kBodyLive : 0u) | (b.type == kDynamic ? kBodyDynamic : 0u) |
                          (movingAwake(b) ? kBodyMoving : 0u);
                staged[i] = p;
            }
        }
        g.sync();
        if (n > kSweepBodies) {
            prepareSweep(B, g, wi, wc, w);
            return;
        }
        uint32_t* count = &s_count[g.id];
        for (uint32_t a = g.warp; a + 1 < n; a += g.warps) {
            const PairBody A = useStage ? staged[a] : pairBodyOf(B, wi.bodyFirst + a);
            if (!(A.flags & kBodyLive)) { continue; }
            for (uint32_t b = a + 1 + g.lane; b < n; b += 32) {
                const PairBody Bb = useStage ? staged[b] : pairBodyOf(B, wi.bodyFirst + b);
                if (!(Bb.flags & kBodyLive)) { continue; }
                if (!((A.flags | Bb.flags) & kBodyDynamic)) { continue; }
                if (!((A.flags | Bb.flags) & kBodyMoving)) { continue; }
                const float gg = A.grow + Bb.grow;
                const Vec3 reach{ gg, gg, gg };
                if (!boxesOverlap(A.lo - reach, A.hi + reach, Bb.lo, Bb.hi)) { continue; }
                pairShapes(B, wi, B.bodies[wi.bodyFirst + a], B.bodies[wi.bodyFirst + b], A.grow, Bb.grow, A.lo, A.hi,
                           Bb.lo, Bb.hi, reach, count);
            }
        }
        for (uint32_t pl = 0; pl < wi.planeCount; ++pl) {
            const uint32_t gp = B.planeList[wi.planeFirst + pl];
            for (uint32_t b = g.tid; b < n; b += g.size) { pairPlane(B, wi, gp, wi.bodyFirst + b, count); }
        }
        g.sync();
        finishCandidates(B, g, wi, wc, w, *count, serial, s_class[g.id], s_classBase[g.id]);
    });
}

// The end of a world's broadphase: the raw keys sorted and made unique (src/world.cpp:868-869), then the
// pairs join the flat list of their class: counted per class, a block of each list reserved for the
// world, then scattered into it. A list that did not fit stops this step, and the host grows it.
static __device__ void finishCandidates(const Batch& B, const Group& g, const WorldInfo& wi, WorldCounts& wc, uint32_t w,
                                 uint32_t total, int serial, uint32_t* cls, uint32_t* classBase) {
    {
        if (total > wi.candCap) {
            // The list did not fit: this step stops here and the host grows the world's lists.
            if (g.tid == 0) {
                wc.flags |= kDevPairOverflow;
                wc.candNeeded = max(wc.candNeeded, total);
                atomicMin(B.abortStep, (uint32_t)serial);
            }
            g.sync();
            return;
        }
        const uint32_t unique = sortKeys(g, B, wi, total);
        if (g.tid == 0) {
            wc.candCount = unique;
            wc.candNeeded = max(wc.candNeeded, total);
            wc.partCount = 0;
            wc.boundsCount = 0;
        }
        if (g.tid < kPairClasses) { cls[g.tid] = 0; }
        g.sync();
        auto classOf = [&](uint32_t i) {
            const uint64_t key = B.cand[wi.candFirst + i];
            return pairClassOf(B, wi.shapeFirst + (uint32_t)(key >> 32), wi.shapeFirst + (uint32_t)(key & 0xffffffffu));
        };
        for (uint32_t i = g.tid; i < unique; i += g.size) { atomicAdd(&cls[classOf(i)], 1u); }
        g.sync();
        if (g.tid < kPairClasses) {
            classBase[g.tid] = atomicAdd(B.work + kSlotCandItems + g.tid, cls[g.tid]);
            cls[g.tid] = 0;
        }
        g.sync();
        for (uint32_t i = g.tid; i < unique; i += g.size) {
            const int c = classOf(i);
            const uint32_t pos = classBase[c] + atomicAdd(&cls[c], 1u);
            B.candItems[(size_t)c * B.candItemStride + pos] = make_uint2(w, i);
        }
        g.sync();
    }
}

// The pair half of a big world's broadphase: each body takes the bodies whose intervals along x start
// within its own interval (the one starting first takes a pair, so each pair is taken once) and applies the
// same pair test as the small worlds, in the pair's lower-body-first order. A warp per body, its lanes
// across the contiguous run of records in the buckets its interval covers, over every big world.
template <int Unused = 0>
__global__ void __launch_bounds__(256) k_broad_pairs(const __grid_constant__ Batch B, int serial) {
    if (stepAborted(B, serial)) { return; }
    const uint32_t total = B.bigBodyStart[B.nBigWorlds];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; item < total; item += warps) {
        uint32_t k = 0;
        while (k + 1 < B.nBigWorlds && B.bigBodyStart[k + 1] <= item) { ++k; }
        const uint32_t w = B.bigWorlds[k];
        const WorldInfo wi = B.info[w];
        WorldCounts& wc = B.counts[w];
        const SweepRec* recs = B.sweepRecs + wi.bodyFirst;
        const uint32_t* start = B.sweepStart + wi.bodyFirst + w;
        const SweepRec ri = recs[item - B.bigBodyStart[k]];
        if (!(ri.flags & kBodyLive)) { continue; }
        const float lo = ri.start, hi = B.sweepHi[wi.bodyFirst + ri.body];
        const SweepGrid grid = sweepGrid(wi, wc);
        const uint32_t b0 = sweepBucket(grid, lo), b1 = sweepBucket(grid, hi);
        const uint32_t q0 = b0 ? start[b0 - 1] : 0u, q1 = start[b1];
        for (uint32_t q = q0 + lane; q < q1; q += 32) {
            const SweepRec rj = recs[q];
            const uint32_t i = ri.body, j = rj.body;
            if (j == i || !(rj.start > lo || (rj.start == lo && j > i)) || rj.start > hi) { continue; }
            const SweepRec& A = i < j ? ri : rj;
            const SweepRec& Bb = i < j ? rj : ri;
            if (!(A.flags & kBodyLive) || !(Bb.flags & kBodyLive)) { continue; }
            if (!((A.flags | Bb.flags) & kBodyDynamic)) { continue; }
            if (!((A.flags | Bb.flags) & kBodyMoving)) { continue; }
            const float gg = A.grow + Bb.grow;
            const Vec3 reach{ gg, gg, gg };
            if (!boxesOverlap(A.lo - reach, A.hi + reach, Bb.lo, Bb.hi)) { continue; }
            pairShapes(B, wi, B.bodies[wi.bodyFirst + A.body], B.bodies[wi.bodyFirst + Bb.body], A.grow, Bb.grow, A.lo,
                       A.hi, Bb.lo, Bb.hi, reach, &wc.candRaw);
        }
    }
}

// The rest of a big world's broadphase: half-space pairs, then the keys sorted and sent to their lists.
template <int Unused = 0>
__global__ void __launch_bounds__(kMaxBlock) k_broad_finish(const __grid_constant__ Batch B, const __grid_constant__ Split sp, int serial) {
    __shared__ uint32_t s_class[kMaxGroups][kPairClasses], s_classBase[kMaxGroups][kPairClasses];
    if (stepAborted(B, serial)) { return; }
    forWorlds(B, kSlotBroadFinish, sp, nullptr, [&](const Group& g, uint32_t w, unsigned char*, const StageSizes&) {
        const WorldInfo wi = B.info[w];
        if (wi.bodyCount <= kSweepBodies) { return; }
        WorldCounts& wc = B.counts[w];
        for (uint32_t pl = 0; pl < wi.planeCount; ++pl) {
            const uint32_t gp = B.planeList[wi.planeFirst + pl];
            for (uint32_t b = g.tid; b < wi.bodyCount; b += g.size) { pairPlane(B, wi, gp, wi.bodyFirst + b, &wc.candRaw); }
        }
        g.sync();
        const uint32_t total = *(volatile uint32_t*)&wc.candRaw;
        finishCandidates(B, g, wi, wc, w, total, serial, s_class[g.id], s_classBase[g.id]);
    });
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
static __device__ void measureAgain(const DBody& a, const DBody& b, DContact& c, const StepParams& P) {
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
static __device__ void carryImpulses(const DContact& old, DContact& c, float matchSq) {
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

// A pair whose dynamic bodies are locked to the plane n (src/world.cpp:514-518): both bodies are placed in
// the plane, whatever the profiles turn out to be, and marked so the round's placements are kept once every
// pair is done. Returns collidePlanar's answer. Kept out of line: the 3D paths around it need its registers.
static __device__ __noinline__ int collidePlanarPair(const Batch& B, const StepParams& P, const DShape& sa, const DShape& sb,
                                              const Vec3& n, float margin, Manifold& m) {
    DBody& ba = B.bodies[sa.body];
    DBody& bb = B.bodies[sb.body];
    const PlanePose pa = placeInPlane(ba, n);
    const PlanePose pb = placeInPlane(bb, n);
    ba.posePending = 1;
    bb.posePending = 1;
    m.featKind = kFeatNone;
    m.featA = m.featB = -1;
    m.normal = zero3();
    return collidePlanar(B.cx.pt, sa, pa, sb, pb, margin, P.tol.linearSlop, m);
}

// Stores the placements of the round of collisions that just ended for the bodies of one world that were
// placed in it; nothing reads a body's pose while its world is here.
static __device__ void keepPlacements(const Batch& B, const Group& g, const WorldInfo& wi) {
    if (wi.planeBody == UINT32_MAX) { return; }
    if (!TF_OK_INDEX(B, wi.planeBody < B.totalBodies, 31, wi.bodyFirst, wi.planeBody)) { return; }
    const Vec3 n = planeNormal(B.bodies[wi.planeBody]);
    for (uint32_t i = g.tid; i < wi.bodyCount; i += g.size) {
        DBody& b = B.bodies[wi.bodyFirst + i];
        if (!b.posePending) { continue; }
        keepPose(b, placeInPlane(b, n));
        b.posePending = 0;
    }
}

// Collides one shape pair over dt as Impl::collidePair does for non-mesh pairs (src/world.cpp:505-533).
// Returns false for a pair this build cannot collide.
template <int Cls = kClassAny>
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
    if constexpr (Cls == kClassAny || Cls == kClassPlanar) {
        Vec3 n;
        if (sa.kind != kMesh && sb.kind != kMesh && usePlanar(ba, bb, n)) {
            const int r = collidePlanarPair(B, P, sa, sb, n, margin, m);
            if (r > 0) { return true; }
            if (r < 0) {
                m.count = 0;
                return false;
            }
        }
    }
    const Transform xa = ba.xf * sa.local;
    const Transform xb = bb.xf * sb.local;
    const Motion mo{ ba.v, ba.w, ba.com, bb.v, bb.w, bb.com, dt, travel > P.tol.speculative };
    constexpr int Shapes = Cls == kClassPlanar ? kClassAny : Cls;
    return collideShapes<Shapes>(B.cx, sa, xa, sb, xb, margin, mo, m, reuseKind, reuseA, reuseB);
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
template <int Cls = kClassAny>
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
        out.boundsFirst = out.boundsCount = 0;
        used = 1;
    } else {
        Manifold m;
        if (!collidePair<Cls>(B, P, sa, sb, P.dt, m, kFeatNone, -1, -1)) { atomicOr(&wc.flags, kDevUnsupported); }
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
            c.boundsFirst = c.boundsCount = 0;
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

// A pair with a mesh over dt (src/world.cpp:505-533): manifolds with normals from sa to sb, into out. Warp: the
// warp's lanes collide the triangles together (collideMeshWarp, warpFound its shared room); else one thread.
template <bool Warp>
static __device__ int collideMeshPair(const Batch& B, const StepParams& P, const DShape& sa, const DShape& sb, float dt,
                               Manifold* out, int& outCount, MeshBounds* bounds, Manifold* warpFound = nullptr,
                               uint32_t lane = 0) {
    const DBody& ba = B.bodies[sa.body];
    const DBody& bb = B.bodies[sb.body];
    const float travel = relativeTravel(ba, bb, dt);
    const float margin = P.tol.speculative + travel;
    const Transform xa = ba.xf * sa.local;
    const Transform xb = bb.xf * sb.local;
    const Motion mo{ ba.v, ba.w, ba.com, bb.v, bb.w, bb.com, dt, travel > P.tol.speculative };
    const bool meshFirst = sa.kind == kMesh;
    const DShape& mesh = meshFirst ? sa : sb;
    const DShape& other = meshFirst ? sb : sa;
    const Transform& xm = meshFirst ? xa : xb;
    const Transform& xo = meshFirst ? xb : xa;
    const Motion m = meshFirst ? mo : mo.swapped();
    int status;
    if constexpr (Warp) {
        status = collideMeshWarp(B.cx, mesh, xm, other, xo, margin, m, out, outCount, bounds, warpFound, lane);
    } else {
        status = collideMesh(B.cx, mesh, xm, other, xo, margin, m, out, outCount, bounds);
    }
    if (!meshFirst) {
        for (int i = 0; i < outCount; ++i) { out[i].normal = -out[i].normal; }
    }
    return status;
}

// A warp's shared room for one mesh pair: its triangle manifolds and the triangles it rules out. The mesh pair
// kernels run 4 warps to a CTA.
struct MeshWarpRoom {
    Manifold found[kMaxMeshFound];
    TriangleBound ruled[kMaxMeshBounds];
};
constexpr int kMeshWarps = 4;

// A contact of pair (sa, sb) from one manifold (src/world.cpp:912-939): points on both surfaces, anchors,
// tangents and the reuse record.
static __device__ void contactFromManifold(const StepParams& P, const DBody& ba, const DBody& bb, const Manifold& m, DContact& c) {
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
    c.localNormal = unrotate(ba.xf.q, c.normal);
    c.baseOffset = unrotate(ba.xf.q, bb.com - ba.com);
    c.baseTurn = conjugate(ba.xf.q) * bb.xf.q;
    c.flags |= kCReusable;
}

// Stops this step (the host grows the world's lists and runs it again) when a mesh pair's parts or triangle
// bounds do not fit the world's room for them.
static __device__ void meshRoomOverflow(const Batch& B, const WorldInfo& wi, WorldCounts& wc, int serial) {
    atomicOr(&wc.flags, kDevPairOverflow);
    atomicMax(&wc.candNeeded, 2 * wi.candCap);
    atomicMin(B.abortStep, (uint32_t)serial);
}

// One mesh candidate (src/world.cpp:883-959): the old contacts kept and measured again when the pair barely
// moved, else one contact per manifold the mesh collision makes, each carrying the impulses of the old
// contact whose normal is closest. The first contact goes to the candidate's staging slot, the others to
// the world's extra parts. A fast pair records the triangles it ruled out, for the refresh within the step.
// Warp: every lane of the warp calls it alike with the warp's room; the lanes collide the triangles together and
// lane 0 writes the results.
template <bool Warp>
static __device__ void narrowMesh(const Batch& B, const StepParams& P, const WorldInfo& wi, WorldCounts& wc, uint32_t i,
                           const DContact* old, uint32_t oldCount, int serial, MeshWarpRoom* room = nullptr,
                           uint32_t lane = 0) {
    const bool lead = !Warp || lane == 0;
    if (lead) { B.stageUsed[wi.candFirst + i] = 0; }
    const uint64_t key = B.cand[wi.candFirst + i];
    const uint32_t ia = (uint32_t)(key >> 32), ib = (uint32_t)(key & 0xffffffffu);
    if (!TF_OK_INDEX(B, ia < wi.shapeCount && ib < wi.shapeCount, 34, wi.bodyFirst, ia)) { return; }
    const uint32_t gsa = wi.shapeFirst + ia, gsb = wi.shapeFirst + ib;
    const DShape sa = B.shapes[gsa];
    const DShape sb = B.shapes[gsb];
    if (!TF_OK_INDEX(B, oldCount <= wi.contactCap, 35, wi.bodyFirst, oldCount)) { return; }
    const DBody& ba = B.bodies[sa.body];
    const DBody& bb = B.bodies[sb.body];
    const uint32_t lo = lowerKey(old, oldCount, key);
    uint32_t hi = lo;
    while (hi < oldCount && old[hi].key == key) { ++hi; }
    const bool hasOld = lo < hi;
    bool keep = hasOld;
    for (uint32_t it = lo; it < hi && keep; ++it) { keep = stillFits(old[it], ba, bb, P); }
    const bool touched = hasOld && (old[lo].flags & kCTouched);

    Manifold found[kMaxMeshParts];
    int n = 0;
    uint32_t boundsFirst = 0, boundsCount = 0;
    if (keep) {
        if (!lead) { return; }
        n = (int)(hi - lo);
        if (n > kMaxMeshParts) {
            atomicOr(&wc.flags, kDevUnsupported);
            return;
        }
    } else {
        const bool record = relativeTravel(ba, bb, P.dt) > P.tol.speculative;
        TriangleBound own[Warp ? 1 : kMaxMeshBounds];
        TriangleBound* ruled = Warp ? room->ruled : own;
        MeshBounds mb{ record ? ruled : nullptr, 0, nullptr, 0, 0.0f };
        const int status = collideMeshPair<Warp>(B, P, sa, sb, P.dt, found, n, &mb, Warp ? room->found : nullptr, lane);
        if (!lead) { return; }
        if (status != kMeshOk) {
            atomicOr(&wc.flags, kDevUnsupported);
            return;
        }
        if (mb.foundCount > 0) {
            // By triangle, as the reference sorts each pair's run.
            for (int x = 1; x < mb.foundCount; ++x) {
                const TriangleBound t = ruled[x];
                int y = x - 1;
                while (y >= 0 && ruled[y].triangle > t.triangle) {
                    ruled[y + 1] = ruled[y];
                    --y;
                }
                ruled[y + 1] = t;
            }
            boundsFirst = atomicAdd(&wc.boundsCount, (uint32_t)mb.foundCount);
            boundsCount = (uint32_t)mb.foundCount;
            if (boundsFirst + boundsCount > wi.boundsCap) {
                meshRoomOverflow(B, wi, wc, serial);
                return;
            }
            for (int x = 0; x < mb.foundCount; ++x) { B.triBounds[wi.boundsFirst + boundsFirst + x] = ruled[x]; }
        }
    }
    if (n == 0) { return; }
    uint32_t extra = 0;
    if (n > 1) {
        extra = atomicAdd(&wc.partCount, (uint32_t)(n - 1));
        if (extra + (uint32_t)(n - 1) > wi.partCap) {
            meshRoomOverflow(B, wi, wc, serial);
            return;
        }
    }
    for (int k = 0; k < n; ++k) {
        DContact& out = k == 0 ? B.stage[wi.candFirst + i] : B.stageExtra[wi.partFirst + extra + (uint32_t)(k - 1)];
        if (keep) {
            out = old[lo + (uint32_t)k];
            measureAgain(ba, bb, out, P);
            out.boundsFirst = out.boundsCount = 0;
        } else {
            DContact c{};
            c.key = key;
            c.part = (uint32_t)k;
            c.shapeA = gsa;
            c.shapeB = gsb;
            c.bodyA = sa.body;
            c.bodyB = sb.body;
            c.flags = touched ? kCTouched : 0u;
            contactFromManifold(P, ba, bb, found[k], c);
            c.boundsFirst = boundsFirst;
            c.boundsCount = boundsCount;
            int best = -1;
            for (uint32_t it = lo; it < hi; ++it) {
                if (old[it].count > 0 && (best < 0 || dot(old[it].normal, c.normal) > dot(old[best].normal, c.normal))) {
                    best = (int)it;
                }
            }
            if (best >= 0) { carryImpulses(old[best], c, P.tol.speculative * P.tol.speculative); }
            out = c;
        }
        out.friction = sqrtf(sa.friction * sb.friction);
        out.restitution = maxf(sa.restitution, sb.restitution);
        out.rollingResistance = maxf(sa.rollingResistance, sb.rollingResistance);
    }
    if (ba.type == kDynamic && !ba.awake && movingAwake(bb)) {
        B.wakeMark[sa.body] = 1;
        wc.wakePending = 1;
    }
    if (bb.type == kDynamic && !bb.awake && movingAwake(ba)) {
        B.wakeMark[sb.body] = 1;
        wc.wakePending = 1;
    }
    B.stagePart[wi.candFirst + i] = extra;
    B.stageUsed[wi.candFirst + i] = (uint8_t)n;
}

// The candidate pairs of one class, over every world, one thread per pair (src/world.cpp:874-960); each
// result lands in the pair's own staging slot, so pairs need no order among themselves.
template <int Cls>
__device__ __forceinline__ void collideClass(const Batch& B, const StepParams& P, int serial) {
    const uint32_t n = *(volatile uint32_t*)(B.work + kSlotCandItems + Cls);
    const uint2* items = B.candItems + (size_t)Cls * B.candItemStride;
    for (uint32_t item = blockIdx.x * blockDim.x + threadIdx.x; item < n; item += gridDim.x * blockDim.x) {
        const uint2 it = items[item];
        const WorldInfo wi = B.info[it.x];
        WorldCounts& wc = B.counts[it.x];
        if constexpr (Cls == kClassMesh) {
            narrowMesh<false>(B, P, wi, wc, it.y, B.previous + wi.contactFirst, wc.contactCount, serial);
        } else {
            narrowOne<Cls>(B, P, wi, wc, it.y, B.previous + wi.contactFirst, wc.contactCount);
        }
    }
}

// The mesh candidates over every world, a warp per pair, the warp's lanes over the pair's triangles: a pair
// near many triangles (a large or fast shape on a fine mesh) no longer holds a whole launch on one thread.
// Launched with at most kMeshWarps warps to a CTA.
__device__ __forceinline__ void collideMeshPairs(const Batch& B, const StepParams& P, int serial) {
    __shared__ MeshWarpRoom s_rooms[kMeshWarps];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t perCta = min(blockDim.x >> 5, (uint32_t)kMeshWarps);  // warps past the rooms stay idle
    if (warp >= perCta) { return; }
    const uint32_t n = *(volatile uint32_t*)(B.work + kSlotCandItems + kClassMesh);
    const uint2* items = B.candItems + (size_t)kClassMesh * B.candItemStride;
    const uint32_t warps = gridDim.x * perCta;
    for (uint32_t item = blockIdx.x * perCta + warp; item < n; item += warps) {
        const uint2 it = items[item];
        const WorldInfo wi = B.info[it.x];
        WorldCounts& wc = B.counts[it.x];
        narrowMesh<true>(B, P, wi, wc, it.y, B.previous + wi.contactFirst, wc.contactCount, serial, &s_rooms[warp], lane);
        __syncwarp();
    }
}

template <int Cls>
__global__ void __launch_bounds__(256) k_collide(const __grid_constant__ Batch B, const __grid_constant__ StepParams P,
                                                 int serial) {
    if (stepAborted(B, serial)) { return; }
    if constexpr (Cls == kClassMesh) {
        collideMeshPairs(B, P, serial);
    } else {
        collideClass<Cls>(B, P, serial);
    }
}

// Small batches collide every pair class in one launch, each class's list in turn over the whole grid (the
// classes' pairs are disjoint); large batches launch a kernel per class, which keeps a warp on one code path.
template <int Unused = 0>
__global__ void __launch_bounds__(256) k_collide_all(const __grid_constant__ Batch B, const __grid_constant__ StepParams P,
                                                     int serial) {
    if (stepAborted(B, serial)) { return; }
    collideClass<kClassSpheres>(B, P, serial);
    collideClass<kClassSpherePoly>(B, P, serial);
    collideClass<kClassPlane>(B, P, serial);
    collideClass<kClassConvex>(B, P, serial);
    collideClass<kClassPlanar>(B, P, serial);
    collideClass<kClassMesh>(B, P, serial);
}

__device__ __forceinline__ bool keyLess(uint64_t ka, uint32_t pa, uint64_t kb, uint32_t pb) {
    return ka != kb ? ka < kb : pa < pb;
}

template <int Unused = 0>
__global__ void __launch_bounds__(kMaxBlock) k_narrowphase(const __grid_constant__ Batch B, const __grid_constant__ StepParams P, const __grid_constant__ Split sp, int serial) {
    if (stepAborted(B, serial)) { return; }
    forWorlds(B, kSlotNarrow, sp, nullptr, [&](const Group& g, uint32_t w, unsigned char*, const StageSizes&) {
        const WorldInfo wi = B.info[w];
        WorldCounts& wc = B.counts[w];
        if (g.tid == 0) {
            wc.touchEvents = 0;
            wc.hitEvents = 0;
            wc.touching = 0;
        }
        keepPlacements(B, g, wi);
        const uint32_t nc = wc.candCount;
        const uint32_t oldCount = wc.contactCount;
        const DContact* old = B.previous + wi.contactFirst;
        const uint32_t cf = wi.contactFirst;
        // Every candidate's contacts in part order: the first in its staging slot, the others (mesh pairs) in
        // the world's extra parts, named with the high bit set.
        const uint32_t nC = groupExpand(
            g, nc, [&](uint32_t i) { return (uint32_t)B.stageUsed[wi.candFirst + i]; },
            [&](uint32_t i, uint32_t pos, uint32_t k) {
                const uint32_t x = k == 0 ? i : (0x80000000u | (B.stagePart[wi.candFirst + i] + k - 1));
                const DContact* c = k == 0 ? B.stage + wi.candFirst + i : B.stageExtra + wi.partFirst + (x & 0x7fffffffu);
                B.mergeKeyA[cf + pos] = c->key;
                B.mergePartA[cf + pos] = c->part;
                B.mergeIdxA[cf + pos] = x;
            });
        // Contacts of pairs where nothing moves and one body is dynamic (asleep) stay as they were
        // (src/world.cpp:961-988).
        auto keepOld = [&](uint32_t j) {
            const DContact& c = old[j];
            if (!TF_OK_INDEX(B, c.bodyA - wi.bodyFirst < wi.bodyCount && c.bodyB - wi.bodyFirst < wi.bodyCount, 4,
                             wi.bodyFirst, j)) {
                return false;
            }
            const DBody& a = B.bodies[c.bodyA];
            const DBody& b = B.bodies[c.bodyB];
            if ((c.flags & kCRemoved) || movingAwake(a) || movingAwake(b)) { return false; }
            return !(a.type != kDynamic && b.type != kDynamic);
        };
        const uint32_t nK = groupCompact(
            g, oldCount, keepOld,
            [&](uint32_t j, uint32_t pos) {
                B.mergeKeyB[cf + pos] = old[j].key;
                B.mergePartB[cf + pos] = old[j].part;
                B.mergeIdxB[cf + pos] = j;
            });
        const uint32_t total = nC + nK;
        if (total > wi.contactCap) {
            if (g.tid == 0) {
                wc.flags |= kDevContactOverflow;
                wc.contactNeeded = max(wc.contactNeeded, total);
                atomicMin(B.abortStep, (uint32_t)serial);
            }
            g.sync();
            return;
        }
        // Stable merge by (key, part): collided contacts first among equals, as std::inplace_merge keeps them.
        for (uint32_t x = g.tid; x < nC; x += g.size) {
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
            const uint32_t src = B.mergeIdxA[cf + x];
            const DContact* from = (src & 0x80000000u) ? B.stageExtra + wi.partFirst + (src & 0x7fffffffu)
                                                        : B.stage + wi.candFirst + src;
            B.contacts[cf + x + l] = *from;
        }
        for (uint32_t y = g.tid; y < nK; y += g.size) {
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
        // A touching pair whose old contacts were dropped and that was not collided again has ended
        // (src/world.cpp:963-981): one event per pair, from its first such contact.
        for (uint32_t j = g.tid; j < oldCount; j += g.size) {
            const uint64_t key = old[j].key;
            if (!(old[j].flags & kCTouched) || keepOld(j)) { continue; }
            bool first = true;
            for (uint32_t k = j; k > 0 && old[k - 1].key == key && first; --k) {
                first = !((old[k - 1].flags & kCTouched) && !keepOld(k - 1));
            }
            if (!first) { continue; }
            uint32_t l = 0, h = nC;
            while (l < h) {
                const uint32_t mid = (l + h) >> 1;
                if (B.mergeKeyA[cf + mid] < key) {
                    l = mid + 1;
                } else {
                    h = mid;
                }
            }
            if (l < nC && B.mergeKeyA[cf + l] == key) { continue; }
            const uint32_t at = atomicAdd(&wc.touchEvents, 1u);
            B.touchEvents[2 * (size_t)cf + at] = TouchEvent{ key, 0u, 0u };
        }
        g.sync();
        if (g.tid == 0) {
            wc.nextContactCount = total;
            wc.contactNeeded = max(wc.contactNeeded, total);
        }
        g.sync();
    });
}

// ---------------------------------------------------------------------------------------------------------
// Waking (src/world.cpp:705-735): sleeping bodies a moving body reached wake, and so does everything linked
// to them by a contact with points. Runs on the group's first thread; it is rare.

template <int Unused = 0>
__global__ void __launch_bounds__(kMaxBlock) k_wake(const __grid_constant__ Batch B, const __grid_constant__ Split sp, int serial) {
    if (stepAborted(B, serial)) { return; }
    forWorlds(B, kSlotWake, sp, nullptr, [&](const Group& g, uint32_t w, unsigned char*, const StageSizes&) {
        if (g.tid != 0) { return; }
        const WorldInfo wi = B.info[w];
        WorldCounts& wc = B.counts[w];
        if (!wc.wakePending) { return; }
        wc.wakePending = 0;
        uint32_t* stack = B.unionParent + wi.bodyFirst;
        uint32_t top = 0;
        for (uint32_t i = 0; i < wi.bodyCount; ++i) {
            const uint32_t gb = wi.bodyFirst + i;
            if (!B.wakeMark[gb]) { continue; }
            const DBody& b = B.bodies[gb];
            if (b.alive && b.type == kDynamic && !b.awake && top < wi.bodyCount) {
                stack[top++] = gb;
            } else {
                B.wakeMark[gb] = 0;
            }
        }
        wakeStack(B, wi, B.contacts + wi.contactFirst, wc.nextContactCount, stack, top);
    });
}

// ---------------------------------------------------------------------------------------------------------
// Step state, lists, preparation and coloring (src/world.cpp:1589-1657, src/lanes.cpp:356-407).

constexpr uint32_t kNone = 0x7fffffffu;
constexpr uint32_t kNotColorable = 0x80000000u;

// ---------------------------------------------------------------------------------------------------------
// The laned contacts' solver record.
//
// The reference solves a color's contacts from a packed per-batch record rather than from its Contact
// (ContactLanes, src/internal.h:579-621, built by prepareBatch, src/lanes.cpp:66-110). Here each laned contact
// has one at its slot (contactFirst + its position in the world's colored list), component-major: component k
// of every slot is one float4 array, so the lanes of a color read consecutive 16-byte words. It holds what the
// substep's passes read of a contact and its points, and the impulses, which stay in it from k_prepare to
// k_finish (k_finish writes them back into the contact; a mid-step refresh takes them back first and builds
// the record again). Of each axis (makeAxis, src/solver.cpp:5-17) it keeps the velocity changes per unit
// impulse and the effective mass; the linear ones are the same for every point of a contact and are kept once;
// the lever arms, a cross product each, are formed again by every pass, with makeAxis's own arithmetic, so each
// pass sees the bits of the axes as built. 144 bytes a point and 144 a contact, against 240 bytes a point of
// stored axes plus the lines of the 560-byte contact a pass read before.
enum RowWord : int {
    kRowHead = 0,    // bodyA, bodyB (global), point count, contact index within the world (as integer bits)
    kRowNormal = 1,  // normal, friction
    kRowT1 = 2,      // tangent1, unused
    kRowT2 = 3,      // tangent2, unused
    kRowLinear = 4,  // 5 words: linearA, linearB of the normal, tangent1 and tangent2 axes (18 floats, 2 unused)
    kRowPoint = 9,   // point i, 9 words from kRowPoint + 9 i: anchorA and adjusted separation; anchorB and normal
                     // mass; tangent masses, normal impulse, largest normal impulse; tangent impulse; then 5
                     // words: angularA, angularB of the normal, tangent1 and tangent2 axes (2 floats unused)
    kRowPointWords = 9,
    kRowWords = kRowPoint + 4 * kRowPointWords
};
constexpr uint32_t kNoSlot = 0xffffffffu;

__device__ __forceinline__ float4 f4(const Vec3& v, float w) { return make_float4(v.x, v.y, v.z, w); }
__device__ __forceinline__ Vec3 xyz(const float4& v) { return Vec3{ v.x, v.y, v.z }; }

// Six vectors (18 floats) into 5 consecutive components at R + first * S, and back.
__device__ __forceinline__ void putSix(float4* R, size_t S, int first, const Vec3 (&v)[6]) {
    R[first * S] = make_float4(v[0].x, v[0].y, v[0].z, v[1].x);
    R[(first + 1) * S] = make_float4(v[1].y, v[1].z, v[2].x, v[2].y);
    R[(first + 2) * S] = make_float4(v[2].z, v[3].x, v[3].y, v[3].z);
    R[(first + 3) * S] = make_float4(v[4].x, v[4].y, v[4].z, v[5].x);
    R[(first + 4) * S] = make_float4(v[5].y, v[5].z, 0.0f, 0.0f);
}

struct SixVec {
    Vec3 v[6];
};

__device__ __forceinline__ SixVec getSix(const float4* R, size_t S, int first) {
    const float4 a = R[first * S], b = R[(first + 1) * S], c = R[(first + 2) * S], d = R[(first + 3) * S],
                 e = R[(first + 4) * S];
    SixVec x;
    x.v[0] = { a.x, a.y, a.z };
    x.v[1] = { a.w, b.x, b.y };
    x.v[2] = { b.z, b.w, c.x };
    x.v[3] = { c.y, c.z, c.w };
    x.v[4] = { d.x, d.y, d.z };
    x.v[5] = { d.w, e.x, e.y };
    return x;
}

// Builds the record of laned contact ci (world-local) at global slot `slot`, from the contact as prepared and
// its bodies' current world inverse mass and inertia (the axes are makeAxis's).
static __device__ void buildRow(const Batch& B, const WorldInfo& wi, uint32_t slot, uint32_t ci) {
    const DContact& c = B.contacts[wi.contactFirst + ci];
    const AxisBody xa = axisBodyOf(B.bodies[c.bodyA]), xb = axisBodyOf(B.bodies[c.bodyB]);
    float4* R = B.rows + slot;
    const size_t S = B.rowStride;
    const int n = c.count;
    R[kRowHead * S] = make_float4(__uint_as_float(c.bodyA), __uint_as_float(c.bodyB), __uint_as_float((uint32_t)n),
                                  __uint_as_float(ci));
    R[kRowNormal * S] = f4(c.normal, c.friction);
    R[kRowT1 * S] = f4(c.tangent1, 0.0f);
    R[kRowT2 * S] = f4(c.tangent2, 0.0f);
    const Vec3 linear[6] = { xa.invMassWorld * c.normal, xb.invMassWorld * c.normal, xa.invMassWorld * c.tangent1,
                             xb.invMassWorld * c.tangent1, xa.invMassWorld * c.tangent2, xb.invMassWorld * c.tangent2 };
    putSix(R, S, kRowLinear, linear);
    for (int i = 0; i < n; ++i) {
        const DPoint& p = c.points[i];
        const Axis xn = makeAxis(xa, xb, p.anchorA, p.anchorB, c.normal);
        const Axis x1 = makeAxis(xa, xb, p.anchorA, p.anchorB, c.tangent1);
        const Axis x2 = makeAxis(xa, xb, p.anchorA, p.anchorB, c.tangent2);
        const int at = kRowPoint + kRowPointWords * i;
        R[at * S] = f4(p.anchorA, p.adjustedSeparation);
        R[(at + 1) * S] = f4(p.anchorB, xn.mass);
        R[(at + 2) * S] = make_float4(x1.mass, x2.mass, p.normalImpulse, p.maxNormalImpulse);
        R[(at + 3) * S] = f4(p.tangentImpulse, 0.0f);
        const Vec3 angular[6] = { xn.angularA, xn.angularB, x1.angularA, x1.angularB, x2.angularA, x2.angularB };
        putSix(R, S, at + 4, angular);
    }
}

// The impulses a laned contact's record holds, back into the contact.
__device__ __forceinline__ void returnImpulses(const Batch& B, uint32_t slot, DContact& c) {
    const float4* R = B.rows + slot;
    const size_t S = B.rowStride;
    for (int i = 0; i < c.count; ++i) {
        const int at = kRowPoint + kRowPointWords * i;
        const float4 m = R[(at + 2) * S];
        const float4 t = R[(at + 3) * S];
        c.points[i].normalImpulse = m.z;
        c.points[i].maxNormalImpulse = m.w;
        c.points[i].tangentImpulse = xyz(t);
    }
}

constexpr uint32_t kOrderRounds = 64;       // rounds of visitInBodyOrder at most before one thread takes the rest
constexpr uint32_t kOrderRoundsMin = 64;    // shorter lists go to one thread at once
constexpr uint8_t kColorPending = 0xff;

// Visits the n entries of a contact list so that, at every moving body, its contacts are visited in list
// order: in each round every pending entry that is the first pending one at each of its bodies is visited
// (round r marks a body with (tag of r, its first pending entry) by atomicMin, tags falling from round to
// round so a round's marks replace the last one's). Entries visited in one round share no body, so visit(x)
// may read and write its own bodies' state without atomics. A result that depends, per body, only on the
// entries before x at that body (a greedy color, a level) therefore comes out as a pass in list order gives
// it. Once a round visits too few entries to pay for its two passes over the list (a long chain of contacts
// through a stack), or after kOrderRounds rounds, one thread visits what is left in list order, which keeps
// that property: the entries visited so far include every entry before them at a shared body. ends(x, a, b)
// gives an entry's bodies (kNone for one that does not count); firstAt holds a word per body, set to kNone
// beforehand.
template <class Ends, class Pending, class Visit>
static __device__ void visitInBodyOrder(const Group& g, uint32_t n, uint32_t* firstAt, Ends ends, Pending pending,
                                        Visit visit) {
    __shared__ uint32_t s_visits[kMaxGroups][2];
    if (n >= kOrderRoundsMin && n < (1u << 24)) {
        // A round costs two passes of n / size entries per thread; one thread takes an entry in about as long.
        const uint32_t worth = (n + g.size - 1) / g.size + 4;
        if (g.tid == 0) { s_visits[g.id][0] = 0; }
        for (uint32_t r = 0; r < kOrderRounds; ++r) {
            const uint32_t tag = (kOrderRounds - 1 - r) << 24;
            bool left = false;
            for (uint32_t x = g.tid; x < n; x += g.size) {
                if (!pending(x)) { continue; }
                left = true;
                uint32_t a, b;
                ends(x, a, b);
                if (a != kNone) { atomicMin(&firstAt[a], tag | x); }
                if (b != kNone) { atomicMin(&firstAt[b], tag | x); }
            }
            if (!g.any(left)) { return; }
            if (g.tid == 0) { s_visits[g.id][(r + 1) & 1] = 0; }
            uint32_t visited = 0;
            for (uint32_t x = g.tid; x < n; x += g.size) {
                if (!pending(x)) { continue; }
                uint32_t a, b;
                ends(x, a, b);
                if ((a == kNone || firstAt[a] == (tag | x)) && (b == kNone || firstAt[b] == (tag | x))) {
                    visit(x);
                    ++visited;
                }
            }
            if (visited) { atomicAdd(&s_visits[g.id][r & 1], visited); }
            g.sync();
            if (s_visits[g.id][r & 1] < worth) { break; }
        }
    }
    if (g.tid == 0) {
        for (uint32_t x = 0; x < n; ++x) {
            if (pending(x)) { visit(x); }
        }
    }
    g.sync();
}

// Greedy lowest free color of 32 over the moving bodies, in list order (src/lanes.cpp:356-374). endA/endB
// hold each contact's moving bodies (kNone for one that does not move); endA carries kNotColorable for a
// planar or rolling contact, which takes no color. masks (a word per body) start at 0, firstAt at kNone.
static __device__ void colorInOrder(const Group& g, uint32_t n, const uint32_t* endA, const uint32_t* endB,
                                    uint32_t* masks, uint32_t* firstAt, uint8_t* color) {
    for (uint32_t x = g.tid; x < n; x += g.size) { color[x] = (endA[x] & kNotColorable) ? kNoColor : kColorPending; }
    g.sync();
    visitInBodyOrder(
        g, n, firstAt, [&](uint32_t x, uint32_t& a, uint32_t& b) { a = endA[x], b = endB[x]; },
        [&](uint32_t x) { return color[x] == kColorPending; },
        [&](uint32_t x) {
            const uint32_t a = endA[x], b = endB[x];
            const uint32_t taken = (a != kNone ? masks[a] : 0u) | (b != kNone ? masks[b] : 0u);
            uint8_t k = kNoColor;
            if (taken != 0xffffffffu) {
                const int f = __ffs(~taken) - 1;
                if (a != kNone) { masks[a] |= 1u << f; }
                if (b != kNone) { masks[b] |= 1u << f; }
                k = (uint8_t)f;
            }
            color[x] = k;
        });
}

// Groups a contact list by color: every color's contacts (any order within a color, which solves the same)
// into colored, colors in ascending order, the uncolored ones into rest in list order.
static __device__ void bucketByColor(const Group& g, uint32_t n, const uint32_t* list, const uint8_t* colorOf, uint32_t* colored,
                              uint32_t* rest, uint32_t* startOut, uint32_t& colorsUsed, uint32_t& restCount) {
    __shared__ uint32_t s_size[kMaxGroups][kColors + 1];
    __shared__ uint32_t s_fill[kMaxGroups][kColors + 1];
    uint32_t* size = s_size[g.id];
    uint32_t* fill = s_fill[g.id];
    for (uint32_t k = g.tid; k <= kColors; k += g.size) { size[k] = 0; }
    g.sync();
    for (uint32_t x = g.tid; x < n; x += g.size) { atomicAdd(&size[colorOf[list[x]]], 1u); }
    g.sync();
    if (g.tid == 0) {
        uint32_t sum = 0, used = 0;
        for (int k = 0; k <= kColors; ++k) {
            startOut[k] = sum;
            fill[k] = sum;
            sum += size[k];
            if (k < kColors && size[k] > 0) { used = (uint32_t)k + 1; }
        }
        colorsUsed = used;
    }
    g.sync();
    for (uint32_t x = g.tid; x < n; x += g.size) {
        const uint8_t k = colorOf[list[x]];
        if (k != kNoColor) {
            const uint32_t at = atomicAdd(&fill[k], 1u);
#if defined(TF_DEVICE_CHECKS)
            if (at >= n) { continue; }
#endif
            colored[at] = list[x];
        }
    }
    const uint32_t r = groupCompact(g, n, [&](uint32_t x) { return colorOf[list[x]] == kNoColor; },
                                    [&](uint32_t x, uint32_t pos) { rest[pos] = list[x]; });
    if (g.tid == 0) { restCount = r; }
    g.sync();
}

// The contacts solved one at a time (planar, rolling, those past the colors) are swept in list order. Only
// contacts that share a moving body depend on that order: each takes a level one past the last earlier
// contact on either of its moving bodies, so that the contacts of a level share no moving body and run
// together while every body still meets its contacts in list order, which gives the sweep's own bits. The
// levels come from visitInBodyOrder; one thread then reorders list by level (stably, within the level in list
// order) and writes each level's end. last and firstAt (one word per body, zero and kNone on entry), tmp and
// out (one word per entry) are scratch. Returns the levels.
static __device__ uint32_t levelList(const Group& g, const Batch& B, const WorldInfo& wi, const DContact* cs,
                                     uint32_t* list, uint32_t n, uint32_t* levelEnd, uint32_t* last,
                                     uint32_t* firstAt, uint32_t* tmp, uint32_t* out) {
    __shared__ uint32_t s_levels[kMaxGroups];
    // Each entry's moving bodies (tmp, out) and its level (levelEnd, kNone until set).
    for (uint32_t x = g.tid; x < n; x += g.size) {
        const DContact& c = cs[list[x]];
        const uint32_t a = c.bodyA - wi.bodyFirst, b = c.bodyB - wi.bodyFirst;
        tmp[x] = a < wi.bodyCount && movingBody(B.bodies[c.bodyA]) ? a : kNone;
        out[x] = b < wi.bodyCount && movingBody(B.bodies[c.bodyB]) ? b : kNone;
        levelEnd[x] = kNone;
    }
    if (g.tid == 0) { s_levels[g.id] = 0; }
    g.sync();
    visitInBodyOrder(
        g, n, firstAt, [&](uint32_t x, uint32_t& a, uint32_t& b) { a = tmp[x], b = out[x]; },
        [&](uint32_t x) { return levelEnd[x] == kNone; },
        [&](uint32_t x) {
            const uint32_t a = tmp[x], b = out[x];
            uint32_t lev = 0;
            if (a != kNone) { lev = max(lev, last[a]); }
            if (b != kNone) { lev = max(lev, last[b]); }
            if (a != kNone) { last[a] = lev + 1; }
            if (b != kNone) { last[b] = lev + 1; }
            levelEnd[x] = lev;
            atomicMax(&s_levels[g.id], lev + 1);
        });
    for (uint32_t x = g.tid; x < n; x += g.size) { tmp[x] = levelEnd[x]; }
    g.sync();
    const uint32_t levels = s_levels[g.id];
    if (g.tid == 0) {
        for (uint32_t l = 0; l < levels; ++l) { levelEnd[l] = 0; }
        for (uint32_t x = 0; x < n; ++x) { ++levelEnd[tmp[x]]; }
        uint32_t sum = 0;
        for (uint32_t l = 0; l < levels; ++l) {
            const uint32_t size = levelEnd[l];
            levelEnd[l] = sum;  // the level's fill position, its end once filled
            sum += size;
        }
        for (uint32_t x = 0; x < n; ++x) { out[levelEnd[tmp[x]]++] = list[x]; }
    }
    g.sync();
    for (uint32_t x = g.tid; x < n; x += g.size) { list[x] = out[x]; }
    g.sync();
    return levels;
}

// Runs f on every entry of a leveled list, a level at a time.
template <class F>
__device__ void forEachLevel(const Group& g, const uint32_t* list, const uint32_t* levelEnd, uint32_t levels, F f) {
    uint32_t begin = 0;
    for (uint32_t l = 0; l < levels; ++l) {
        const uint32_t end = levelEnd[l];
        for (uint32_t x = begin + g.tid; x < end; x += g.size) { f(list[x]); }
        g.sync();
        begin = end;
    }
}

// Coloring is staged in the group's shared slice (masks by body, endpoints by active contact) when the world
// fits stageBodies bodies and stageContacts active contacts, else in the world's global scratch.
template <int Unused = 0>
__global__ void __launch_bounds__(kMaxBlock) k_prepare(const __grid_constant__ Batch B, const __grid_constant__ StepParams P, const __grid_constant__ Split sp, int serial) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    __shared__ uint32_t s_fast[kMaxGroups], s_fastSolid[kMaxGroups], s_points[kMaxGroups];
    __shared__ uint32_t s_class[kMaxGroups][kPairClasses + 1], s_classBase[kMaxGroups][kPairClasses + 1];
    if (stepAborted(B, serial)) { return; }
    forWorlds(B, kSlotPrepare, sp, s_raw, [&](const Group& g, uint32_t w, unsigned char* slice, const StageSizes& ss) {
        const uint32_t stageBodies = ss.bodies, stageContacts = ss.contacts;
        const WorldInfo wi = B.info[w];
        WorldCounts& wc = B.counts[w];
        uint32_t nc = wc.nextContactCount;
        if (!TF_OK_INDEX(B, nc <= wi.contactCap, 6, w, nc)) { nc = 0; }
        if (g.tid == 0) {
            wc.contactCount = nc;
            s_fast[g.id] = 0;
            s_fastSolid[g.id] = 0;
            s_points[g.id] = 0;
        }
        for (uint32_t i = g.tid; i < wi.bodyCount; i += g.size) {
            const uint32_t gb = wi.bodyFirst + i;
            DBody& b = B.bodies[gb];
            B.struck[gb] = 0;
            if (!b.alive) { continue; }
            b.q0 = b.xf.q;
            b.qBase = b.xf.q;
            b.com0 = b.com;
            b.expectedTravel = (length(b.v) + length(b.w) * b.extent) * P.dt;
            b.dp = zero3();
            b.dq = qid();
            updateInverseMass(b);
        }
        g.sync();
        // Joints: what the step will report for them starts over (src/world.cpp:1647).
        for (uint32_t x = g.tid; x < wi.jointCount; x += g.size) {
            DJoint& j = B.joints[wi.jointFirst + x];
            j.brokeNow = 0;
            const JBody a = j.bodyA == kWorldEnd ? worldEnd() : jointBodyOf(B.bodies[j.bodyA]);
            const JBody b = jointBodyOf(B.bodies[j.bodyB]);
            if (jointActive(j, a, b)) {
                j.force = zero3();
                j.torque = zero3();
            }
        }
        const uint32_t cf = wi.contactFirst;
        DContact* cs = B.contacts + cf;
        const uint32_t nActive = groupCompact(
            g, nc,
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
                    atomicAdd(&s_fast[g.id], 1u);
                    if (!isPlanar(a) && !isPlanar(b)) {
                        f |= kFlagFastSolid;
                        atomicAdd(&s_fastSolid[g.id], 1u);
                    }
                }
                B.cflags[cf + i] = f | (on ? kFlagActive : 0);
                return on;
            },
            [&](uint32_t i, uint32_t pos) { B.active[cf + pos] = i; });
        const uint32_t* act = B.active + cf;
        // A world with fast contacts is refreshed between substeps: its fast contacts join the flat list of
        // their pair class, its other active contacts the light list.
        if (s_fast[g.id] > 0) {
            uint32_t* cls = s_class[g.id];
            if (g.tid <= kPairClasses) { cls[g.tid] = 0; }
            g.sync();
            auto listOf = [&](uint32_t x) {
                const uint32_t ci = act[x];
                if (!(B.cflags[cf + ci] & kFlagFast)) { return kPairClasses; }
                return pairClassOf(B, cs[ci].shapeA, cs[ci].shapeB);
            };
            for (uint32_t x = g.tid; x < nActive; x += g.size) { atomicAdd(&cls[listOf(x)], 1u); }
            g.sync();
            if (g.tid <= kPairClasses) {
                s_classBase[g.id][g.tid] = atomicAdd(B.work + kSlotFastItems + g.tid, cls[g.tid]);
                cls[g.tid] = 0;
            }
            g.sync();
            for (uint32_t x = g.tid; x < nActive; x += g.size) {
                const int l = listOf(x);
                const uint32_t pos = s_classBase[g.id][l] + atomicAdd(&cls[l], 1u);
                B.contactItems[(size_t)l * B.contactItemStride + pos] = make_uint2(w, act[x]);
            }
            g.sync();
        }
        const bool staged = wi.bodyCount <= stageBodies && nActive <= stageContacts;
        uint32_t* masks = staged ? reinterpret_cast<uint32_t*>(slice) : B.bodyColors + wi.bodyFirst;
        uint32_t* endA = staged ? masks + stageBodies : B.mergeIdxA + cf;
        uint32_t* endB = staged ? endA + stageContacts : B.mergeIdxB + cf;
        // Each body's first pending contact while coloring and leveling (the island scratch is free here).
        uint32_t* firstAt = staged ? endB + stageContacts : B.unionParent + wi.bodyFirst;
        // Colors by active position; moved to contact order below. The merge scratch is free by now.
        uint8_t* colorTmp = reinterpret_cast<uint8_t*>(B.mergePartA + cf);
        for (uint32_t i = g.tid; i < wi.bodyCount; i += g.size) {
            masks[i] = 0;
            firstAt[i] = kNone;
        }
        uint32_t points = 0;
        for (uint32_t x = g.tid; x < nActive; x += g.size) {
            if (!TF_OK_INDEX(B, act[x] < nc, 7, w, x)) { continue; }
            DContact& c = cs[act[x]];
            const DBody& a = B.bodies[c.bodyA];
            const DBody& b = B.bodies[c.bodyB];
            prepareContact(a, b, c);
            c.flags &= ~kCLaned;
            points += (uint32_t)c.count;
            const bool can = !(c.flags & kCPlanar) && !(c.rollingResistance > 0.0f);
            endA[x] = (movingBody(a) ? c.bodyA - wi.bodyFirst : kNone) | (can ? 0u : kNotColorable);
            endB[x] = movingBody(b) ? c.bodyB - wi.bodyFirst : kNone;
            // Bodies of pairs closing faster than the restitution threshold are struck (src/world.cpp:1029-1049).
            for (int i = 0; i < c.count; ++i) {
                if (c.points[i].relativeVelocity >= -P.restitutionThreshold) { continue; }
                if (a.type == kDynamic) { B.struck[c.bodyA] = 1; }
                if (b.type == kDynamic) { B.struck[c.bodyB] = 1; }
                break;
            }
        }
        atomicAdd(&s_points[g.id], points);
        g.sync();
        colorInOrder(g, nActive, endA, endB, masks, firstAt, colorTmp);
        uint8_t* colorOf = B.color + cf;
        for (uint32_t x = g.tid; x < nActive; x += g.size) {
            const uint8_t k = colorTmp[x];
            colorOf[act[x]] = k;
            if (k != kNoColor) { cs[act[x]].flags |= kCLaned; }
        }
        g.sync();
        const uint32_t nImpact = groupCompact(
            g, nActive,
            [&](uint32_t x) {
                const DContact& c = cs[act[x]];
                return B.struck[c.bodyA] || B.struck[c.bodyB];
            },
            [&](uint32_t x, uint32_t pos) { B.impact[cf + pos] = act[x]; });
        bucketByColor(g, nActive, act, colorOf, B.colored + cf, B.rest + cf, wc.colorStart, wc.colorCount, wc.restCount);
        bucketByColor(g, nImpact, B.impact + cf, colorOf, B.impactColored + cf, B.impactRest + cf, wc.impactColorStart,
                      wc.impactColorCount, wc.impactRestCount);
        // The laned contacts' records, in color order; the axes of the contacts solved one at a time.
        const uint32_t nColored = wc.colorStart[kColors];
        for (uint32_t x = g.tid; x < nColored; x += g.size) {
            const uint32_t ci = B.colored[cf + x];
            if (!TF_OK_INDEX(B, ci < nc, 7, w, x)) { continue; }
            B.slotOf[cf + ci] = cf + x;
            buildRow(B, wi, cf + x, ci);
        }
        for (uint32_t x = g.tid; x < wc.restCount; x += g.size) {
            const uint32_t ci = B.rest[cf + x];
            if (!TF_OK_INDEX(B, ci < nc, 7, w, x)) { continue; }
            B.slotOf[cf + ci] = kNoSlot;
            const DContact& c = cs[ci];
            makeContactAxes(axisBodyOf(B.bodies[c.bodyA]), axisBodyOf(B.bodies[c.bodyB]), c,
                            B.axes + (size_t)(cf + ci) * kAxesPerContact);
        }
        // The one-at-a-time lists by level; the coloring's scratch is free by now.
        for (int which = 0; which < 2; ++which) {
            const uint32_t n = which == 0 ? wc.restCount : wc.impactRestCount;
            if (n == 0) {
                if (g.tid == 0) { (which == 0 ? wc.restLevels : wc.impactRestLevels) = 0; }
                continue;
            }
            for (uint32_t i = g.tid; i < wi.bodyCount; i += g.size) {
                masks[i] = 0;
                firstAt[i] = kNone;
            }
            g.sync();
            uint32_t* list = (which == 0 ? B.rest : B.impactRest) + cf;
            uint32_t* ends = (which == 0 ? B.restLevel : B.impactRestLevel) + cf;
            const uint32_t levels = levelList(g, B, wi, cs, list, n, ends, masks, firstAt, endA, endB);
            if (g.tid == 0) { (which == 0 ? wc.restLevels : wc.impactRestLevels) = levels; }
            g.sync();
        }
        if (g.tid == 0) {
            wc.activeCount = nActive;
            wc.impactCount = nImpact;
            wc.fastCount = s_fast[g.id];
            wc.fastSolidCount = s_fastSolid[g.id];
            wc.activePoints = s_points[g.id];
        }
        g.sync();
    });
}
// ---------------------------------------------------------------------------------------------------------
// The substep (src/world.cpp:1658-1681).

// Calls f(contact index) for every contact of each color in turn, the colors apart by a group barrier.
template <class F>
__device__ void forEachColor(const Group& g, const uint32_t* list, const uint32_t* start, uint32_t colors, F f) {
    for (uint32_t k = 0; k < colors; ++k) {
        const uint32_t end = start[k + 1];
        for (uint32_t x = start[k] + g.tid; x < end; x += g.size) { f(list[x]); }
        g.sync();
    }
}

// Calls f(slot) for the record slot (first + position) of every laned contact, a color at a time.
template <class F>
__device__ void forEachColorSlot(const Group& g, uint32_t first, const uint32_t* start, uint32_t colors, F f) {
    for (uint32_t k = 0; k < colors; ++k) {
        const uint32_t end = start[k + 1];
        for (uint32_t x = start[k] + g.tid; x < end; x += g.size) { f(first + x); }
        g.sync();
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

// A contact takes a manifold of its pair collided again mid-step: new points on body A, the approach speed
// and largest impulse of the nearest old point, and the old impulses carried (src/world.cpp:1106-1137).
static __device__ void takeRefreshed(const Batch& B, const StepParams& P, const DBody& a, const DBody& b, DContact& c,
                              const Manifold& m) {
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

// A fast pair collided again with the remaining time (src/world.cpp:1074-1138).
template <int Cls = kClassAny>
__device__ void refreshContact(const Batch& B, const StepParams& P, DContact& c, float remaining) {
    const DBody& a = B.bodies[c.bodyA];
    const DBody& b = B.bodies[c.bodyB];
    const DShape sa = B.shapes[c.shapeA];
    const DShape sb = B.shapes[c.shapeB];
    // Polyhedra that turned little against each other keep the edge pair they met on (src/world.cpp:1051-1055).
    const Quat now = conjugate(a.xf.q) * b.xf.q, then = conjugate(a.q0) * b.q0;
    const bool little = fabsf(dot(now, then)) >= P.featureTurnCos;
    Manifold m;
    collidePair<Cls>(B, P, sa, sb, remaining, m, little ? c.featKind : kFeatNone, c.featA, c.featB);
    if (m.count == 0) {
        c.count = 0;
        return;
    }
    takeRefreshed(B, P, a, b, c, m);
}

// How far any point of the body moved since the step started (src/world.cpp:484-488).
__device__ __forceinline__ float movedThisStep(const DBody& b) {
    const Quat turn = conjugate(b.q0) * b.xf.q;
    const float s = minf(sqrtf(turn.x * turn.x + turn.y * turn.y + turn.z * turn.z), 1.0f);
    return length(b.com - b.com0) + 2.0f * asinRounded(s) * b.extent;
}

// The contacts of a fast mesh pair, one key run, collided again with the remaining time: the pair is
// collided once, skipping the triangles its collision at the step's start ruled out while they stay out of
// reach, and each contact in turn takes the new manifold whose normal is closest to its own; a contact left
// without one keeps no points (src/world.cpp:1078-1137).
// Warp: every lane of the warp calls it alike with the warp's room; the lanes collide the triangles together and
// lane 0 hands the manifolds to the contacts.
template <bool Warp>
static __device__ void refreshMeshRun(const Batch& B, const StepParams& P, const WorldInfo& wi, WorldCounts& wc, DContact* run,
                               int count, float remaining, MeshWarpRoom* room = nullptr, uint32_t lane = 0) {
    const DBody& a = B.bodies[run[0].bodyA];
    const DBody& b = B.bodies[run[0].bodyB];
    const DShape sa = B.shapes[run[0].shapeA];
    const DShape sb = B.shapes[run[0].shapeB];
    MeshBounds mb{ nullptr, 0, nullptr, 0, 0.0f };
    if (run[0].boundsCount > 0 && TF_OK_INDEX(B, run[0].boundsFirst + run[0].boundsCount <= wi.boundsCap, 36, wi.bodyFirst, 0)) {
        mb.known = B.triBounds + wi.boundsFirst + run[0].boundsFirst;
        mb.knownCount = (int)run[0].boundsCount;
        mb.moved = movedThisStep(a) + movedThisStep(b);
    }
    Manifold found[kMaxMeshParts];
    int n = 0;
    const int status = collideMeshPair<Warp>(B, P, sa, sb, remaining, found, n, &mb, Warp ? room->found : nullptr, lane);
    if (Warp && lane != 0) { return; }
    if (status != kMeshOk) {
        atomicOr(&wc.flags, kDevUnsupported);
        n = 0;
    }
    bool taken[kMaxMeshParts];
    for (int k = 0; k < n; ++k) { taken[k] = false; }
    for (int x = 0; x < count; ++x) {
        DContact& c = run[x];
        int pick = -1;
        for (int k = 0; k < n; ++k) {
            if (taken[k]) { continue; }
            if (pick < 0 || dot(found[k].normal, c.normal) > dot(found[pick].normal, c.normal)) { pick = k; }
        }
        if (pick < 0) {
            c.count = 0;
            continue;
        }
        taken[pick] = true;
        takeRefreshed(B, P, a, b, c, found[pick]);
    }
}

// The solver state of one body as a contact solved on its own (planar, rolling or past the last color) reads
// and writes it. Field names match DBody so the same solver templates run on either.
struct SBody {
    Vec3 v, w, dp;
    Quat dq;
    Mat3 invInertiaWorld;
    float planeInvMass, planeInvInertia;
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

// Staged words per body: v 0-2, w 3-5, dp 6-8, dq 9-12, type | awake << 8 in 13: what a laned solve reads
// and writes. The inverse world inertia (torques, contacts solved on their own) stays in global memory, so
// more bodies fit a slice.
constexpr int kSBodyWords = 14;

// Where one world's solver state lives during a substep: shared memory (structure of arrays, stride words
// apart) for worlds that fit, else the bodies in global memory.
struct SolverStore {
    float* s;
    uint32_t stride;
    bool staged;
    DBody* g;

    __device__ __forceinline__ float& at(int word, uint32_t i) const { return s[word * stride + i]; }

    __device__ LanedBody loadLaned(uint32_t i) const {
        LanedBody b;
        if (!staged) {
            const DBody& d = g[i];
            b.v = d.v;
            b.w = d.w;
            b.dp = d.dp;
            b.dq = d.dq;
            b.type = d.type;
            b.awake = d.awake;
            return b;
        }
        b.v = { at(0, i), at(1, i), at(2, i) };
        b.w = { at(3, i), at(4, i), at(5, i) };
        b.dp = { at(6, i), at(7, i), at(8, i) };
        b.dq = { at(9, i), at(10, i), at(11, i), at(12, i) };
        const uint32_t f = __float_as_uint(at(13, i));
        b.type = f & 0xffu;
        b.awake = f >> 8;
        return b;
    }

    __device__ SBody load(uint32_t i) const {
        SBody b;
        if (!staged) {
            const DBody& d = g[i];
            b.v = d.v;
            b.w = d.w;
            b.dp = d.dp;
            b.dq = d.dq;
            b.invInertiaWorld = d.invInertiaWorld;
            b.planeInvMass = d.planeInvMass;
            b.planeInvInertia = d.planeInvInertia;
            b.type = d.type;
            b.awake = d.awake;
            return b;
        }
        const LanedBody l = loadLaned(i);
        b.v = l.v;
        b.w = l.w;
        b.dp = l.dp;
        b.dq = l.dq;
        b.type = l.type;
        b.awake = l.awake;
        b.invInertiaWorld = g[i].invInertiaWorld;
        b.planeInvMass = g[i].planeInvMass;
        b.planeInvInertia = g[i].planeInvInertia;
        return b;
    }

    template <class BodyT>
    __device__ void storeVW(uint32_t i, const BodyT& b) const {
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
        at(13, i) = __uint_as_float(d.type | (d.awake << 8));
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
        b.invInertiaWorld = d.invInertiaWorld;
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

// One direction's axis at a point of a laned contact from its record: the lever arms formed as makeAxis forms
// them, the velocity changes and the effective mass as stored.
__device__ __forceinline__ Axis rowAxis(const Vec3& ra, const Vec3& rb, const Vec3& d, const Vec3& linA, const Vec3& angA,
                                        const Vec3& linB, const Vec3& angB, float mass) {
    Axis x;
    x.armA = cross(ra, d);
    x.armB = cross(rb, d);
    x.linearA = linA;
    x.angularA = angA;
    x.linearB = linB;
    x.angularB = angB;
    x.mass = mass;
    return x;
}

// warmStartLaned from the record: each point's normal and tangent impulses pushed in point order
// (src/lanes.cpp:195-217).
__device__ __forceinline__ void warmStartRow(const float4* R, size_t S, LanedBody& a, LanedBody& b, int n) {
    const bool moveA = !anchored(a), moveB = !anchored(b);
    const Vec3 normal = xyz(R[kRowNormal * S]), t1 = xyz(R[kRowT1 * S]), t2 = xyz(R[kRowT2 * S]);
    const SixVec lin = getSix(R, S, kRowLinear);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (i < n) {
            const int at = kRowPoint + kRowPointWords * i;
            const float4 pa = R[at * S], pb = R[(at + 1) * S], pm = R[(at + 2) * S], pt = R[(at + 3) * S];
            const SixVec ang = getSix(R, S, at + 4);
            const Vec3 ra = xyz(pa), rb = xyz(pb), ti = xyz(pt);
            pushMoving(a, b, rowAxis(ra, rb, normal, lin.v[0], ang.v[0], lin.v[1], ang.v[1], pb.w), pm.z, moveA, moveB);
            pushMoving(a, b, rowAxis(ra, rb, t1, lin.v[2], ang.v[2], lin.v[3], ang.v[3], pm.x), dot(ti, t1), moveA, moveB);
            pushMoving(a, b, rowAxis(ra, rb, t2, lin.v[4], ang.v[4], lin.v[5], ang.v[5], pm.y), dot(ti, t2), moveA, moveB);
        }
    }
}

// solveLaned from the record: the soft normal rows, then friction forward in the biased pass and in reverse in
// relax, with the operations and order of solveContact (src/solver.cpp:360-421, src/lanes.cpp:220-315). The
// impulses go back to the record.
__device__ __forceinline__ void solveRow(float4* R, size_t S, LanedBody& a, LanedBody& b, int n, const StepParams& P,
                                         bool useBias) {
    const bool moveA = !anchored(a), moveB = !anchored(b);
    const Softness soft = (!moveA || !moveB) ? P.staticSoft : P.contactSoft;
    const float4 nf = R[kRowNormal * S];
    const Vec3 normal = xyz(nf), t1 = xyz(R[kRowT1 * S]), t2 = xyz(R[kRowT2 * S]);
    const float friction = nf.w;
    const SixVec lin = getSix(R, S, kRowLinear);
    float ni[4] = { 0, 0, 0, 0 }, mi[4] = { 0, 0, 0, 0 };
    Vec3 ti[4] = {};
    const Vec3 dp = b.dp - a.dp;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (i < n) {
            const int at = kRowPoint + kRowPointWords * i;
            const float4 pa = R[at * S], pb = R[(at + 1) * S], pm = R[(at + 2) * S];
            ti[i] = xyz(R[(at + 3) * S]);
            ni[i] = pm.z;
            mi[i] = pm.w;
            const float4 g0 = R[(at + 4) * S], g1 = R[(at + 5) * S];
            const Vec3 ra = xyz(pa), rb = xyz(pb);
            const Vec3 d = dp + turned(b, rb) - turned(a, ra);
            const float sep = dot(d, normal) + pa.w;
            float bias = 0.0f, massScale = 1.0f, impulseScale = 0.0f;
            if (sep > 0.0f) {
                bias = sep * P.invH;
            } else if (useBias) {
                bias = maxf(soft.biasRate * sep, -P.maxPushout);
                massScale = soft.massScale;
                impulseScale = soft.impulseScale;
            }
            const Axis x = rowAxis(ra, rb, normal, lin.v[0], Vec3{ g0.x, g0.y, g0.z }, lin.v[1],
                                   Vec3{ g0.w, g1.x, g1.y }, pb.w);
            const float vn = speedAlong(a, b, normal, x);
            float impulse = -x.mass * massScale * (vn + bias) - impulseScale * ni[i];
            const float total = maxf(ni[i] + impulse, 0.0f);
            impulse = total - ni[i];
            ni[i] = total;
            mi[i] = maxf(mi[i], impulse);
            pushMoving(a, b, x, impulse, moveA, moveB);
        }
    }
    auto row = [&](int i) {
        const int at = kRowPoint + kRowPointWords * i;
        const Vec3 ra = xyz(R[at * S]), rb = xyz(R[(at + 1) * S]);
        const float4 pm = R[(at + 2) * S];
        const SixVec ang = getSix(R, S, at + 4);
        const Axis x1 = rowAxis(ra, rb, t1, lin.v[2], ang.v[2], lin.v[3], ang.v[3], pm.x);
        const Axis x2 = rowAxis(ra, rb, t2, lin.v[4], ang.v[4], lin.v[5], ang.v[5], pm.y);
        const float old1 = dot(ti[i], t1), old2 = dot(ti[i], t2);
        float f1 = old1 - x1.mass * speedAlong(a, b, t1, x1);
        float f2 = old2 - x2.mass * speedAlong(a, b, t2, x2);
        const float limit = friction * ni[i];
        const float mag = sqrtf(f1 * f1 + f2 * f2);
        if (mag > limit) {
            const float scale = mag > 0.0f ? limit / mag : 0.0f;
            f1 *= scale;
            f2 *= scale;
        }
        ti[i] = t1 * f1 + t2 * f2;
        pushMoving(a, b, x1, f1 - old1, moveA, moveB);
        pushMoving(a, b, x2, f2 - old2, moveA, moveB);
    };
    if (useBias) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (i < n) { row(i); }
        }
    } else {
#pragma unroll
        for (int i = 3; i >= 0; --i) {
            if (i < n) { row(i); }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (i < n) {
            const int at = kRowPoint + kRowPointWords * i;
            float4* m = R + (at + 2) * S;
            // The tangent masses stay; only the impulses are written.
            reinterpret_cast<float2*>(m)[1] = make_float2(ni[i], mi[i]);
            R[(at + 3) * S] = f4(ti[i], 0.0f);
        }
    }
}

// In checked builds, whether a record's bodies lie in the world and its point count is at most 4.
__device__ __forceinline__ bool rowOk(const Batch& B, const WorldInfo& wi, uint32_t ia, uint32_t ib, int n, int code) {
#if defined(TF_DEVICE_CHECKS)
    return TF_OK_INDEX(B, ia < wi.bodyCount && ib < wi.bodyCount && n >= 0 && n <= 4, code, wi.bodyFirst, ia);
#else
    return true;
#endif
}

// A refresh works on the contact itself: a laned contact first takes its impulses back from its record, and
// afterwards gets its record built again; a contact solved on its own gets its axes built again.
__device__ __forceinline__ void takeImpulsesBack(const Batch& B, const WorldInfo& wi, uint32_t ci, DContact& c) {
    if (c.flags & kCLaned) { returnImpulses(B, B.slotOf[wi.contactFirst + ci], c); }
}

__device__ __forceinline__ void rebuildSolverData(const Batch& B, const WorldInfo& wi, uint32_t ci, const DContact& c) {
    if (c.flags & kCLaned) {
        buildRow(B, wi, B.slotOf[wi.contactFirst + ci], ci);
        return;
    }
    makeContactAxes(axisBodyOf(B.bodies[c.bodyA]), axisBodyOf(B.bodies[c.bodyB]), c,
                    B.axes + (size_t)(wi.contactFirst + ci) * kAxesPerContact);
}

// The flat solve's store: the solver state of every body in global memory, kFlatBodyWords float4 a body
// (velocity and spin, the substep's displacement and turn, type | awake << 8 | alive << 16), small enough that
// a batch's bodies stay in L2 while its contacts are solved, indexed from a first body (a world's, or 0 for
// global indices). The same loads and stores as SolverStore's, over that array. For whole-batch views it also
// holds each body's pose (kFlatPoseWords) and the step's velocity-update terms (kFlatMotionWords), so that the
// body phases of a substep read a few coalesced words instead of the body's whole record.
constexpr int kFlatBodyWords = 4;
constexpr int kFlatPoseWords = 5;    // com; xf.p; xf.q; qBase; localCenter
constexpr int kFlatMotionWords = 7;  // gravity-and-force term, linear damping factor; torque term, angular
                                     // damping factor; linear then angular projection (18 floats, 2 unused)

struct FlatStore {
    float4* s;
    DBody* g;
    float4* pose = nullptr;
    float4* motion = nullptr;
    static constexpr bool staged = true;

    __device__ __forceinline__ uint32_t flags(uint32_t i) const { return __float_as_uint(s[kFlatBodyWords * i + 3].y); }

    __device__ __forceinline__ LanedBody loadLaned(uint32_t i) const {
        const float4 a = s[kFlatBodyWords * i], b = s[kFlatBodyWords * i + 1], c = s[kFlatBodyWords * i + 2],
                     d = s[kFlatBodyWords * i + 3];
        LanedBody x;
        x.v = { a.x, a.y, a.z };
        x.w = { a.w, b.x, b.y };
        x.dp = { b.z, b.w, c.x };
        x.dq = { c.y, c.z, c.w, d.x };
        const uint32_t f = __float_as_uint(d.y);
        x.type = f & 0xffu;
        x.awake = (f >> 8) & 0xffu;
        return x;
    }

    __device__ SBody load(uint32_t i) const {
        const LanedBody l = loadLaned(i);
        SBody b;
        b.v = l.v;
        b.w = l.w;
        b.dp = l.dp;
        b.dq = l.dq;
        b.type = l.type;
        b.awake = l.awake;
        b.invInertiaWorld = g[i].invInertiaWorld;
        b.planeInvMass = g[i].planeInvMass;
        b.planeInvInertia = g[i].planeInvInertia;
        return b;
    }

    template <class BodyT>
    __device__ __forceinline__ void storeVW(uint32_t i, const BodyT& b) const {
        s[kFlatBodyWords * i] = make_float4(b.v.x, b.v.y, b.v.z, b.w.x);
        reinterpret_cast<float2*>(s + kFlatBodyWords * i + 1)[0] = make_float2(b.w.y, b.w.z);
    }

    __device__ __forceinline__ void put(uint32_t i, const Vec3& v, const Vec3& w, const Vec3& dp, const Quat& dq,
                                        uint32_t f) const {
        s[kFlatBodyWords * i] = make_float4(v.x, v.y, v.z, w.x);
        s[kFlatBodyWords * i + 1] = make_float4(w.y, w.z, dp.x, dp.y);
        s[kFlatBodyWords * i + 2] = make_float4(dp.z, dq.x, dq.y, dq.z);
        s[kFlatBodyWords * i + 3] = make_float4(dq.w, __uint_as_float(f), 0.0f, 0.0f);
    }
};

__device__ __forceinline__ float4 q4(const Quat& q) { return make_float4(q.x, q.y, q.z, q.w); }
__device__ __forceinline__ Quat quatOf(const float4& v) { return Quat{ v.x, v.y, v.z, v.w }; }

// integrateVelocity's terms that stay fixed over a step (gravity and force, the damping factors, the
// projections) and the torque term, which changes only with the world inverse inertia. Stored as the very
// values integrateVelocity forms from them (src/world.cpp:1141-1151), so adding them gives its bits.
__device__ __forceinline__ void storeTorqueTerm(const FlatStore& f, uint32_t i, const DBody& d, const StepParams& P) {
    float4* m = f.motion + (size_t)kFlatMotionWords * i;
    const Vec3 t = d.invInertiaWorld * d.torque * P.h;
    m[1] = make_float4(t.x, t.y, t.z, m[1].w);
}

__device__ __forceinline__ void storeMotion(const FlatStore& f, uint32_t i, const DBody& d, const StepParams& P) {
    float4* m = f.motion + (size_t)kFlatMotionWords * i;
    const float h = P.h;
    const Vec3 gv = (P.gravity * d.gravityScale + d.force * d.invMass) * h;
    const Vec3 t = d.invInertiaWorld * d.torque * h;
    m[0] = f4(gv, 1.0f / (1.0f + h * d.linearDamping));
    m[1] = f4(t, 1.0f / (1.0f + h * d.angularDamping));
    const Mat3& L = d.linearProj;
    const Mat3& A = d.angularProj;
    m[2] = make_float4(L.r[0].x, L.r[0].y, L.r[0].z, L.r[1].x);
    m[3] = make_float4(L.r[1].y, L.r[1].z, L.r[2].x, L.r[2].y);
    m[4] = make_float4(L.r[2].z, A.r[0].x, A.r[0].y, A.r[0].z);
    m[5] = make_float4(A.r[1].x, A.r[1].y, A.r[1].z, A.r[2].x);
    m[6] = make_float4(A.r[2].y, A.r[2].z, 0.0f, 0.0f);
}

// The first substep's staging: the body's solver state, pose and velocity terms from its record.
static __device__ void flatBegin(const FlatStore& f, uint32_t i, const StepParams& P) {
    const DBody& d = f.g[i];
    f.put(i, d.v, d.w, d.dp, d.dq, d.type | (d.awake << 8) | (d.alive << 16));
    float4* q = f.pose + (size_t)kFlatPoseWords * i;
    q[0] = f4(d.com, 0.0f);
    q[1] = f4(d.xf.p, 0.0f);
    q[2] = q4(d.xf.q);
    q[3] = q4(d.qBase);
    q[4] = f4(d.localCenter, 0.0f);
    if (d.alive && d.type == kDynamic && d.awake) { storeMotion(f, i, d, P); }
}

// What limitSpeed reads and writes.
struct SpeedBody {
    Vec3 v, w;
    float kept;
    uint32_t type, awake;
};

// integrateVelocity from the store and the step's terms: the same operations on the same values.
static __device__ void flatVelocity(const FlatStore& f, uint32_t i, const StepParams& P) {
    const uint32_t fl = f.flags(i);
    const uint32_t type = fl & 0xffu, awake = (fl >> 8) & 0xffu, alive = fl >> 16;
    if (!alive || type != kDynamic || !awake) { return; }
    const LanedBody l = f.loadLaned(i);
    const float4* m = f.motion + (size_t)kFlatMotionWords * i;
    const float4 m0 = m[0], m1 = m[1], a = m[2], b = m[3], c = m[4], d = m[5], e = m[6];
    Mat3 L, A;
    L.r[0] = { a.x, a.y, a.z };
    L.r[1] = { a.w, b.x, b.y };
    L.r[2] = { b.z, b.w, c.x };
    A.r[0] = { c.y, c.z, c.w };
    A.r[1] = { d.x, d.y, d.z };
    A.r[2] = { d.w, e.x, e.y };
    SpeedBody s;
    s.type = type;
    s.awake = awake;
    s.kept = f.g[i].kept;
    s.v = l.v + xyz(m0);
    s.v = L * (s.v * m0.w);
    s.w = l.w + xyz(m1);
    s.w = A * (s.w * m1.w);
    limitSpeed(s, P.maxLinearSpeed, P.maxAngularSpeed);
    f.storeVW(i, s);
    f.g[i].kept = s.kept;
}

// integratePosition from the store and the pose: the new pose goes to the store and to the body's record (joints
// of the relaxing pass read it there).
static __device__ void flatPosition(const FlatStore& f, uint32_t i, const StepParams& P) {
    const uint32_t fl = f.flags(i);
    const LanedBody l = f.loadLaned(i);
    float4* q = f.pose + (size_t)kFlatPoseWords * i;
    DBody& d = f.g[i];
    PosBody b;
    b.alive = fl >> 16;
    b.type = l.type;
    b.awake = l.awake;
    b.v = l.v;
    b.w = l.w;
    b.dp = l.dp;
    b.dq = l.dq;
    b.com = xyz(q[0]);
    b.xf.p = xyz(q[1]);
    b.xf.q = quatOf(q[2]);
    b.qBase = quatOf(q[3]);
    b.localCenter = xyz(q[4]);
    b.kept = d.kept;
    integratePosition(b, P);
    f.put(i, b.v, b.w, b.dp, b.dq, fl);
    q[0] = f4(b.com, 0.0f);
    q[1] = f4(b.xf.p, 0.0f);
    q[2] = q4(b.xf.q);
    d.com = b.com;
    d.xf = b.xf;
    d.kept = b.kept;
}

// One contact's passes, for either store, with body indices counted from the store's first body (`base`: the
// same first body). A laned contact runs from its record, by slot; a contact solved on its own from the contact
// and its stored axes. A laned contact's bodies are stored only where they move, so a static body shared by a
// color's contacts is never written concurrently; a contact solved on its own stores both, as the reference
// does.
template <class Store>
__device__ __forceinline__ void warmRowAt(const Batch& B, const Store& st, uint32_t base, uint32_t limit,
                                          uint32_t slot) {
    const size_t S = B.rowStride;
    const float4* R = B.rows + slot;
    const float4 h = R[kRowHead * S];
    const uint32_t ia = __float_as_uint(h.x) - base, ib = __float_as_uint(h.y) - base;
    const int n = (int)__float_as_uint(h.z);
#if defined(TF_DEVICE_CHECKS)
    if (!TF_OK_INDEX(B, ia < limit && ib < limit && n >= 0 && n <= 4, 10, base, ia)) { return; }
#endif
    if (n == 0) { return; }
    LanedBody a = st.loadLaned(ia), b = st.loadLaned(ib);
    warmStartRow(R, S, a, b, n);
    if (!anchored(a)) { st.storeVW(ia, a); }
    if (!anchored(b)) { st.storeVW(ib, b); }
}

template <class Store>
__device__ __forceinline__ void solveRowAt(const Batch& B, const StepParams& P, const Store& st, uint32_t base,
                                           uint32_t limit, uint32_t slot, bool bias) {
    const size_t S = B.rowStride;
    float4* R = B.rows + slot;
    const float4 h = R[kRowHead * S];
    const uint32_t ia = __float_as_uint(h.x) - base, ib = __float_as_uint(h.y) - base;
    const int n = (int)__float_as_uint(h.z);
#if defined(TF_DEVICE_CHECKS)
    if (!TF_OK_INDEX(B, ia < limit && ib < limit && n >= 0 && n <= 4, 12, base, ia)) { return; }
#endif
    if (n == 0) { return; }
    LanedBody a = st.loadLaned(ia), b = st.loadLaned(ib);
    solveRow(R, S, a, b, n, P, bias);
    if (!anchored(a)) { st.storeVW(ia, a); }
    if (!anchored(b)) { st.storeVW(ib, b); }
}

template <class Store>
__device__ __forceinline__ void warmOne(const Batch& B, const WorldInfo& wi, const WorldCounts& wc, const Store& st,
                                        uint32_t ci) {
    if (!contactOk(B, wi, wc, ci, 10)) { return; }
    DContact& c = B.contacts[wi.contactFirst + ci];
    const uint32_t ia = c.bodyA - wi.bodyFirst, ib = c.bodyB - wi.bodyFirst;
    SBody a = st.load(ia), b = st.load(ib);
    warmStartContact(a, b, c, false, B.axes + (size_t)(wi.contactFirst + ci) * kAxesPerContact);
    st.storeVW(ia, a);
    st.storeVW(ib, b);
}

template <class Store>
__device__ __forceinline__ void solveOne(const Batch& B, const StepParams& P, const WorldInfo& wi, const WorldCounts& wc,
                                         const Store& st, uint32_t ci, bool bias) {
    if (!contactOk(B, wi, wc, ci, 12)) { return; }
    DContact& c = B.contacts[wi.contactFirst + ci];
    const uint32_t ia = c.bodyA - wi.bodyFirst, ib = c.bodyB - wi.bodyFirst;
    SBody a = st.load(ia), b = st.load(ib);
    solveContact(a, b, c, P, bias, B.axes + (size_t)(wi.contactFirst + ci) * kAxesPerContact);
    st.storeVW(ia, a);
    st.storeVW(ib, b);
}

// Whether the substep `sub` starts with a refresh of world wc: fast pairs are collided again at the middle
// substep, pairs of solid bodies also at every other substep but the first (src/world.cpp:1658-1668).
__device__ __forceinline__ bool refreshedAt(const WorldCounts& wc, int sub, int n) {
    return sub > 0 && (sub == n / 2 ? wc.fastCount : wc.fastSolidCount) > 0;
}

// The contact half of a refresh, over the worlds refreshed at this substep: other contacts are rebased,
// fast ones collided again with the time left, and every active contact's axes built again. One thread per
// contact; the contacts come from one flat list, a pair class of fast contacts (Cls) or the other active
// contacts (kClassAny). The body half runs in the substeps around it: the substep before updates the world
// inverse inertia at its end, the substep after resets dp and dq before anything reads them.
template <int Cls>
__device__ __forceinline__ void refreshClass(const Batch& B, const StepParams& P, int sub) {
    const int n = P.substeps;
    const uint8_t againFlag = sub == n / 2 ? kFlagFast : kFlagFastSolid;
    const float remaining = (float)(n - sub) * P.h;
    const int list = Cls == kClassAny ? kPairClasses : Cls;
    const uint32_t items = *(volatile uint32_t*)(B.work + kSlotFastItems + list);
    const uint2* its = B.contactItems + (size_t)list * B.contactItemStride;
    for (uint32_t item = blockIdx.x * blockDim.x + threadIdx.x; item < items; item += gridDim.x * blockDim.x) {
        const uint2 it = its[item];
        const WorldCounts& wc = B.counts[it.x];
        if (!refreshedAt(wc, sub, n)) { continue; }
        const WorldInfo wi = B.info[it.x];
        const uint32_t ci = it.y;
        if (!contactOk(B, wi, wc, ci, 16)) { continue; }
        DContact& c = B.contacts[wi.contactFirst + ci];
        bool again = false;
        if constexpr (Cls != kClassAny) { again = (B.cflags[wi.contactFirst + ci] & againFlag) != 0; }
        if constexpr (Cls == kClassMesh) {
            // The contacts of a mesh pair share a key and sit together; the first takes the whole run.
            const DContact* cs = B.contacts + wi.contactFirst;
            if (ci > 0 && cs[ci - 1].key == c.key) { continue; }
            uint32_t end = ci + 1;
            while (end < wc.contactCount && cs[end].key == c.key) { ++end; }
            DContact* run = B.contacts + wi.contactFirst + ci;
            const int count = (int)(end - ci);
            for (int x = 0; x < count; ++x) { takeImpulsesBack(B, wi, ci + x, run[x]); }
            if (again) {
                refreshMeshRun<false>(B, P, wi, B.counts[it.x], run, count, remaining);
            } else {
                for (int x = 0; x < count; ++x) { rebaseContact(B.bodies[run[x].bodyA], B.bodies[run[x].bodyB], run[x]); }
            }
            for (int x = 0; x < count; ++x) { rebuildSolverData(B, wi, ci + x, run[x]); }
            continue;
        }
        takeImpulsesBack(B, wi, ci, c);
        if constexpr (Cls != kClassAny) {
            if (again) { refreshContact<Cls>(B, P, c, remaining); }
        }
        if (!again) { rebaseContact(B.bodies[c.bodyA], B.bodies[c.bodyB], c); }
        rebuildSolverData(B, wi, ci, c);
    }
}

// The fast mesh pairs' contacts, a warp per item (the first contact of a pair's run takes the run), the warp's
// lanes over the pair's triangles when it is collided again. Launched with at most kMeshWarps warps to a CTA.
__device__ __forceinline__ void refreshMeshPairs(const Batch& B, const StepParams& P, int sub) {
    __shared__ MeshWarpRoom s_rooms[kMeshWarps];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t perCta = min(blockDim.x >> 5, (uint32_t)kMeshWarps);  // warps past the rooms stay idle
    if (warp >= perCta) { return; }
    const int n = P.substeps;
    const uint8_t againFlag = sub == n / 2 ? kFlagFast : kFlagFastSolid;
    const float remaining = (float)(n - sub) * P.h;
    const uint32_t items = *(volatile uint32_t*)(B.work + kSlotFastItems + kClassMesh);
    const uint2* its = B.contactItems + (size_t)kClassMesh * B.contactItemStride;
    const uint32_t warps = gridDim.x * perCta;
    for (uint32_t item = blockIdx.x * perCta + warp; item < items; item += warps) {
        const uint2 it = its[item];
        const WorldCounts& wc = B.counts[it.x];
        if (!refreshedAt(wc, sub, n)) { continue; }
        const WorldInfo wi = B.info[it.x];
        const uint32_t ci = it.y;
        if (!contactOk(B, wi, wc, ci, 16)) { continue; }
        const DContact* cs = B.contacts + wi.contactFirst;
        // The contacts of a mesh pair share a key and sit together; the first takes the whole run.
        if (ci > 0 && cs[ci - 1].key == cs[ci].key) { continue; }
        uint32_t end = ci + 1;
        while (end < wc.contactCount && cs[end].key == cs[ci].key) { ++end; }
        DContact* run = B.contacts + wi.contactFirst + ci;
        const int count = (int)(end - ci);
        const bool again = (B.cflags[wi.contactFirst + ci] & againFlag) != 0;
        if (lane == 0) {
            for (int x = 0; x < count; ++x) { takeImpulsesBack(B, wi, ci + x, run[x]); }
        }
        __syncwarp();
        if (again) {
            refreshMeshRun<true>(B, P, wi, B.counts[it.x], run, count, remaining, &s_rooms[warp], lane);
        } else if (lane == 0) {
            for (int x = 0; x < count; ++x) { rebaseContact(B.bodies[run[x].bodyA], B.bodies[run[x].bodyB], run[x]); }
        }
        if (lane == 0) {
            for (int x = 0; x < count; ++x) { rebuildSolverData(B, wi, ci + x, run[x]); }
        }
        __syncwarp();
    }
}

template <int Cls>
__global__ void __launch_bounds__(256) k_refresh(const __grid_constant__ Batch B, const __grid_constant__ StepParams P,
                                                 int sub, int serial) {
    if (stepAborted(B, serial)) { return; }
    if constexpr (Cls == kClassMesh) {
        refreshMeshPairs(B, P, sub);
    } else {
        refreshClass<Cls>(B, P, sub);
    }
}

// Small batches refresh every list in one launch (the lists hold disjoint contacts: a pair's contacts are fast
// or not together); large batches launch a kernel per list.
template <int Unused = 0>
__global__ void __launch_bounds__(256) k_refresh_all(const __grid_constant__ Batch B, const __grid_constant__ StepParams P,
                                                     int sub, int serial) {
    if (stepAborted(B, serial)) { return; }
    refreshClass<kClassAny>(B, P, sub);
    refreshClass<kClassSpheres>(B, P, sub);
    refreshClass<kClassSpherePoly>(B, P, sub);
    refreshClass<kClassPlane>(B, P, sub);
    refreshClass<kClassConvex>(B, P, sub);
    refreshClass<kClassPlanar>(B, P, sub);
    refreshClass<kClassMesh>(B, P, sub);
}

// One pass over a world's joints on one thread, before the contacts of that pass (src/world.cpp:1670-1680,
// src/joint.cpp:568-590): kind 0 scales warm starts by the speed the ends kept under the speed limits
// (src/joint.cpp:570-593) and warm starts, 1 is the biased solve, 2 the relaxing solve with its reaction. The
// ends' velocities come from the substep's store.
template <class Store>
__device__ void runJoints(const Batch& B, const StepParams& P, const WorldInfo& wi, const Store& st, int kind) {
    const uint32_t nj = wi.jointCount;
    DJoint* js = B.joints + wi.jointFirst;
    auto endOf = [&](uint32_t gbody) {
        if (gbody == kWorldEnd) { return worldEnd(); }
        JBody e = jointBodyOf(B.bodies[gbody]);
        if (st.staged) {
            const LanedBody l = st.loadLaned(gbody - wi.bodyFirst);
            e.v = l.v;
            e.w = l.w;
        }
        return e;
    };
    auto putEnd = [&](uint32_t gbody, const JBody& e) {
        if (gbody == kWorldEnd || e.type != kDynamic || !e.awake) { return; }
        st.storeVW(gbody - wi.bodyFirst, e);
    };
    if (kind == 0) {
        for (uint32_t x = 0; x < nj; ++x) {
            DJoint& j = js[x];
            const JBody a = endOf(j.bodyA), b = endOf(j.bodyB);
            if (!jointActive(j, a, b)) { continue; }
            const float f = minf(a.kept, b.kept);
            if (f >= 1.0f) { continue; }
            j.linearImpulse = j.linearImpulse * f;
            j.angularImpulse = j.angularImpulse * f;
            j.frictionTurn = j.frictionTurn * f;
            j.axialImpulse *= f;
            j.motorImpulse *= f;
            j.lowerImpulse *= f;
            j.upperImpulse *= f;
            j.frictionImpulse *= f;
            j.swingImpulse *= f;
        }
        for (uint32_t x = 0; x < nj; ++x) {
            const DJoint& j = js[x];
            if (!jointActive(j, endOf(j.bodyA), endOf(j.bodyB))) { continue; }
            if (j.bodyA != kWorldEnd) { B.bodies[j.bodyA].kept = 1.0f; }
            B.bodies[j.bodyB].kept = 1.0f;
        }
    }
    for (uint32_t x = 0; x < nj; ++x) {
        DJoint& j = js[x];
        JBody a = endOf(j.bodyA), b = endOf(j.bodyB);
        if (!jointActive(j, a, b)) { continue; }
        if (kind == 0) {
            warmStartJoint(a, b, j);
        } else {
            solveJoint(a, b, j, P, P.jointSoft, kind == 1);
            if (kind == 2) { addReaction(j); }
        }
        putEnd(j.bodyA, a);
        putEnd(j.bodyB, b);
    }
}

// Integrate velocities, warm start, biased solve, integrate positions, relax (src/world.cpp:1669-1680). The
// world's solver state is staged in the group's shared slice when it has at most stageN bodies.
// Joints is false for batches without joints: that instantiation carries no joint code, which would cost the
// contact solve registers.
template <bool Joints>
__global__ void __launch_bounds__(kMaxBlock) k_substep(const __grid_constant__ Batch B, const __grid_constant__ StepParams P, const __grid_constant__ Split sp, int sub, int serial) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    if (stepAborted(B, serial)) { return; }
    forWorlds(B, kSlotSubstep + sub, sp, s_raw, [&](const Group& g, uint32_t w, unsigned char* sliceRaw, const StageSizes& ss) {
        float* slice = reinterpret_cast<float*>(sliceRaw);
        const uint32_t stageN = ss.bodies;
        const WorldInfo wi = B.info[w];
        const WorldCounts& wc = B.counts[w];
        const uint32_t cf = wi.contactFirst;
        DContact* cs = B.contacts + cf;
        const uint32_t nb = wi.bodyCount;
        const SolverStore st{ slice, stageN, nb <= stageN, B.bodies + wi.bodyFirst };
        if (refreshedAt(wc, sub, P.substeps)) {
            // The body half of this substep's refresh: the planar placements of its collisions are kept, and
            // every body takes a new base pose (src/world.cpp:1663-1666).
            keepPlacements(B, g, wi);
            for (uint32_t i = g.tid; i < nb; i += g.size) {
                DBody& d = st.g[i];
                d.dp = zero3();
                d.dq = qid();
                d.qBase = d.xf.q;
            }
            g.sync();
        }
        if (st.staged) {
            for (uint32_t i = g.tid; i < nb; i += g.size) { st.stage(i); }
            g.sync();
        }
        for (uint32_t i = g.tid; i < nb; i += g.size) { st.integrateVelocityAt(i, P); }
        g.sync();
        const uint32_t nj = wi.jointCount;
        if constexpr (Joints) {
            if (nj > 0) {
                if (g.tid == 0) { runJoints(B, P, wi, st, 0); }
                g.sync();
            }
        }
        const uint32_t base = wi.bodyFirst;
        auto warmRow = [&](uint32_t slot) { warmRowAt(B, st, base, nb, slot); };
        auto solveRowAtSlot = [&](uint32_t slot, bool bias) { solveRowAt(B, P, st, base, nb, slot, bias); };
        auto warm = [&](uint32_t ci) { warmOne(B, wi, wc, st, ci); };
        auto solve = [&](uint32_t ci, bool bias) { solveOne(B, P, wi, wc, st, ci, bias); };
        const uint32_t* rest = B.rest + cf;
        const uint32_t* icolored = B.impactColored + cf;
        const uint32_t* irest = B.impactRest + cf;
        const uint32_t* slotOf = B.slotOf + cf;
        forEachColorSlot(g, cf, wc.colorStart, wc.colorCount, [&](uint32_t slot) { warmRow(slot); });
        forEachLevel(g, rest, B.restLevel + cf, wc.restLevels, [&](uint32_t ci) { warm(ci); });
        for (int pass = 0; pass < 2; ++pass) {
            const bool bias = pass == 0;
            if constexpr (Joints) {
                if (nj > 0) {
                    if (g.tid == 0) { runJoints(B, P, wi, st, bias ? 1 : 2); }
                    g.sync();
                }
            }
            forEachColorSlot(g, cf, wc.colorStart, wc.colorCount, [&](uint32_t slot) { solveRowAtSlot(slot, bias); });
            forEachLevel(g, rest, B.restLevel + cf, wc.restLevels, [&](uint32_t ci) { solve(ci, bias); });
            if (wc.impactCount > 0) {
                forEachColor(g, icolored, wc.impactColorStart, wc.impactColorCount,
                             [&](uint32_t ci) { solveRowAtSlot(slotOf[ci], bias); });
                forEachLevel(g, irest, B.impactRestLevel + cf, wc.impactRestLevels,
                             [&](uint32_t ci) { solve(ci, bias); });
            }
            if (bias) {
                for (uint32_t i = g.tid; i < nb; i += g.size) { st.integratePositionAt(i, P); }
                g.sync();
            }
        }
        if (st.staged) {
            for (uint32_t i = g.tid; i < nb; i += g.size) { st.unstage(i); }
            g.sync();
        }
        if (sub + 1 < P.substeps && refreshedAt(wc, sub + 1, P.substeps)) {
            // The next substep starts with a refresh, whose axes use the inverse inertia at the new pose
            // (src/world.cpp:1660-1662).
            for (uint32_t i = g.tid; i < nb; i += g.size) {
                DBody& d = st.g[i];
                if (d.alive && d.type == kDynamic && d.awake) { updateInverseMass(d); }
            }
        }
    });
}

// ---------------------------------------------------------------------------------------------------------
// The flat solve: one substep of every world of a batch of many small worlds as one cooperative launch.
//
// The world kernels above walk a world's colors with the world's own thread group, so a batch of thousands of
// worlds runs as thousands of short dependent chains, each waiting on its own barriers. Here the barrier is the
// grid's instead: each color's contacts of every world run at once across the device (contacts of one color
// move no body in common, in any world), then the next color, and the body phases run over every body of the
// batch. Contacts solved one at a time (by level), joints and a world's uncolored contacts keep their order
// inside their world, each world's on one warp or thread. Every contact and body sees exactly the operations,
// in the order, of the world kernel, so the results are the same bits.
//
// The grid barrier needs every CTA resident: the kernel is launched cooperatively, with at most as many CTAs
// as fit at once. Its wait is bounded: a CTA that has waited kBarrierSpins polls records kDevTimeout in world
// 0's flags and goes on (the host reports the step as failed), so a fault here cannot hang the device.
constexpr uint32_t kBarrierSpins = 1u << 24;

__device__ __forceinline__ uint32_t loadAcquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void storeRelease(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t addAcqRel(uint32_t* p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Arrivals only grow within a step (the step's work slots start at zero and every flat launch of a step has
// the same grid), so arrival t is at barrier t / gridDim of the step. The last arrival of a barrier publishes
// the number of barriers passed with a release store; the other CTAs wait for it with acquire loads. Nothing
// is reset between barriers, so a barrier costs one atomic round trip, a store and the waiters' polls.
static __device__ void gridBarrier(const Batch& B) {
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t* arrive = B.work + kSlotFlatBarrier;
        uint32_t* passed = B.work + kSlotFlatBarrier + 1;
        __threadfence();  // the CTA's writes before the barrier, ahead of its arrival
        const uint32_t ticket = addAcqRel(arrive, 1u);
        const uint32_t after = ticket / gridDim.x + 1;  // barriers passed once this one is
        if (ticket % gridDim.x == gridDim.x - 1) {
            storeRelease(passed, after);
        } else {
            uint32_t spins = 0;
            while ((int32_t)(loadAcquire(passed) - after) < 0) {
                if (++spins > kBarrierSpins) {
                    atomicOr(&B.counts[0].flags, kDevTimeout);
                    break;
                }
                __nanosleep(32);
            }
        }
    }
    __syncthreads();
}

// The substep `sub` of every world (src/world.cpp:1669-1680), in the world kernel's order. At the first
// substep the step's per-color lists over all worlds are built from the worlds' color ranges.
template <bool Joints>
__global__ void __launch_bounds__(256, 2) k_substep_flat(const __grid_constant__ Batch B, const __grid_constant__ StepParams P,
                                                      int sub, int serial) {
    const bool skip = stepAborted(B, serial);  // the same for every CTA: nothing changes it during the launch
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, threads = gridDim.x * blockDim.x;
    const uint32_t lane = threadIdx.x & 31, warp = tid >> 5, warps = threads >> 5;
    const uint32_t nw = (uint32_t)B.nWorlds, nb = B.totalBodies;
    uint32_t* colorTotal = B.work + kSlotFlatColor;
    uint32_t* impactTotal = B.work + kSlotFlatImpact;
    const FlatStore all{ B.flatBodies, B.bodies, B.flatPose, B.flatMotion };
    if (sub == 0) {
        // Every world's share of each color list, and the most colors any world has.
        if (!skip) {
            for (uint32_t w = tid; w < nw; w += threads) {
                WorldCounts& wc = B.counts[w];
                atomicMax(B.work + kSlotFlatMaxColors, wc.colorCount);
                atomicMax(B.work + kSlotFlatMaxImpact, wc.impactColorCount);
                if (wc.restLevels) { atomicMax(B.work + kSlotFlatMaxRestLevels, wc.restLevels); }
                if (wc.impactRestLevels) { atomicMax(B.work + kSlotFlatMaxImpactRestLevels, wc.impactRestLevels); }
                for (uint32_t k = 0; k < wc.colorCount; ++k) {
                    const uint32_t n = wc.colorStart[k + 1] - wc.colorStart[k];
                    wc.flatColorAt[k] = n ? atomicAdd(colorTotal + k, n) : 0u;
                }
                for (uint32_t k = 0; k < wc.impactColorCount; ++k) {
                    const uint32_t n = wc.impactColorStart[k + 1] - wc.impactColorStart[k];
                    wc.flatImpactAt[k] = n ? atomicAdd(impactTotal + k, n) : 0u;
                }
            }
        }
        gridBarrier(B);
        // The record slots, a warp per world: color k of every world from the sum of the colors before it.
        if (!skip) {
            for (uint32_t w = warp; w < nw; w += warps) {
                const WorldInfo& wi = B.info[w];
                const WorldCounts& wc = B.counts[w];
                const uint32_t cf = wi.contactFirst;
                uint32_t before = 0;
                for (uint32_t k = 0; k < wc.colorCount; ++k) {
                    const uint32_t from = before + wc.flatColorAt[k], s0 = wc.colorStart[k], s1 = wc.colorStart[k + 1];
                    for (uint32_t x = s0 + lane; x < s1; x += 32) { B.flatColored[from + (x - s0)] = cf + x; }
                    before += colorTotal[k];
                }
                before = 0;
                for (uint32_t k = 0; k < wc.impactColorCount; ++k) {
                    const uint32_t from = before + wc.flatImpactAt[k], s0 = wc.impactColorStart[k];
                    const uint32_t s1 = wc.impactColorStart[k + 1];
                    for (uint32_t x = s0 + lane; x < s1; x += 32) {
                        B.flatImpact[from + (x - s0)] = B.slotOf[cf + B.impactColored[cf + x]];
                    }
                    before += impactTotal[k];
                }
            }
        }
        gridBarrier(B);
    }
    const uint32_t colors = B.work[kSlotFlatMaxColors], impactColors = B.work[kSlotFlatMaxImpact];
    // Whether any world has contacts solved one at a time (the same for every CTA: set before a barrier).
    const bool anyRest = B.work[kSlotFlatMaxRestLevels] != 0, anyImpactRest = B.work[kSlotFlatMaxImpactRestLevels] != 0;

    // At the first substep every body's state, pose and velocity terms are staged; at a later one, the body half
    // of a refresh (planar placements kept, a new base pose) for the worlds refreshed there. Then the velocity
    // update.
    if (!skip) {
        for (uint32_t gb = tid; gb < nb; gb += threads) {
            if (sub == 0) {
                flatBegin(all, gb, P);
            } else {
                DBody& d = B.bodies[gb];
                const uint32_t w = d.world;
                if (refreshedAt(B.counts[w], sub, P.substeps)) {
                    const uint32_t pb = B.info[w].planeBody;
                    if (pb != UINT32_MAX && d.posePending) {
                        keepPose(d, placeInPlane(d, planeNormal(B.bodies[pb])));
                        d.posePending = 0;
                    }
                    const LanedBody l = all.loadLaned(gb);
                    all.put(gb, l.v, l.w, zero3(), qid(), all.flags(gb));
                    float4* q = B.flatPose + (size_t)kFlatPoseWords * gb;
                    q[3] = q[2];
                }
            }
            flatVelocity(all, gb, P);
        }
    }
    gridBarrier(B);
    auto jointsPass = [&](int kind) {
        if constexpr (Joints) {
            if (!skip) {
                for (uint32_t w = tid; w < nw; w += threads) {
                    const WorldInfo& wi = B.info[w];
                    if (wi.jointCount == 0) { continue; }
                    runJoints(B, P, wi, FlatStore{ B.flatBodies + (size_t)kFlatBodyWords * wi.bodyFirst, B.bodies + wi.bodyFirst },
                              kind);
                }
            }
            gridBarrier(B);
        }
    };
    // Each color's contacts of every world, a color at a time.
    auto colorsPass = [&](const uint32_t* list, const uint32_t* totals, uint32_t count, auto&& f) {
        uint32_t from = 0;
        for (uint32_t k = 0; k < count; ++k) {
            const uint32_t n = totals[k];
            if (!skip) {
                for (uint32_t i = tid; i < n; i += threads) { f(list[from + i]); }
            }
            from += n;
            gridBarrier(B);
        }
    };
    // A world's contacts solved on their own, level by level on one warp of the world; nothing, not even the
    // barrier, when no world has any.
    auto restPass = [&](bool impact, auto&& f) {
        if (!(impact ? anyImpactRest : anyRest)) { return; }
        if (!skip) {
            const Group g = makeGroup(32);
            for (uint32_t w = warp; w < nw; w += warps) {
                const WorldInfo& wi = B.info[w];
                const WorldCounts& wc = B.counts[w];
                const uint32_t levels = impact ? wc.impactRestLevels : wc.restLevels;
                if (levels == 0) { continue; }
                const uint32_t cf = wi.contactFirst;
                const FlatStore st{ B.flatBodies + (size_t)kFlatBodyWords * wi.bodyFirst, B.bodies + wi.bodyFirst };
                forEachLevel(g, (impact ? B.impactRest : B.rest) + cf, (impact ? B.impactRestLevel : B.restLevel) + cf,
                             levels, [&](uint32_t ci) { f(wi, wc, st, ci); });
            }
        }
        gridBarrier(B);
    };
    const uint32_t limit = nb;
    jointsPass(0);
    colorsPass(B.flatColored, colorTotal, colors, [&](uint32_t slot) { warmRowAt(B, all, 0u, limit, slot); });
    restPass(false, [&](const WorldInfo& wi, const WorldCounts& wc, const FlatStore& st, uint32_t ci) {
        warmOne(B, wi, wc, st, ci);
    });
    for (int pass = 0; pass < 2; ++pass) {
        const bool bias = pass == 0;
        jointsPass(bias ? 1 : 2);
        colorsPass(B.flatColored, colorTotal, colors, [&](uint32_t slot) { solveRowAt(B, P, all, 0u, limit, slot, bias); });
        restPass(false, [&](const WorldInfo& wi, const WorldCounts& wc, const FlatStore& st, uint32_t ci) {
            solveOne(B, P, wi, wc, st, ci, bias);
        });
        colorsPass(B.flatImpact, impactTotal, impactColors, [&](uint32_t slot) { solveRowAt(B, P, all, 0u, limit, slot, bias); });
        restPass(true, [&](const WorldInfo& wi, const WorldCounts& wc, const FlatStore& st, uint32_t ci) {
            solveOne(B, P, wi, wc, st, ci, bias);
        });
        if (bias) {
            if (!skip) {
                for (uint32_t gb = tid; gb < nb; gb += threads) { flatPosition(all, gb, P); }
            }
            gridBarrier(B);
        }
    }
    // Back into the bodies' records (the pose is there already); a world whose next substep starts with a refresh
    // takes its inverse inertia at the new pose (src/world.cpp:1660-1662), and the torque term with it.
    if (!skip) {
        for (uint32_t gb = tid; gb < nb; gb += threads) {
            const LanedBody l = all.loadLaned(gb);
            DBody& d = B.bodies[gb];
            d.v = l.v;
            d.w = l.w;
            d.dp = l.dp;
            d.dq = l.dq;
            d.qBase = quatOf(B.flatPose[(size_t)kFlatPoseWords * gb + 3]);
            if (sub + 1 < P.substeps && refreshedAt(B.counts[d.world], sub + 1, P.substeps) && d.alive &&
                d.type == kDynamic && d.awake) {
                updateInverseInertia(d);
                storeTorqueTerm(all, gb, d, P);
            }
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

// bound(): every shape's bounds at the body's pose, and the union of those that are not half-spaces
// (src/world.cpp:240-253).
static __device__ void boundBody(const Batch& B, DBody& b) {
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
}

constexpr unsigned long long kNoHit = ~0ull;

// The root of x among bodies whose unions may still be running: parents only ever point to lower bodies.
__device__ __forceinline__ uint32_t hitRoot(const uint32_t* parent, uint32_t x) {
    for (;;) {
        const uint32_t y = ((const volatile uint32_t*)parent)[x];
        if (y == x) { return x; }
        x = y;
    }
}

// Joins the groups of a and b, the higher root under the lower, so each group's root is its lowest body
// whatever order the unions run in. A link that loses a race to another is tried again, a bounded number
// of times.
static __device__ bool uniteHits(uint32_t* parent, uint32_t a, uint32_t b) {
    for (int attempt = 0; attempt < 4096; ++attempt) {
        a = hitRoot(parent, a);
        b = hitRoot(parent, b);
        if (a == b) { return true; }
        if (a > b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(&parent[b], b, a) == b) { return true; }
    }
    return false;
}

// The continuous pass of one world after the leaf refit (src/world.cpp:1271-1418). Each fast shape is swept
// against every shape whose bounds over the step meet its own; a body keeps its earliest hit (time, then pair
// order: fast shape, then other shape); dynamic bodies that hit each other form groups, and each awake
// dynamic body of a group with a hit moves back to the group's earliest hit (time, then lowest body),
// carried along by the kinematic body that hit, if one did.
// Shapes wider than this along x (and half-spaces and meshes) are tested against every fast shape.
constexpr float kWideSweep = 16.0f;

// The continuous pass of a large world: the swept bounds of shapes that are not wide are bucketed by their low
// x (a counting sort into the world's per-shape scratch), and each fast shape, a warp at a time, runs test on
// the shapes of the buckets its bounds can overlap (low x within the widest narrow shape's extent below its
// own low x, up to its high x) and on every wide shape. Each pair is visited once, as the full scan would.
template <class Test>
__device__ void sweepCandidates(const Batch& B, const Group& g, const WorldInfo& wi, uint32_t nf, Test& test) {
    __shared__ uint32_t s_minX[kMaxGroups], s_maxX[kMaxGroups], s_ext[kMaxGroups], s_wide[kMaxGroups];
    const uint32_t sf = wi.shapeFirst, ns = wi.shapeCount;
    uint32_t* order = B.rowScratch + sf;
    uint32_t* ends = B.rowLong + sf;
    uint32_t* wide = B.rowCount + sf;
    if (g.tid == 0) {
        s_minX[g.id] = orderedKey(FLT_MAX);
        s_maxX[g.id] = orderedKey(-FLT_MAX);
        s_ext[g.id] = 0;
        s_wide[g.id] = 0;
    }
    g.sync();
    auto kindOf = [&](uint32_t i) {  // 0 skipped, 1 narrow, 2 wide
        const DShape& s = B.shapes[sf + i];
        if (!s.alive || s.sensor) { return 0; }
        const float w = B.sweptHi[sf + i].x - B.sweptLo[sf + i].x;
        return (s.kind == kHalfSpace || s.kind == kMesh || !(w <= kWideSweep)) ? 2 : 1;
    };
    for (uint32_t i = g.tid; i < ns; i += g.size) {
        const int k = kindOf(i);
        if (k == 2) { wide[atomicAdd(&s_wide[g.id], 1u)] = i; }
        if (k != 1) { continue; }
        atomicMin(&s_minX[g.id], orderedKey(B.sweptLo[sf + i].x));
        atomicMax(&s_maxX[g.id], orderedKey(B.sweptHi[sf + i].x));
        atomicMax(&s_ext[g.id], __float_as_uint(B.sweptHi[sf + i].x - B.sweptLo[sf + i].x));
    }
    g.sync();
    const uint32_t buckets = max(1u, ns / 4);
    const float minX = fromOrderedKey(s_minX[g.id]), maxX = fromOrderedKey(s_maxX[g.id]);
    const float scale = (float)buckets / fmaxf(maxX - minX, 1e-6f);
    auto bucketOf = [&](float x) {
        const float t = fminf(fmaxf((x - minX) * scale, 0.0f), (float)(buckets - 1));
        return (uint32_t)t;
    };
    for (uint32_t b = g.tid; b < buckets; b += g.size) { ends[b] = 0; }
    g.sync();
    for (uint32_t i = g.tid; i < ns; i += g.size) {
        if (kindOf(i) == 1) { atomicAdd(&ends[bucketOf(B.sweptLo[sf + i].x)], 1u); }
    }
    g.sync();
    if (g.tid == 0) {
        uint32_t sum = 0;
        for (uint32_t b = 0; b < buckets; ++b) {
            const uint32_t n = ends[b];
            ends[b] = sum;  // the bucket's fill position, its end once filled
            sum += n;
        }
    }
    g.sync();
    for (uint32_t i = g.tid; i < ns; i += g.size) {
        if (kindOf(i) == 1) { order[atomicAdd(&ends[bucketOf(B.sweptLo[sf + i].x)], 1u)] = i; }
    }
    g.sync();
    // Padded, so that rounding in the widths and the subtraction below never drops a pair.
    const float ext = __uint_as_float(s_ext[g.id]) * 1.001f + 1e-3f;
    const uint32_t nWide = s_wide[g.id];
    for (uint32_t k = g.warp; k < nf; k += g.warps) {
        const uint32_t fi = B.sweepList[sf + k];
        const uint32_t b0 = bucketOf(B.sweptLo[sf + fi].x - ext), b1 = bucketOf(B.sweptHi[sf + fi].x);
        const uint32_t from = b0 > 0 ? ends[b0 - 1] : 0u, to = ends[b1];
        for (uint32_t p = from + g.lane; p < to; p += 32) { test(k, order[p]); }
        for (uint32_t p = g.lane; p < nWide; p += 32) { test(k, wide[p]); }
    }
}

static __device__ void sweepWorld(const Batch& B, const StepParams& P, const Group& g, const WorldInfo& wi, WorldCounts& wc,
                           uint32_t* pairs, uint32_t* impacts) {
    const uint32_t sf = wi.shapeFirst, ns = wi.shapeCount, bf = wi.bodyFirst, nb = wi.bodyCount;
    uint32_t* parent = B.hitParent + bf;
    for (uint32_t i = g.tid; i < ns; i += g.size) {
        const DShape& s = B.shapes[sf + i];
        Vec3 lo = s.lo, hi = s.hi;
        if (s.alive && B.bodies[s.body].type != kStatic) {
            Vec3 l, h;
            shapeBounds(s, B.cx.pt, sweepAt(sweepOf(B.bodies[s.body]), 0.0f) * s.local, l, h);
            lo = minVec(lo, l);
            hi = maxVec(hi, h);
        }
        B.sweptLo[sf + i] = lo;
        B.sweptHi[sf + i] = hi;
    }
    for (uint32_t i = g.tid; i < nb; i += g.size) {
        B.hitKey[bf + i] = kNoHit;
        B.groupKey[bf + i] = kNoHit;
        parent[i] = i;
    }
    const uint32_t nf = groupCompact(
        g, ns,
        [&](uint32_t i) {
            const DShape& s = B.shapes[sf + i];
            if (!s.alive || !TF_OK_INDEX(B, s.body - bf < nb, 32, bf, i)) { return false; }
            const DBody& b = B.bodies[s.body];
            if (!b.alive || b.type != kDynamic || !b.awake) { return false; }
            return sweepsShape(B.cx.pt, s, b, length(b.com - b.com0), sweepOf(b).angle);
        },
        [&](uint32_t i, uint32_t pos) { B.sweepList[sf + pos] = i; });
    const float target = P.tol.linearSlop;
    // Fast shape k against shape oi; x = k ns + oi orders equal hit times, whatever order the pairs run in.
    auto testPair = [&](uint32_t k, uint32_t oi) {
        const unsigned long long x = (unsigned long long)k * ns + oi;
        const uint32_t fi = B.sweepList[sf + k];
        const DShape& f = B.shapes[sf + fi];
        const DShape& o = B.shapes[sf + oi];
        if (!o.alive || o.sensor || o.body == f.body) { return; }
        if (!TF_OK_INDEX(B, o.body - bf < nb, 33, bf, oi)) { return; }
        if (joinedBodies(B, wi, o.body, f.body)) { return; }
        if (!boxesOverlap(B.sweptLo[sf + fi], B.sweptHi[sf + fi], B.sweptLo[sf + oi], B.sweptHi[sf + oi])) { return; }
        if (!(f.category & o.mask) || !(o.category & f.mask)) { return; }
        atomicAdd(pairs, 1u);
        const DBody& bo = B.bodies[o.body];
        float t = 1.0f;
        bool ok = true;
        const bool hit = sweepPair(B.cx, f, B.bodies[f.body], o, bo, B.sweptLo[sf + fi], B.sweptHi[sf + fi], target, t, ok);
        if (!ok) { atomicOr(&wc.flags, kDevUnsupported); }
        if (!hit) { return; }
        const unsigned long long order = x < 0xffffffffull ? x : 0xfffffffeull;
        atomicMin(&B.hitKey[f.body], ((unsigned long long)__float_as_uint(t) << 32) | order);
        if (bo.type == kDynamic && !uniteHits(parent, f.body - bf, o.body - bf)) { atomicOr(&wc.flags, kDevTimeout); }
    };
    if (ns <= kSweepBodies || nf <= 32) {
        const unsigned long long total = (unsigned long long)nf * ns;
        for (unsigned long long x = g.tid; x < total; x += g.size) { testPair((uint32_t)(x / ns), (uint32_t)(x % ns)); }
    } else {
        sweepCandidates(B, g, wi, nf, testPair);
    }
    g.sync();
    for (uint32_t i = g.tid; i < nb; i += g.size) {
        const unsigned long long hk = B.hitKey[bf + i];
        if (hk == kNoHit) { continue; }
        atomicMin(&B.groupKey[bf + rootOf(parent, i)], (hk & 0xffffffff00000000ull) | i);
    }
    g.sync();
    for (uint32_t i = g.tid; i < nb; i += g.size) {
        const unsigned long long gk = B.groupKey[bf + rootOf(parent, i)];
        if (gk == kNoHit) { continue; }
        const float t = __uint_as_float((uint32_t)(gk >> 32));
        DBody& b = B.bodies[bf + i];
        if (t >= 1.0f || !b.alive || b.type != kDynamic || !b.awake) { continue; }
        // The member whose hit came first, and what it hit.
        const unsigned long long first = B.hitKey[bf + (uint32_t)gk];
        const uint32_t oi = (uint32_t)((first & 0xffffffffull) % ns);
        const DBody& other = B.bodies[B.shapes[sf + oi].body];
        b.xf = sweepAt(sweepOf(b), t);
        if (other.type == kKinematic) {
            // A kinematic body keeps moving after the hit, so what hit it rides along to the end of the step.
            const Transform k = sweepAt(sweepOf(other), t);
            const Transform ride{ applyInverse(k, b.xf.p), normalize(conjugate(k.q) * b.xf.q) };
            b.xf = other.xf * ride;
        }
        b.com = apply(b.xf, b.localCenter);
        updateInverseMass(b);
        boundBody(B, b);
        atomicAdd(impacts, 1u);
    }
    g.sync();
}

// Union-find is staged in the group's shared slice (parent and island time by body, union pairs by contact)
// when the world fits, else in its global scratch.
// After the solve (src/world.cpp:1685-1691): active joints turn the step's impulses into a force and torque
// and break past their limits (src/world.cpp:1543-1560), the rest settle positions in order, twice over, and
// every awake dynamic body's world inverse mass is built again at its settled pose. One thread runs the
// joints; every thread first finds whether any joint was active.
static __device__ void finishJoints(const Batch& B, const StepParams& P, const Group& g, const WorldInfo& wi) {
    DJoint* js = B.joints + wi.jointFirst;
    auto endOf = [&](uint32_t gbody) { return gbody == kWorldEnd ? worldEnd() : jointBodyOf(B.bodies[gbody]); };
    bool anyActive = false;
    for (uint32_t x = 0; x < wi.jointCount && !anyActive; ++x) {
        anyActive = jointActive(js[x], endOf(js[x].bodyA), endOf(js[x].bodyB));
    }
    g.sync();
    if (!anyActive) { return; }
    if (g.tid == 0) {
        for (uint32_t x = 0; x < wi.jointCount; ++x) {
            DJoint& j = js[x];
            if (!jointActive(j, endOf(j.bodyA), endOf(j.bodyB))) { continue; }
            j.force = j.force / P.dt;
            j.torque = j.torque / P.dt;
            if (length(j.force) > j.breakForce || length(j.torque) > j.breakTorque) {
                j.broken = 1;
                j.brokeNow = 1;
                j.linearImpulse = zero3();
                j.angularImpulse = zero3();
                j.frictionTurn = zero3();
                j.axialImpulse = j.motorImpulse = j.lowerImpulse = j.upperImpulse = 0.0f;
                j.frictionImpulse = j.swingImpulse = 0.0f;
            }
        }
        auto putPose = [&](uint32_t gbody, const JBody& e) {
            if (gbody == kWorldEnd || e.type != kDynamic || !e.awake) { return; }
            B.bodies[gbody].com = e.com;
            B.bodies[gbody].xf = e.xf;
        };
        for (int it = 0; it < kSettleIterations; ++it) {
            for (uint32_t x = 0; x < wi.jointCount; ++x) {
                const DJoint& j = js[x];
                JBody a = endOf(j.bodyA), b = endOf(j.bodyB);
                if (!jointActive(j, a, b)) { continue; }
                settleJoint(a, b, j);
                putPose(j.bodyA, a);
                putPose(j.bodyB, b);
            }
        }
    }
    g.sync();
    for (uint32_t i = g.tid; i < wi.bodyCount; i += g.size) {
        DBody& b = B.bodies[wi.bodyFirst + i];
        if (b.alive && b.type == kDynamic && b.awake) { updateInverseMass(b); }
    }
    g.sync();
}

// Counts the touching contacts, reports the pairs that began or stopped touching and the fastest struck point
// of each touching pair (src/world.cpp:1424-1468). The first contact of each pair walks the pair's contacts:
// a pair touches where the solver pushed on a point or a point overlaps (by more than the linear slop once it
// touched); a hit is a pushed point approaching faster than the threshold in a contact solved this step.
// Runs after restitution, on the poses the solve left, before kinematic bodies snap to their targets.
static __device__ void reportTouches(const Batch& B, const StepParams& P, const Group& g, const WorldInfo& wi, WorldCounts& wc) {
    const uint32_t nc = wc.contactCount;
    DContact* cs = B.contacts + wi.contactFirst;
    uint32_t touchingHere = 0;
    for (uint32_t first = g.tid; first < nc; first += g.size) {
        const uint64_t key = cs[first].key;
        if (first > 0 && cs[first - 1].key == key) { continue; }
        const bool was = (cs[first].flags & kCTouched) != 0;
        const float apart = was ? P.tol.linearSlop : 0.0f;
        bool touching = false;
        float fastest = P.hitThreshold;
        uint32_t struck = UINT32_MAX;
        int point = 0;
        uint32_t last = first;
        for (; last < nc && cs[last].key == key; ++last) {
            const DContact& c = cs[last];
            bool pressed = false;
            for (int i = 0; i < c.count; ++i) {
                pressed = pressed || c.points[i].separation < 0.0f || c.points[i].normalImpulse > 0.0f;
            }
            touchingHere += pressed ? 1u : 0u;
            if (!TF_OK_INDEX(B, c.bodyA - wi.bodyFirst < wi.bodyCount && c.bodyB - wi.bodyFirst < wi.bodyCount, 22,
                             wi.bodyFirst, last)) {
                continue;
            }
            const DBody& a = B.bodies[c.bodyA];
            const DBody& b = B.bodies[c.bodyB];
            const bool solved = (a.type == kDynamic && a.awake) || (b.type == kDynamic && b.awake);
            for (int i = 0; i < c.count; ++i) {
                const DPoint& p = c.points[i];
                if (p.maxNormalImpulse > 0.0f) {
                    touching = true;
                    if (-p.relativeVelocity > fastest && solved) {
                        fastest = -p.relativeVelocity;
                        struck = last;
                        point = i;
                    }
                } else if (p.separation < apart) {
                    touching = true;
                }
            }
        }
        if (touching != was) {
            const uint32_t at = atomicAdd(&wc.touchEvents, 1u);
            B.touchEvents[2 * (size_t)wi.contactFirst + at] = TouchEvent{ key, touching ? 1u : 0u, 1u };
            for (uint32_t k = first; k < last; ++k) {
                cs[k].flags = touching ? (cs[k].flags | kCTouched) : (cs[k].flags & ~kCTouched);
            }
        }
        if (struck != UINT32_MAX) {
            const DContact& c = cs[struck];
            const uint32_t at = atomicAdd(&wc.hitEvents, 1u);
            B.hitEvents[(size_t)wi.contactFirst + at] =
                HitRecord{ key, apply(B.bodies[c.bodyA].xf, c.points[point].localA), c.normal, fastest, 0u };
        }
    }
    if (touchingHere > 0) { atomicAdd(&wc.touching, touchingHere); }
}

template <bool Joints>
__global__ void __launch_bounds__(kMaxBlock) k_finish(const __grid_constant__ Batch B, const __grid_constant__ StepParams P, const __grid_constant__ Split sp, int serial) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    __shared__ uint32_t s_awake[kMaxGroups], s_islands[kMaxGroups], s_sweep[kMaxGroups], s_pairs[kMaxGroups],
        s_impacts[kMaxGroups], s_linked[kMaxGroups];
    if (stepAborted(B, serial)) { return; }
    forWorlds(B, kSlotFinish, sp, s_raw, [&](const Group& g, uint32_t w, unsigned char* slice, const StageSizes& ss) {
        const uint32_t stageBodies = ss.bodies, stageContacts = ss.contacts;
        const WorldInfo wi = B.info[w];
        WorldCounts& wc = B.counts[w];
        const uint32_t cf = wi.contactFirst;
        DContact* cs = B.contacts + cf;
        const Axis* axes = B.axes + (size_t)cf * kAxesPerContact;
        if (g.tid == 0) {
            s_awake[g.id] = 0;
            s_islands[g.id] = 0;
            s_sweep[g.id] = 0;
        }
        // The laned contacts' impulses come back from their records.
        const uint32_t nColored = wc.colorStart[kColors];
        for (uint32_t x = g.tid; x < nColored; x += g.size) {
            const uint32_t ci = __float_as_uint(B.rows[kRowHead * B.rowStride + cf + x].w);
            if (!contactOk(B, wi, wc, ci, 18)) { continue; }
            returnImpulses(B, cf + x, cs[ci]);
        }
        g.sync();
        // Restitution: colored contacts by color (their normal axes built again as the record's passes build
        // them), then the rest in active order.
        forEachColor(g, B.colored + cf, wc.colorStart, wc.colorCount, [&](uint32_t ci) {
            if (!contactOk(B, wi, wc, ci, 18)) { return; }
            DContact& c = cs[ci];
            restituteLaned(B.bodies[c.bodyA], B.bodies[c.bodyB], c, P);
        });
        forEachLevel(g, B.rest + cf, B.restLevel + cf, wc.restLevels, [&](uint32_t ci) {
            if (!contactOk(B, wi, wc, ci, 20)) { return; }
            DContact& c = cs[ci];
            restituteContact(B.bodies[c.bodyA], B.bodies[c.bodyB], c, P, false, axes + (size_t)ci * kAxesPerContact);
        });
        if constexpr (Joints) {
            if (wi.jointCount > 0) { finishJoints(B, P, g, wi); }
        }
        reportTouches(B, P, g, wi, wc);
        g.sync();
        const uint32_t nc = wc.contactCount;
        const bool staged = wi.bodyCount <= stageBodies && nc <= stageContacts;
        uint32_t* parent = staged ? reinterpret_cast<uint32_t*>(slice) : B.unionParent + wi.bodyFirst;
        uint32_t* islandTime = staged ? parent + stageBodies : reinterpret_cast<uint32_t*>(B.islandTime + wi.bodyFirst);
        uint32_t* uA = staged ? islandTime + stageBodies : B.mergeIdxA + cf;
        uint32_t* uB = staged ? uA + stageContacts : B.mergeIdxB + cf;
        const float threshold = P.sleepThreshold;
        for (uint32_t i = g.tid; i < wi.bodyCount; i += g.size) {
            const uint32_t gb = wi.bodyFirst + i;
            DBody& b = B.bodies[gb];
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
                // Leaf refit over the new pose (src/world.cpp:1713-1718).
                boundBody(B, b);
                // Shapes that moved well past what the speculative contacts covered are swept against their
                // surroundings below (src/world.cpp:1280-1292).
                if (P.continuous && b.type == kDynamic && b.awake) {
                    const float moved = length(b.com - b.com0);
                    const float angle = sweepOf(b).angle;
                    for (uint32_t x = 0; x < b.shapeCount; ++x) {
                        const DShape& s = B.shapes[B.shapeList[b.shapeFirst + x]];
                        if (sweepsShape(B.cx.pt, s, b, moved, angle)) { atomicAdd(&s_sweep[g.id], 1u); }
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
        g.sync();
        if (g.tid == 0) {
            s_pairs[g.id] = 0;
            s_impacts[g.id] = 0;
        }
        if (P.continuous && s_sweep[g.id] > 0) { sweepWorld(B, P, g, wi, wc, &s_pairs[g.id], &s_impacts[g.id]); }
        // Islands over contacts with points (src/world.cpp:1187-1233). The roots are each component's lowest
        // body whatever order the unions run in, so only the unions themselves run on one thread.
        const uint32_t nu = groupCompact(
            g, nc,
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
        // The unions run in parallel: each round links the higher of a pair's roots under the lower (parents
        // only ever point to lower bodies, so an atomicMin keeps the lowest link), then points every body at
        // its root, until a round links nothing. Each component ends rooted at its lowest body, which is what
        // the reference's sequential unions give.
        for (;;) {
            if (g.tid == 0) { s_linked[g.id] = 0; }
            g.sync();
            for (uint32_t x = g.tid; x < nu; x += g.size) {
                if (!TF_OK_INDEX(B, uA[x] < wi.bodyCount && uB[x] < wi.bodyCount, 24, w, x)) { continue; }
                const uint32_t ra = rootOf(parent, uA[x]), rb = rootOf(parent, uB[x]);
                if (ra != rb) {
                    atomicMin(&parent[ra > rb ? ra : rb], ra < rb ? ra : rb);
                    s_linked[g.id] = 1;
                }
            }
            g.sync();
            const bool again = s_linked[g.id] != 0;
            for (uint32_t i = g.tid; again && i < wi.bodyCount; i += g.size) { parent[i] = rootOf(parent, i); }
            g.sync();
            if (!again) { break; }
        }
        if (g.tid == 0) {
            // Joints that hold link their bodies too (src/world.cpp:1210-1222).
            const DJoint* js = B.joints + wi.jointFirst;
            for (uint32_t x = 0; x < wi.jointCount; ++x) {
                const DJoint& j = js[x];
                if (!j.alive || j.broken) { continue; }
                DBody* a = j.bodyA == kWorldEnd ? nullptr : &B.bodies[j.bodyA];
                DBody& b = B.bodies[j.bodyB];
                const bool da = a && a->type == kDynamic && a->awake;
                const bool db = b.type == kDynamic && b.awake;
                if (da && db) {
                    const uint32_t ra = findRoot(parent, j.bodyA - wi.bodyFirst), rb = findRoot(parent, j.bodyB - wi.bodyFirst);
                    if (ra != rb) { parent[ra > rb ? ra : rb] = ra < rb ? ra : rb; }
                } else if (da && b.type == kKinematic && movingAwake(b)) {
                    a->sleepTime = 0.0f;
                } else if (db && a && a->type == kKinematic && movingAwake(*a)) {
                    b.sleepTime = 0.0f;
                }
            }
        }
        g.sync();
        for (uint32_t i = g.tid; i < wi.bodyCount; i += g.size) {
            DBody& b = B.bodies[wi.bodyFirst + i];
            if (!b.alive || b.type != kDynamic || !b.awake) { continue; }
            const uint32_t r = rootOf(parent, i);
            b.island = r;
            atomicAdd(&s_awake[g.id], 1u);
            if (r == i) { atomicAdd(&s_islands[g.id], 1u); }
            atomicMin(&islandTime[r], __float_as_uint(b.sleepTime));
        }
        g.sync();
        for (uint32_t i = g.tid; i < wi.bodyCount; i += g.size) {
            DBody& b = B.bodies[wi.bodyFirst + i];
            if (!b.alive || b.type != kDynamic || !b.awake) { continue; }
            if (__uint_as_float(islandTime[rootOf(parent, i)]) < P.timeToSleep) { continue; }
            b.awake = 0;
            b.v = zero3();
            b.w = zero3();
            updateInverseMass(b);
        }
        g.sync();
        if (g.tid == 0) {
            wc.awakeBodies = s_awake[g.id];
            wc.awakeIslands = s_islands[g.id];
            wc.bodySteps += s_awake[g.id];
            wc.sweepShapes += s_sweep[g.id];
            wc.sweptPairs = s_pairs[g.id];
            wc.impacts = s_impacts[g.id];
        }
        g.sync();
    });
}
// ---------------------------------------------------------------------------------------------------------
// Host traffic of a running batch: per-step forces in, poses out.

// World::addForce / addTorque with wake = false on every body (src/world.cpp:2118-2142).
// Records what this step's solve will see, right after preparation: every contact of every world with its
// lists and the awake dynamic bodies. One group per world.
template <int Unused = 0>
__global__ void __launch_bounds__(kMaxBlock) k_tape_record(const __grid_constant__ Batch B, const __grid_constant__ Split sp,
                                                           TapeStep T, int serial) {
    if (stepAborted(B, serial)) { return; }
    forWorlds(B, kSlotTape, sp, nullptr, [&](const Group& g, uint32_t w, unsigned char*, const StageSizes&) {
        const WorldInfo wi = B.info[w];
        const WorldCounts& wc = B.counts[w];
        const uint32_t cf = wi.contactFirst;
        if (g.tid == 0) {
            TapeWorld& tw = T.worlds[w];
            tw.contactFirst = cf;
            tw.contactCount = wc.contactCount;
            tw.colorCount = wc.colorCount;
            tw.impactColorCount = wc.impactColorCount;
            tw.restCount = wc.restCount;
            tw.impactRestCount = wc.impactRestCount;
            for (int k = 0; k < kTapeColors; ++k) {
                tw.colorStart[k] = wc.colorStart[k];
                tw.impactColorStart[k] = wc.impactColorStart[k];
            }
        }
        for (uint32_t i = g.tid; i < wc.contactCount; i += g.size) {
            const DContact& c = B.contacts[cf + i];
            TapeContact t;
            t.a = c.bodyA - wi.bodyFirst;
            t.b = c.bodyB - wi.bodyFirst;
            t.shapeA = c.shapeA - wi.shapeFirst;
            t.shapeB = c.shapeB - wi.shapeFirst;
            t.count = c.count;
            t.restitution = c.restitution;
            const Vec3 dirs[3] = { c.normal, c.tangent1, c.tangent2 };
            float* out[3] = { t.normal, t.t1, t.t2 };
            for (int d = 0; d < 3; ++d) {
                out[d][0] = dirs[d].x;
                out[d][1] = dirs[d].y;
                out[d][2] = dirs[d].z;
            }
            for (int k = 0; k < 4; ++k) {
                const DPoint& p = c.points[k];
                const bool on = k < c.count;
                t.anchorA[k][0] = on ? p.anchorA.x : 0.0f, t.anchorA[k][1] = on ? p.anchorA.y : 0.0f;
                t.anchorA[k][2] = on ? p.anchorA.z : 0.0f;
                t.anchorB[k][0] = on ? p.anchorB.x : 0.0f, t.anchorB[k][1] = on ? p.anchorB.y : 0.0f;
                t.anchorB[k][2] = on ? p.anchorB.z : 0.0f;
                t.adjSep[k] = on ? p.adjustedSeparation : 0.0f;
                t.relVel[k] = on ? p.relativeVelocity : 0.0f;
                t.normalImpulse[k] = on ? p.normalImpulse : 0.0f;
                t.tangentImpulse[k][0] = on ? p.tangentImpulse.x : 0.0f;
                t.tangentImpulse[k][1] = on ? p.tangentImpulse.y : 0.0f;
                t.tangentImpulse[k][2] = on ? p.tangentImpulse.z : 0.0f;
            }
            T.contacts[cf + i] = t;
        }
        const uint32_t nColored = wc.colorStart[wc.colorCount], nImpact = wc.impactColorStart[wc.impactColorCount];
        for (uint32_t x = g.tid; x < nColored; x += g.size) { T.colored[cf + x] = B.colored[cf + x]; }
        for (uint32_t x = g.tid; x < nImpact; x += g.size) { T.impactColored[cf + x] = B.impactColored[cf + x]; }
        for (uint32_t x = g.tid; x < wc.restCount; x += g.size) { T.rest[cf + x] = B.rest[cf + x]; }
        for (uint32_t x = g.tid; x < wc.impactRestCount; x += g.size) { T.impactRest[cf + x] = B.impactRest[cf + x]; }
        for (uint32_t i = g.tid; i < wi.bodyCount; i += g.size) {
            T.awake[wi.bodyFirst + i] = movingBody(B.bodies[wi.bodyFirst + i]) ? 1 : 0;
        }
        g.sync();
    });
}

template <int Unused = 0>
__global__ void k_add_forces(DBody* bodies, uint32_t n, const float* __restrict__ f, const float* __restrict__ t) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) { return; }
    DBody& b = bodies[i];
    if (!b.alive || b.type != kDynamic || !b.awake) { return; }
    if (f) { b.force += Vec3{ f[3 * i], f[3 * i + 1], f[3 * i + 2] }; }
    if (t) { b.torque += Vec3{ t[3 * i], t[3 * i + 1], t[3 * i + 2] }; }
}

// What the host checks after every step, from every world's counts in one CTA: the OR of the worlds' flags
// and the sum of their body steps (out[0] flags, out[1..2] the sum's low and high words).
template <int Unused = 0>
__global__ void __launch_bounds__(256) k_step_summary(const WorldCounts* counts, uint32_t nWorlds, uint32_t* out) {
    __shared__ uint32_t s_flags;
    __shared__ unsigned long long s_steps;
    if (threadIdx.x == 0) {
        s_flags = 0;
        s_steps = 0;
    }
    __syncthreads();
    uint32_t flags = 0;
    unsigned long long steps = 0;
    for (uint32_t w = threadIdx.x; w < nWorlds; w += blockDim.x) {
        flags |= counts[w].flags;
        steps += counts[w].bodySteps;
    }
    atomicOr(&s_flags, flags);
    atomicAdd(&s_steps, steps);
    __syncthreads();
    if (threadIdx.x == 0) {
        out[0] = s_flags;
        out[1] = (uint32_t)s_steps;
        out[2] = (uint32_t)(s_steps >> 32);
    }
}

template <int Unused = 0>
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

