// Every device array of a batch, passed by value to each kernel.
#pragma once

#include "tf_dispatch.cuh"
#include "tf_mesh_collide.cuh"
#include "tf_solver.cuh"
#include "tf_types.cuh"

namespace tfb {

// A body of a big world as the sweep reads it, stored in bucket order: its pair-test record, where its
// interval along x starts, and which body it is.
struct SweepRec {
    Vec3 lo, hi;
    float grow;
    uint32_t flags;
    float start;
    uint32_t body;
};

struct Batch {
    int nWorlds;
    const uint32_t* order;  // worlds, largest first; CTA k takes order[k], order[k + gridDim.x], ...
    const WorldInfo* info;
    WorldCounts* counts;
    // Index (within the current launch sequence) of the first step that overflowed a list; later kernels
    // of that step and every step after it do nothing, so the host can grow the lists and run it again.
    uint32_t* abortStep;

    DBody* bodies;
    DShape* shapes;
    const uint32_t* shapeList;  // per body, its shapes (global indices)
    const uint32_t* planeList;  // per world, its half-space shapes (global indices)
    CollideCtx cx;

    // Per body.
    float* grow;
    uint32_t* bodyColors;
    uint8_t* struck;
    uint8_t* wakeMark;
    uint32_t* unionParent;
    float* islandTime;

    // Per candidate (candFirst + i): the key, its first contact, how many contacts it made (more than one for
    // a mesh pair), and where the ones after the first went (partFirst + stagePart[i], in stageExtra).
    uint64_t* cand;
    DContact* stage;
    uint8_t* stageUsed;
    uint32_t* stagePart;
    DContact* stageExtra;
    // Per world (boundsFirst + i): triangles fast mesh pairs ruled out, each pair's run sorted by triangle.
    TriangleBound* triBounds;

    // Per contact slot (contactFirst + i). Contacts double-buffer across steps.
    DContact* contacts;   // current
    DContact* previous;   // last step's, read while the current list is built
    uint32_t* active;
    uint32_t* impact;
    uint32_t* colored;        // active contacts grouped by color
    uint32_t* impactColored;
    uint32_t* rest;           // active contacts solved one at a time, in active order
    uint32_t* impactRest;
    uint32_t* restLevel;        // each level's end in the rest list
    uint32_t* impactRestLevel;
    uint8_t* color;           // by contact
    Axis* axes;               // by contact, kAxesPerContact each; built for the contacts solved one at a time
    // The laned contacts' solver records: kRowWords float4 components, component k of slot s at
    // rows[k * rowStride + s], a laned contact's slot being contactFirst + its position in the world's colored
    // list; slotOf maps a contact (contactFirst + i) to its slot.
    float4* rows;
    size_t rowStride;
    uint32_t* slotOf;
    // The flat solve of batches of many worlds: every body's solver state (kFlatBodyWords float4 per body:
    // velocity, spin, displacement and turn of the substep, type and awake flags), and per color the record
    // slots of that color's contacts in every world (color k from the batch-wide start of color k, both lists
    // totalling at most one entry per contact slot).
    float4* flatBodies;
    float4* flatPose;    // kFlatPoseWords float4 per body
    float4* flatMotion;  // kFlatMotionWords float4 per body
    uint32_t* flatColored;
    uint32_t* flatImpact;
    uint8_t* cflags;          // by contact: kFast, kFastSolid
    uint64_t* mergeKeyA;
    uint32_t* mergePartA;
    uint32_t* mergeIdxA;
    uint64_t* mergeKeyB;
    uint32_t* mergePartB;
    uint32_t* mergeIdxB;
    // Joints and joined body pairs, per world from jointFirst.
    DJoint* joints;
    const uint64_t* joined;
    // The step's events: contact events from 2 * contactFirst (room for the pairs the narrowphase dropped
    // and for the end-of-step report), hits from contactFirst.
    TouchEvent* touchEvents;
    HitRecord* hitEvents;

    // Flat work lists, filled as the step goes, each item a (world, index within the world) pair. Candidate
    // pairs, one list per pair class (candItemStride apart), for the pair collisions; the active contacts of
    // worlds refreshed mid-step, one list per pair class of fast contacts and one more for the rest
    // (contactItemStride apart). Their lengths are the work counters from kSlotCandItems and kSlotFastItems.
    uint2* candItems;
    uint2* contactItems;
    uint32_t candItemStride, contactItemStride;

    uint32_t* work;        // per launch of a step, the next world to hand out (zeroed when the step starts)
    uint32_t* rowScratch;  // per shape, the candidate key sort's row counts
    uint32_t* rowLong;     // per shape, the sort's long rows
    uint32_t* rowCount;    // per shape, the sort's counts within one long row

    // Broadphase of worlds of more than kSweepBodies bodies: per body its interval along x (sweepLo, sweepHi)
    // and, from bodyFirst, the bodies bucketed by the interval's start (sweepOrder); per world, from
    // bodyFirst + world, the buckets' starts (sweepStart). bigWorlds lists those worlds, bigBodyStart the
    // running total of their bodies.
    float* sweepLo;
    float* sweepHi;
    uint32_t* sweepOrder;
    struct SweepRec* sweepRecs;  // per body, from bodyFirst, in bucket order: what the pair test reads
    uint32_t* sweepStart;
    const uint32_t* bigWorlds;
    const uint32_t* bigBodyStart;
    uint32_t nBigWorlds;

    // Continuous collision: per shape, its bounds over the whole step and (from shapeFirst) the world's fast
    // shapes in shape order; per body, its earliest hit as (time bits << 32 | pair order), its group's
    // earliest as (time bits << 32 | body), and the union-find parent of the bodies that hit one another.
    Vec3* sweptLo;
    Vec3* sweptHi;
    uint32_t* sweepList;
    unsigned long long* hitKey;
    unsigned long long* groupKey;
    uint32_t* hitParent;

    // Debug builds (TF_DEVICE_CHECKS) record the first failed index check here: code, world, value.
    uint32_t* debug;
    uint32_t nPolys;
    uint32_t totalBodies;
};

#if defined(TF_DEVICE_CHECKS)
// Records the first failure and evaluates to false so the caller skips the access.
#define TF_OK_INDEX(B, cond, code, world, value)                                                     \
    ((cond) ? true                                                                                  \
            : (atomicCAS(&(B).debug[0], 0u, (uint32_t)(code)) == 0u                                 \
                   ? ((B).debug[1] = (uint32_t)(world), (B).debug[2] = (uint32_t)(value), false)    \
                   : false))
#else
#define TF_OK_INDEX(B, cond, code, world, value) true
#endif

constexpr uint8_t kFlagFast = 1, kFlagFastSolid = 2, kFlagActive = 4;

}
