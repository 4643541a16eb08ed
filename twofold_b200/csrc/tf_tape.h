// The record of a forward run that the adjoint replays, shared by the step pipeline (which writes it) and
// the differentiable model (which reads it).
//
// The model holds each step's contact set fixed: per step it keeps what the solve saw after preparation
// (src/solver.cpp:264-291 in the reference): the contacts with their anchors, frames, adjusted separations,
// approach speeds and warm-start impulses, the color lists the solve walked, and which bodies were awake.
#pragma once

#include <cstdint>

namespace tfb {

constexpr int kTapeColors = 33;

// One contact of a recorded step, world-local body and shape indices.
struct TapeContact {
    uint32_t a, b;
    uint32_t shapeA, shapeB;
    int32_t count;
    float restitution;
    float normal[3], t1[3], t2[3];
    float anchorA[4][3], anchorB[4][3];
    float adjSep[4], relVel[4];
    float normalImpulse[4];
    float tangentImpulse[4][3];
};

// One world of a recorded step. Lists and contacts of the world start at contactFirst in the step's arrays.
struct TapeWorld {
    uint32_t contactFirst, contactCount;
    uint32_t colorCount, impactColorCount, restCount, impactRestCount;
    uint32_t colorStart[kTapeColors];
    uint32_t impactColorStart[kTapeColors];
};

// Device arrays of one recorded step. Contacts and the four lists are indexed contactFirst + i; awake by
// batch body index (1 for a dynamic body that was awake in the step).
struct TapeStep {
    TapeWorld* worlds;
    TapeContact* contacts;
    uint32_t* colored;
    uint32_t* impactColored;
    uint32_t* rest;
    uint32_t* impactRest;
    uint8_t* awake;
};

// Everything the differentiable model needs, as device pointers (batch body and shape order).
struct AdjointSetup {
    int nWorlds;
    int nSteps;
    uint32_t totalBodies, totalShapes, contactSlots;  // contactSlots: the largest per-step contact arrays
    const uint32_t* bodyFirst;   // per world
    const uint32_t* bodyCount;
    const uint32_t* shapeFirst;
    const TapeStep* steps;       // nSteps entries, device array
    // Per body: 1 when dynamic; gravity scale and damping; mass and local inverse inertia at that mass.
    const uint8_t* dynamic;
    const float* gravityScale;
    const float* linearDamping;
    const float* angularDamping;
    const float* mass;
    const float* invInertiaLocal;  // 9 per body, row-major
    // The recorded initial state per body: center of mass, rotation (x, y, z, w), velocities.
    const float* com0;
    const float* q0;
    const float* v0;
    const float* w0;
    const float* friction;  // per shape
    // Settings of the recorded run.
    float gravity[3];
    float dt;
    int substeps;
    float contactSoft[3], staticSoft[3];  // bias rate, mass scale, impulse scale
    float maxPushout;
    float restitutionThreshold;
};

}  // namespace tfb
