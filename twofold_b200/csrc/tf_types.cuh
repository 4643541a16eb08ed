// Device-resident state of a batch of worlds.
//
// Bodies, shapes and contacts are arrays of plain structs in HBM, one segment per world. Their fields
// follow the reference's Body (src/internal.h:257-325), Shape (:152-187) and Contact (:428-503) so each
// kernel reads like the step it restates; the structs hold no pointers and copy to and from the host as
// bytes. Indices stored in bodies, shapes and contacts are global (across the batch); contact keys use
// the world-local shape indices, as the reference's keys do (src/world.cpp:42).
#pragma once

#include "tf_math.cuh"

namespace tfb {

enum BodyType : uint32_t { kStatic = 0, kKinematic = 1, kDynamic = 2 };

// ShapeKind (src/internal.h:113).
enum ShapeKind : uint32_t { kSphere = 0, kConvex = 1, kHalfSpace = 2, kMesh = 3, kCylinder = 4 };

// Feature::Kind (src/internal.h:335).
enum FeatureKind : int32_t { kFeatNone = 0, kFeatFaceA = 1, kFeatFaceB = 2, kFeatEdges = 3 };

constexpr uint32_t kLockTX = 1u << 0, kLockTY = 1u << 1, kLockTZ = 1u << 2;
constexpr uint32_t kLockRX = 1u << 3, kLockRY = 1u << 4, kLockRZ = 1u << 5;
constexpr uint32_t kLockPlanar = kLockTZ | kLockRX | kLockRY;

constexpr int kColors = 32;
constexpr int kNoColor = kColors;

struct alignas(16) DBody {
    // Read and written by every solve.
    Vec3 v;
    Vec3 w;
    Vec3 dp;
    Quat dq;
    Mat3 invMassWorld;
    Mat3 invInertiaWorld;
    float invMass;
    float planeInvMass;
    float planeInvInertia;
    uint32_t type;
    uint32_t awake;
    uint32_t alive;

    Transform xf;
    Vec3 com;
    Vec3 localCenter;
    float extent;
    Vec3 force;
    Vec3 torque;
    float mass;
    Mat3 inertia;
    float linearDamping;
    float angularDamping;
    float gravityScale;
    uint32_t locks;
    Quat lockFrame;
    uint32_t canSleep;
    float sleepTime;
    uint32_t island;
    uint32_t hasTarget;
    Transform target;
    // Bounds of the body's shapes other than half-spaces; hasBounds is 0 when it has none (no tree leaf).
    Vec3 lo, hi;
    uint32_t hasBounds;
    float kept;
    Mat3 linearProj;
    Mat3 angularProj;
    Quat qBase;
    Quat q0;
    Vec3 com0;
    float expectedTravel;
    // The body's shapes: shapeList[shapeFirst .. shapeFirst + shapeCount), global shape indices.
    uint32_t shapeFirst;
    uint32_t shapeCount;
    uint32_t world;
    // Set by every planar pair that placed the body in the current round of collisions; the round's
    // placement is stored, and this cleared, once all its pairs are done.
    uint32_t posePending;
    // The part of the body's pose in a plane that lasts between rounds (src/internal.h:141-148): the plane
    // normal it was placed for, that normal in the body's frame (the key) with the 2D axes around it, and the
    // plane's own 2D axes. Zero until the body is first placed.
    Vec3 poseNormal, poseKey, poseU, poseV, poseAxisU, poseAxisV;
};

struct alignas(16) DShape {
    uint32_t body;      // global body index
    uint32_t index;     // index within its world, the one contact keys use
    uint32_t kind;      // ShapeKind
    uint32_t geometry;  // tf_geometry
    Transform local;
    float friction;
    float restitution;
    float rollingResistance;
    uint32_t category;
    uint32_t mask;
    uint32_t sensor;
    uint32_t alive;
    float radius;
    float halfHeight;
    Vec3 halfExtents;
    int32_t poly;  // index into the polyhedron table, -1 for none
    int32_t mesh;  // index into the mesh table, -1 for none; a mesh keeps its root node's center in centroid
                   // and half size in halfExtents
    float extent;
    float minExtent;
    Vec3 centroid;
    Vec3 lo, hi;
};

// A convex polyhedron (src/internal.h:89-111) stored as ranges of the shared tables.
struct DPoly {
    int32_t vFirst, vCount;
    int32_t fFirst, fCount;  // faces, normals and offsets share this range
    int32_t eFirst, eCount;  // edges and arcs share this range
    int32_t iFirst, iCount;  // face vertex loops
    Vec3 centroid;
    Vec3 lo, hi;
};

// A triangle mesh (src/internal.h:47-87) stored as ranges of the shared mesh tables: vertex k is
// meshVerts[vFirst + k]; triangle t has corners meshIndices[3 * (tFirst + t) + 0..2] (vertex numbers of
// this mesh), normal meshNormals[tFirst + t] and edge flags meshEdges[tFirst + t]; node i is
// meshNodes[nFirst + i], its first naming a triangle of a leaf or the first child of an inner node.
struct DMesh {
    int32_t vFirst, vCount;
    int32_t tFirst, tCount;
    int32_t nFirst, nCount;
};

// A mesh tree node (src/internal.h:50-54): a leaf holds count triangles from first; an inner node has a
// count of zero and its children at first and first + 1.
struct MeshNode {
    Vec3 lo, hi;
    int32_t first, count;
};

// Face and edge fields index within their own polyhedron (vertex k is verts[vFirst + k]).
struct DFace {
    int32_t first, count;  // into the polyhedron's index range
};

struct DEdge {
    int32_t v0, v1, f0, f1;
    float length;
};

struct alignas(16) DPoint {
    Vec3 anchorA, anchorB;
    float adjustedSeparation;
    float normalImpulse;
    Vec3 tangentImpulse;
    float maxNormalImpulse;
    float relativeVelocity;
    float separation;
    Vec3 surfaceA, surfaceB;
    Vec3 localA;
    float pad;
};

constexpr uint32_t kCPlanar = 1u << 0, kCReusable = 1u << 1, kCRemoved = 1u << 2, kCTouched = 1u << 3,
                   kCLaned = 1u << 4;

struct alignas(16) DContact {
    uint64_t key;
    uint32_t part;
    uint32_t shapeA, shapeB;  // global
    uint32_t bodyA, bodyB;    // global
    int32_t count;
    uint32_t flags;
    Vec3 normal, tangent1, tangent2;
    float friction;
    float restitution;
    float rollingResistance;
    float rollingRadius;
    Vec3 rollingImpulse;
    Vec3 plane;
    Vec3 localNormal;
    Vec3 baseOffset;
    Quat baseTurn;
    int32_t featKind, featA, featB;
    // The mesh triangles this pair ruled out by distance when it was collided at the step's start, as a range
    // of the world's triangle bounds; empty for other pairs and for pairs kept from the last step.
    uint32_t boundsFirst, boundsCount;
    DPoint points[4];
};

// The planar axes of a contact point (src/internal.h:528-531).
struct DPlanarAxes {
    float normalA, normalB, normalMass;
    float tangentA, tangentB, tangentMass;
};

// Per-world placement of every array segment, fixed between re-layouts.
struct WorldInfo {
    uint32_t bodyFirst, bodyCount;
    uint32_t shapeFirst, shapeCount;
    uint32_t candFirst, candCap;      // candidate keys
    uint32_t contactFirst, contactCap;  // contacts, both buffers, and every per-contact list
    uint32_t planeFirst, planeCount;  // half-space shapes, global indices in planeList
    // A body locked to a plane (global index), UINT32_MAX for none. Every such body of a world is locked to
    // the same plane, so this one's normal is the normal of every planar pair in the world.
    uint32_t planeBody;
    // Mesh pairs: the parts after a pair's first (partFirst, partCap: contact records) and the triangles fast
    // pairs ruled out (boundsFirst, boundsCap: triangle bounds). Zero capacity in worlds without meshes.
    uint32_t partFirst, partCap;
    uint32_t boundsFirst, boundsCap;
    // Joints from jointFirst in the world's index order, and the body pairs that joints keep from colliding
    // (sorted keys min << 32 | max of world-local bodies) from the same offset.
    uint32_t jointFirst, jointCount, joinedCount;
};

enum JointType : uint32_t { kJointPoint = 0, kJointFixed, kJointHinge, kJointSlider, kJointDistance, kJointSwingTwist };
// A joint's end that is the world: a static body at the origin.
constexpr uint32_t kWorldEnd = UINT32_MAX;

// A joint (src/internal.h:508-548): its ends (global body indices, kWorldEnd for the world), its frames in
// each body, limits, motor, spring and friction, and the impulses it keeps between substeps and steps.
struct alignas(16) DJoint {
    uint32_t type, alive, broken, limited;
    uint32_t bodyA, bodyB;
    uint32_t collideConnected, brokeNow;  // brokeNow: broke in the current step
    Vec3 localA, localB, axisA, axisB, refA, refB;
    Quat restTurn, frameA, frameB;
    float length, lower, upper, motorSpeed, maxMotor, hertz, dampingRatio, maxFriction;
    float swingY, swingZ, breakForce, breakTorque;
    Vec3 linearImpulse, angularImpulse;
    float axialImpulse, motorImpulse, lowerImpulse, upperImpulse, frictionImpulse, swingImpulse;
    Vec3 frictionTurn;
    Vec3 rowForce[2], rowTorque[2];
    Vec3 force, torque;
};

// Per-world results and lists of the current step.
struct WorldCounts {
    uint32_t candCount;
    uint32_t contactCount;      // in the current contact buffer
    uint32_t nextContactCount;  // in the buffer the narrowphase just filled
    uint32_t activeCount;
    uint32_t impactCount;
    uint32_t fastCount;
    uint32_t fastSolidCount;
    uint32_t restCount;        // active contacts solved one at a time
    uint32_t restLevels;       // levels of the rest lists (contacts of a level share no moving body)
    uint32_t impactRestLevels;
    uint32_t impactRestCount;
    uint32_t colorCount;       // 1 + highest color used, active list
    uint32_t impactColorCount;
    uint32_t awakeBodies;
    uint32_t awakeIslands;
    uint32_t touching;          // contacts touching after the solve (StepProfile::touchingContacts)
    uint32_t touchEvents;       // this step's contact events and hits, in the world's event rooms
    uint32_t hitEvents;
    uint32_t wakePending;
    uint32_t flags;            // tf_device_flags
    uint32_t candNeeded;       // largest count seen, for growing capacities
    uint32_t contactNeeded;
    uint32_t sweepShapes;      // shapes the continuous pass swept, summed over every step since the layout
    uint32_t sweptPairs;       // this step's continuous pass: pairs swept, and bodies moved back
    uint32_t impacts;
    uint32_t activePoints;     // contact points of the active list
    uint32_t partCount;        // this step's extra mesh parts and triangle bounds used
    uint32_t boundsCount;
    // Worlds of more than kSweepBodies bodies: raw pair count of this step's sweep, and the range of the
    // bodies' intervals along x as order-preserving keys.
    uint32_t candRaw;
    uint32_t sweepMinKey, sweepMaxKey;
    uint32_t colorStart[kColors + 1];
    uint32_t impactColorStart[kColors + 1];
    // The flat solve: where this world's contacts of each color (and impact color) start in that color's
    // list over every world.
    uint32_t flatColorAt[kColors];
    uint32_t flatImpactAt[kColors];
    unsigned long long bodySteps;  // awake dynamic bodies summed over every step since the layout
};

// A contact event of the step (ContactEvent, include/twofold/world.h:269-276) as a kernel appends it: the
// pair's key (world-local shapes, lower index first) and whether the pair began touching. `late` is 0 for
// pairs the narrowphase dropped and 1 for the end-of-step report, which is how the reference orders the two
// for one pair (src/world.cpp:1694-1700); the host sorts a world's events by (key, late).
struct TouchEvent {
    uint64_t key;
    uint32_t begin;
    uint32_t late;
};

// A hit (HitEvent, include/twofold/world.h:278-288): the pair's key, the struck point on shape A in the
// world, the contact normal (A to B) and the approach speed.
struct HitRecord {
    uint64_t key;
    Vec3 point;
    Vec3 normal;
    float speed;
    uint32_t pad;
};

struct Tolerances {
    float linearSlop;
    float speculative;
};

struct Softness {
    float biasRate;
    float massScale;
    float impulseScale;
};

// WorldSettings plus everything derived from it that the kernels need (src/world.cpp:222-229, 1634-1642).
struct StepParams {
    Vec3 gravity;
    float lengthUnit;
    int substeps;
    float dt;
    float h;
    float invH;
    Softness contactSoft;
    Softness staticSoft;
    float maxPushout;
    float restitutionThreshold;
    float maxLinearSpeed;   // already scaled by lengthUnit
    float maxAngularSpeed;
    float sleepThreshold;   // scaled
    float timeToSleep;
    float reuseDistance;    // scaled
    float reuseCos;         // cos(0.5 * contactReuseAngle), computed on the host with the C library
    float featureTurnCos;   // cos(0.5 * 0.1), same
    float treeMargin;       // kTreeMargin * lengthUnit
    Tolerances tol;
    int continuous;
    float hitThreshold;     // scaled
    Softness jointSoft;     // src/world.cpp:1640
};

}
