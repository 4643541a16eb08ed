// Host side of the library: the C ABI (include/twofold_b200.h), host mirrors of every world, the device
// arena and the per-step kernel sequence.
//
// Host mirrors are authoritative until the first step; afterwards the device holds the dynamic state and
// the mirrors are refreshed from it on demand. A structural change (a body or shape added after stepping)
// pulls the device state back, rebuilds the layout and pushes everything again, contacts included, so
// warm starting survives it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/twofold_b200.h"
#include "tf_build.h"
#include "tf_kernels.cuh"
#include "tf_launch.h"
#include "tf_tape.h"

namespace tfb {

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& msg) {
    g_error = msg;
    return code;
}

#define TF_CUDA(call)                                                                                    \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) { return fail(TF_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); } \
    } while (0)

constexpr float kTreeMargin = 0.1f;
constexpr float kFeatureTurn = 0.1f;

struct HostBody {
    DBody d{};
    uint32_t generation = 0;
    std::vector<uint32_t> shapes;  // world-local shape indices
    bool massOverride = false;
    MassProps overrideMass;
};

struct HostJoint {
    DJoint d{};  // ends world-local, kWorldEnd for the world
    uint32_t generation = 0;
};

struct HostWorld {
    std::vector<HostJoint> joints;
    std::vector<uint32_t> freeJoints;  // destroyed joints' slots, reused last-in first-out
    std::vector<HostBody> bodies;
    std::vector<uint32_t> freeBodies;
    std::vector<HostShape> shapes;
    std::vector<uint32_t> freeShapes;
    std::vector<uint32_t> planes;  // half-space shapes in the order they were tracked
    std::vector<DContact> contacts;  // last pulled from the device (world-local indices)
    // Contact events that calls between steps queued (pairs ended by removing their shapes or joining their
    // bodies), reported first among the next step's events; and those the last step started with.
    std::vector<tf_contact_event> queued, stepQueued;
};

// One device allocation per array; sized at layout time.
template <class T>
struct DevArray {
    T* ptr = nullptr;
    size_t n = 0;
    DevArray() = default;
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    ~DevArray() { release(); }
    int alloc(size_t count) {
        if (count <= n && ptr) { return TF_OK; }
        if (ptr) { cudaFree(ptr); }
        ptr = nullptr;
        n = 0;
        const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
        cudaError_t e = cudaMalloc(&ptr, bytes);
        if (e != cudaSuccess) { return fail(TF_E_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e)); }
        n = std::max<size_t>(count, 1);
        return TF_OK;
    }
    void release() {
        if (ptr) { cudaFree(ptr); }
        ptr = nullptr;
        n = 0;
    }
};

Vec3 v3of(const float* p) { return { p[0], p[1], p[2] }; }
Quat q4of(const float* p) { return { p[0], p[1], p[2], p[3] }; }

}  // namespace

// Records a failure from another translation unit of the library for tf_last_error.
int noteError(int code, const std::string& msg) { return fail(code, msg); }

// The differentiable model (tf_adjoint.cu).
void* adjointCreate();
void adjointDestroy(void* run);
int adjointForward(void* run, const AdjointSetup& S, void* stream, int precision, const double* init, const double* mass,
                   const double* friction, double* finalState);
int adjointBackward(void* run, const AdjointSetup& S, void* stream, const double* gradFinal, double* gradInit,
                    double* gradMass, double* gradFriction);
void adjointTimes(void* run, float* ms);  // forward, backward, recompute summed, reverse summed
int adjointBranches(void* run, int nWorlds, uint64_t* out);

class Engine {
public:
    tf_settings settings{};
    int device = 0;
    std::vector<HostWorld> worlds;
    std::vector<HostMesh> meshes;  // shared by every world of the handle
    cudaStream_t stream = nullptr;
    int smCount = 148;
    int blockSize = 128;
    int64_t launches = 0;

    bool layoutDirty = true;   // device arrays do not match the mirrors' structure
    bool bodiesDirty = true;   // host body state newer than the device's
    bool onDevice = false;     // the device holds the newest dynamic state
    bool hostFresh = true;     // host mirrors hold the newest dynamic state
    std::vector<tf_profile> profiles;

    // Layout.
    std::vector<WorldInfo> info;
    std::vector<uint32_t> order;
    std::vector<uint32_t> bodyBase, shapeBase;
    size_t totalBodies = 0, totalShapes = 0, totalCand = 0, totalContacts = 0;
    float capFactor = 6.0f;
    BoxTopology boxTopology{};

    // Device arrays.
    DevArray<WorldInfo> dInfo;
    DevArray<WorldCounts> dCounts;
    DevArray<uint32_t> dOrder;
    DevArray<DBody> dBodies;
    DevArray<DShape> dShapes;
    DevArray<uint32_t> dShapeList, dPlaneList;
    DevArray<DPoly> dPolys;
    DevArray<Vec3> dVerts, dNormals, dArcs;
    DevArray<DMesh> dMeshes;
    DevArray<Vec3> dMeshVerts, dMeshNormals;
    DevArray<uint32_t> dMeshIndices;
    DevArray<uint8_t> dMeshEdges;
    DevArray<MeshNode> dMeshNodes;
    DevArray<int32_t> dIndices;
    DevArray<DFace> dFaces;
    DevArray<float> dOffsets;
    DevArray<DEdge> dEdges;
    DevArray<float> dGrow, dIslandTime;
    DevArray<uint32_t> dBodyColors, dUnionParent;
    DevArray<uint8_t> dStruck, dWakeMark;
    DevArray<uint64_t> dCand;
    DevArray<DContact> dStage;
    DevArray<uint8_t> dStageUsed;
    DevArray<uint32_t> dStagePart;
    DevArray<DContact> dStageExtra;
    DevArray<TriangleBound> dTriBounds;
    DevArray<DContact> dContacts[2];
    int cur = 0;
    DevArray<uint32_t> dActive, dImpact, dColored, dImpactColored, dRest, dImpactRest, dRestLevel, dImpactRestLevel;
    DevArray<uint8_t> dColor, dCflags;
    DevArray<Axis> dAxes;
    DevArray<float4> dRows, dFlatBodies, dFlatPose, dFlatMotion;
    DevArray<uint32_t> dSlotOf, dFlatColored, dFlatImpact;
    DevArray<uint64_t> dMergeKeyA, dMergeKeyB;
    DevArray<uint32_t> dMergePartA, dMergePartB, dMergeIdxA, dMergeIdxB;
    bool hasJoints = false;  // some world has joints: the substep and finish kernels with joint code run
    // A batch this small collides and refreshes every pair class in one launch each (k_collide_all,
    // k_refresh_all): its class lists hold few items, and a launch per class costs more than their work.
    bool smallBatch = false;
    static constexpr size_t kSmallBatchCandidates = 8192;
    DevArray<DJoint> dJoints;
    DevArray<uint64_t> dJoined;
    DevArray<TouchEvent> dTouchEvents;
    DevArray<HitRecord> dHitEvents;
    DevArray<uint32_t> dAbort;
    DevArray<uint32_t> dDebug;
    size_t nPolys = 0;

    // How each kernel is launched: threads per CTA, the world size above which a world gets the whole CTA
    // (smaller worlds get a warp each), and the dynamic shared memory a CTA stages worlds in. A caller's
    // choice (tf_world_set_launch) overrides the defaults derived from the batch's world sizes.
    struct LaunchShape {
        uint32_t threads = 256, bigBodies = 0, smemBytes = 0;
        bool chosen = false;
        bool flat = false;  // the substep only: the flat solve over every world (k_substep_flat)
    };
    static constexpr uint32_t kFlatShape = 0xffffffffu;  // bigBodies of a substep shape that selects the flat solve
    // broadphase, narrowphase, wake, prepare, refresh, substep, finish, collide. Refresh and collide run one
    // thread per work item over the whole grid; their shapes use only the thread count.
    static constexpr int kKernels = 8;
    LaunchShape shapes[kKernels];
    Split splits[kKernels];
    int grids[kKernels] = {};
    // k_collide per pair class, then k_refresh for the light list and per pair class.
    static constexpr int kFlatGrids = 2 * kPairClasses + 1;
    int flatGrids[kFlatGrids] = {};
    std::map<const void*, size_t> dynSmemLimit;
    bool kernelsConfigured = false;
    uint32_t maxWorldBodies = 0, maxWorldContacts = 0, medianWorldBodies = 0;
    std::vector<uint32_t> sortedSizes;  // world body counts, largest first
    uint64_t layoutGen = 0;              // bumped by every layout; snapshots hold only within one

    // A copy of the dynamic device state a step reads: bodies, shapes (their bounds), the current contact
    // list, the per-world counts and the per-body wake marks. Valid while the layout it was taken in stands.
    struct Snapshot {
        DevArray<DBody> bodies;
        DevArray<DShape> shapes;
        DevArray<DContact> contacts;
        DevArray<WorldCounts> counts;
        DevArray<uint8_t> struck, wakeMark;
        DevArray<DJoint> joints;
        int cur = 0;
        uint64_t layoutGen = 0;
        int64_t bodyStepsTotal = 0, bodyStepsBase = 0;
    };
    std::map<int, std::unique_ptr<Snapshot>> snapshots;
    bool laidOut = false;
    DevArray<uint32_t> dWork, dRowScratch, dRowLong, dRowCount;
    DevArray<Vec3> dSweptLo, dSweptHi;
    DevArray<float> dSweepLo, dSweepHi;
    DevArray<uint32_t> dSweepOrder, dSweepStart, dBigWorlds, dBigBodyStart;
    DevArray<SweepRec> dSweepRecs;
    std::vector<uint32_t> bigWorlds, bigBodyStart;  // worlds of more than kSweepBodies bodies
    DevArray<uint32_t> dSweepList, dHitParent;
    DevArray<unsigned long long> dHitKey, dGroupKey;
    DevArray<uint2> dCandItems, dContactItems;
    std::vector<uint32_t> minCandCap, minContactCap;

    // Host traffic staging and timing.
    DevArray<float> dHostIn, dHostOut;
    // Queued pose reads: two device staging buffers, the copy stream, and per buffer the events of its pack and
    // of its copy (a copy pending until tf_world_poses_wait).
    DevArray<float> dPoseStage[2];
    cudaStream_t copyStream = nullptr;
    cudaEvent_t posePacked[2] = {}, poseCopied[2] = {};
    bool poseCopyPending[2] = {};
    int poseSlot = 0;
    cudaEvent_t callStart = nullptr, callStop = nullptr;
    float lastElapsedMs = 0.0f;
    int64_t bodyStepsTotal = 0;
    bool profiling = false;
    static constexpr int kKernelKinds = 8;  // broadphase, narrowphase, wake, prepare, refresh, substep, finish, collide
    double kernelMs[kKernelKinds] = {};
    int64_t kernelLaunches[kKernelKinds] = {};
    std::vector<cudaEvent_t> eventPool;
    std::vector<int> eventKind;
    int eventsUsed = 0;

    // Graph replay: one recorded graph per contact buffer a sequence starts from. A graph recorded while
    // per-kernel profiling is on also records an event pair around each kernel group (graphTimers: kind, start,
    // stop), read after every replay, so the per-kernel times come from the replayed steps themselves.
    cudaGraphExec_t graphs[2] = { nullptr, nullptr };
    int graphSteps = 0;
    float graphDt = 0.0f;
    bool graphProfiled = false;
    struct KernelTimer {
        int kind;
        cudaEvent_t start, stop;
    };
    std::vector<KernelTimer> graphTimers[2];
    size_t graphTimersUsed[2] = { 0, 0 };
    std::vector<KernelTimer>* captureTimers = nullptr;
    size_t captureUsed = 0;

    void dropGraphs() {
        for (int b = 0; b < 2; ++b) {
            if (graphs[b]) { cudaGraphExecDestroy(graphs[b]); }
            graphs[b] = nullptr;
            for (KernelTimer& t : graphTimers[b]) {
                cudaEventDestroy(t.start);
                cudaEventDestroy(t.stop);
            }
            graphTimers[b].clear();
            graphTimersUsed[b] = 0;
        }
    }

    // The device arrays free themselves after this body, with the engine's device still current.
    ~Engine() {
        if (stream) { cudaSetDevice(device); }
        if (copyStream) {
            cudaStreamSynchronize(copyStream);
            cudaStreamDestroy(copyStream);
        }
        if (hostSummary) { cudaFreeHost(hostSummary); }
        for (cudaEvent_t e : { posePacked[0], posePacked[1], poseCopied[0], poseCopied[1] }) {
            if (e) { cudaEventDestroy(e); }
        }
        if (adjRun) { adjointDestroy(adjRun); }
        for (cudaEvent_t e : eventPool) { cudaEventDestroy(e); }
        if (callStart) { cudaEventDestroy(callStart); }
        if (callStop) { cudaEventDestroy(callStop); }
        dropGraphs();
        if (stream) { cudaStreamDestroy(stream); }
    }

    int init(const tf_settings* s, int nWorlds, int dev) {
        settings = *s;
        device = dev;
        worlds.resize((size_t)nWorlds);
        profiles.assign((size_t)nWorlds, tf_profile{});
        // Box face and edge numbering from a unit box, as the reference derives it (src/collide3d.cpp:456-476).
        const HostPoly p = makeBox({ 1.0f, 1.0f, 1.0f });
        for (int f = 0; f < (int)p.normals.size(); ++f) {
            const float n[3] = { p.normals[f].x, p.normals[f].y, p.normals[f].z };
            for (int k = 0; k < 3; ++k) {
                if (std::fabs(n[k]) > 0.5f) { boxTopology.face[k][n[k] > 0.0f] = f; }
            }
        }
        auto edgeBetween = [&](int f0, int f1) {
            for (size_t i = 0; i < p.edges.size(); ++i) {
                const DEdge& e = p.edges[i];
                if ((e.f0 == f0 && e.f1 == f1) || (e.f0 == f1 && e.f1 == f0)) { return (int)i; }
            }
            return -1;
        };
        for (int i = 0; i < 3; ++i) {
            for (int s1 = 0; s1 < 2; ++s1) {
                for (int s2 = 0; s2 < 2; ++s2) {
                    boxTopology.edge[i][s1][s2] = edgeBetween(boxTopology.face[(i + 1) % 3][s1], boxTopology.face[(i + 2) % 3][s2]);
                }
            }
        }
        return TF_OK;
    }

    // CUDA is first touched by the first step, so scenes can be built and inspected without a device.
    int ensureDevice() {
        if (stream) { return TF_OK; }
        TF_CUDA(cudaSetDevice(device));
        TF_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        TF_CUDA(cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, device));
        TF_CUDA(cudaEventCreate(&callStart));
        TF_CUDA(cudaEventCreate(&callStop));
        return TF_OK;
    }

    // Launches kernel `id` on the engine's stream; the arguments must have the kernel's parameter types exactly.
    template <class... Args>
    void launch(int id, unsigned grid, unsigned block, size_t smem, Args... args) {
        void* ptrs[] = { (void*)&args... };
        cudaLaunchKernel(kernelEntry(id), dim3(grid), dim3(block), ptrs, smem, stream);
    }

    // A cooperative launch (every CTA resident at once, which the flat solve's grid barrier needs); grid must
    // not exceed what fits on the device.
    template <class... Args>
    void launchCooperative(int id, unsigned grid, unsigned block, Args... args) {
        void* ptrs[] = { (void*)&args... };
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(block);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaLaunchKernelExC(&cfg, kernelEntry(id), ptrs);
    }

    // Brackets one kernel launch with events when per-kernel profiling is on: from the event pool for direct
    // launches, into the graph's own timers while a profiled graph is being captured.
    template <class Launch>
    void timed(int kind, bool record, Launch&& launch) {
        if (captureTimers) {
            // Events made before the capture began; recorded as external event nodes, so that every replay of
            // the graph records them.
            if (captureUsed < captureTimers->size()) {
                KernelTimer& t = (*captureTimers)[captureUsed++];
                t.kind = kind;
                cudaEventRecordWithFlags(t.start, stream, cudaEventRecordExternal);
                launch();
                cudaEventRecordWithFlags(t.stop, stream, cudaEventRecordExternal);
                return;
            }
            launch();
            return;
        }
        if (!record) {
            launch();
            return;
        }
        if (eventsUsed + 2 > (int)eventPool.size()) {
            for (int k = 0; k < 64; ++k) {
                cudaEvent_t e;
                cudaEventCreate(&e);
                eventPool.push_back(e);
                eventKind.push_back(0);
            }
        }
        cudaEventRecord(eventPool[eventsUsed], stream);
        launch();
        cudaEventRecord(eventPool[eventsUsed + 1], stream);
        eventKind[eventsUsed] = kind;
        eventsUsed += 2;
    }

    // Adds the bracketed kernel times of the steps just synchronized to the per-kernel totals.
    void collectKernelTimes() {
        for (int k = 0; k + 1 < eventsUsed; k += 2) {
            float ms = 0.0f;
            if (cudaEventElapsedTime(&ms, eventPool[k], eventPool[k + 1]) == cudaSuccess) {
                kernelMs[eventKind[k]] += ms;
                kernelLaunches[eventKind[k]] += 1;
            }
        }
        eventsUsed = 0;
    }

    // ---- host-side world building (src/world.cpp:1751-1857) ----

    void hostShapeBounds(HostShape& s, const Transform& xf) {
        DPoly poly{};
        PolyTables pt{};
        if (s.hasPoly) {
            poly.vFirst = 0;
            poly.vCount = (int)s.poly.vertices.size();
            pt.polys = &poly;
            pt.verts = s.poly.vertices.data();
        }
        DShape d = s.d;
        d.poly = 0;
        shapeBounds(d, pt, xf, s.d.lo, s.d.hi);
    }

    // Shape bounds and the body's union (Impl::bound, src/world.cpp:244-258).
    bool bound(HostWorld& W, HostBody& hb) {
        bool any = false;
        DBody& b = hb.d;
        for (uint32_t si : hb.shapes) {
            HostShape& s = W.shapes[si];
            hostShapeBounds(s, b.xf * s.d.local);
            if (s.d.kind == kHalfSpace) { continue; }
            b.lo = any ? minVec(b.lo, s.d.lo) : s.d.lo;
            b.hi = any ? maxVec(b.hi, s.d.hi) : s.d.hi;
            any = true;
        }
        b.hasBounds = any ? 1u : 0u;
        return any;
    }

    // src/world.cpp:439-479.
    void updateMass(HostWorld& W, HostBody& hb) {
        DBody& b = hb.d;
        MassProps mp;
        if (hb.massOverride) {
            mp = hb.overrideMass;
        } else {
            Vec3 weighted{ 0, 0, 0 };
            std::vector<MassProps> parts;
            for (uint32_t si : hb.shapes) {
                const HostShape& s = W.shapes[si];
                if (s.d.sensor) { continue; }
                const MassProps sm = shapeMass(s);
                if (sm.mass <= 0.0f) { continue; }
                mp.mass += sm.mass;
                weighted += sm.center * sm.mass;
                parts.push_back(sm);
            }
            if (mp.mass > 0.0f) {
                mp.center = weighted / mp.mass;
                for (const MassProps& sm : parts) {
                    const Vec3 d = sm.center - mp.center;
                    const float dd = dot(d, d);
                    mp.inertia = mp.inertia + sm.inertia + (mdiag({ dd, dd, dd }) - outer(d, d)) * sm.mass;
                }
            }
        }
        b.localCenter = mp.center;
        b.mass = mp.mass;
        b.inertia = mp.inertia;
        if (b.type == kDynamic && b.mass <= 0.0f) {
            b.mass = 1.0f;
            b.inertia = mid();
        }
        b.invMass = (b.type == kDynamic && b.mass > 0.0f) ? 1.0f / b.mass : 0.0f;
        b.com = apply(b.xf, b.localCenter);
        b.extent = 0.0f;
        for (uint32_t si : hb.shapes) {
            const HostShape& s = W.shapes[si];
            if (s.d.kind == kHalfSpace || s.d.sensor) { continue; }
            b.extent = maxf(b.extent, s.d.extent + length(s.d.local.p - b.localCenter));
        }
        updateInverseMass(b);
    }

    int createBody(int w, const tf_body_desc* d, tf_id* out) {
        if (w < 0 || w >= (int)worlds.size() || !d) { return fail(TF_E_INVALID, "createBody: bad world or descriptor"); }
        if (d->type < 0 || d->type > 2) { return fail(TF_E_INVALID, "createBody: bad motion type"); }
        int rc = pull();
        if (rc != TF_OK) { return rc; }
        HostWorld& W = worlds[(size_t)w];
        if ((d->locks & kLockPlanar) == kLockPlanar) {
            // Every planar pair of a world is then solved in one plane, whose placements the kernels keep
            // per body.
            const Quat frame = normalize(q4of(d->lock_frame));
            for (const HostBody& o : W.bodies) {
                if (!o.d.alive || !isPlanar(o.d)) { continue; }
                const Quat f = o.d.lockFrame;
                if (!(f.x == frame.x && f.y == frame.y && f.z == frame.z && f.w == frame.w)) {
                    return fail(TF_E_UNSUPPORTED,
                                "createBody: bodies locked to different planes in one world are not run by this build");
                }
                break;
            }
        }
        uint32_t i;
        if (!W.freeBodies.empty()) {
            i = W.freeBodies.back();
            W.freeBodies.pop_back();
        } else {
            i = (uint32_t)W.bodies.size();
            W.bodies.emplace_back();
        }
        HostBody& hb = W.bodies[i];
        const uint32_t gen = hb.generation;
        hb = HostBody{};
        hb.generation = gen;
        DBody& b = hb.d;
        b.alive = 1;
        b.type = (uint32_t)d->type;
        b.xf = { v3of(d->position), normalize(q4of(d->rotation)) };
        b.v = d->type == TF_STATIC ? zero3() : v3of(d->linear_velocity);
        b.w = d->type == TF_STATIC ? zero3() : v3of(d->angular_velocity);
        b.linearDamping = d->linear_damping;
        b.angularDamping = d->angular_damping;
        b.gravityScale = d->gravity_scale;
        b.locks = d->locks & 0x3fu;
        b.lockFrame = normalize(q4of(d->lock_frame));
        b.awake = d->awake ? 1u : 0u;
        b.canSleep = d->can_sleep ? 1u : 0u;
        b.kept = 1.0f;
        b.island = UINT32_MAX;
        b.dq = qid();
        b.qBase = qid();
        b.q0 = qid();
        b.linearProj = mid();
        b.angularProj = mid();
        updateMass(W, hb);
        b.v = b.linearProj * b.v;
        b.w = b.angularProj * b.w;
        layoutDirty = true;
        if (out) { *out = { i, hb.generation }; }
        return TF_OK;
    }

    HostBody* body(int w, tf_id id) {
        if (w < 0 || w >= (int)worlds.size()) { return nullptr; }
        HostWorld& W = worlds[(size_t)w];
        if (id.index >= W.bodies.size()) { return nullptr; }
        HostBody& b = W.bodies[id.index];
        return (b.d.alive && b.generation == id.generation) ? &b : nullptr;
    }

    int addShape(int w, tf_id bid, const tf_shape_desc* d, tf_id* out) {
        if (out) { *out = { UINT32_MAX, 0 }; }
        if (!d) { return fail(TF_E_INVALID, "addShape: null descriptor"); }
        int rc = pull();
        if (rc != TF_OK) { return rc; }
        HostBody* hb = body(w, bid);
        if (!hb) { return TF_OK; }  // invalid handle: nothing happens, as in the reference
        HostWorld& W = worlds[(size_t)w];
        HostShape s;
        s.d.alive = 1;
        s.d.body = bid.index;
        s.d.local = { v3of(d->position), normalize(q4of(d->rotation)) };
        s.density = d->density;
        s.d.friction = d->friction;
        s.d.restitution = d->restitution;
        s.d.rollingResistance = d->rolling_resistance;
        s.d.category = d->category;
        s.d.mask = d->mask;
        s.d.sensor = d->sensor ? 1u : 0u;
        s.d.poly = -1;
        s.d.mesh = -1;
        if ((d->geometry == TF_PRISM || d->geometry == TF_HULL) && d->point_count > 0 && !d->points) {
            return fail(TF_E_INVALID, "addShape: prism or hull without points");
        }
        const HostMesh* mesh = nullptr;
        if (d->geometry == TF_MESH) {
            if (d->mesh < 0 || (size_t)d->mesh >= meshes.size()) { return fail(TF_E_INVALID, "addShape: unknown mesh"); }
            if (hb->d.type == kDynamic) {
                return fail(TF_E_UNSUPPORTED, "addShape: meshes belong to static and kinematic bodies");
            }
            mesh = &meshes[(size_t)d->mesh];
        }
        if (!buildShapeGeometry(s, d->geometry, d->radius, v3of(d->half_extents), d->points, d->point_count, d->z_min,
                                d->z_max, d->max_vertices, mesh, d->mesh, d->half_height)) {
            return fail(TF_E_INVALID, "addShape: unknown geometry");
        }
        if (s.d.sensor) { return fail(TF_E_UNSUPPORTED, "addShape: sensors are not run by this build"); }
        if (s.d.kind == kHalfSpace && hb->d.type != kStatic) {
            return fail(TF_E_UNSUPPORTED, "addShape: half-spaces belong to static bodies");
        }
        uint32_t i;
        if (!W.freeShapes.empty()) {
            i = W.freeShapes.back();
            W.freeShapes.pop_back();
        } else {
            i = (uint32_t)W.shapes.size();
            W.shapes.emplace_back();
        }
        const uint32_t gen = W.shapes[i].generation;
        s.generation = gen;
        s.d.index = i;
        W.shapes[i] = s;
        hb->shapes.push_back(i);
        if (s.d.kind == kHalfSpace) { W.planes.push_back(i); }
        bound(W, *hb);
        updateMass(W, *hb);
        layoutDirty = true;
        if (out) { *out = { i, gen }; }
        return TF_OK;
    }


    // The reference's Tolerances for the current settings (src/world.cpp:222-229).
    Tolerances tolerances() const {
        Tolerances t;
        t.linearSlop = 0.005f * settings.length_unit;
        t.speculative = 4.0f * t.linearSlop;
        return t;
    }

    // twofold::angularVelocity (include/twofold/math.h:217-224): the spin that turns a into b over dt.
    static Vec3 angularVelocityBetween(const Quat& a, const Quat& b, float dt) {
        Quat d = normalize(b * conjugate(a));
        if (d.w < 0) { d = Quat{ -d.x, -d.y, -d.z, -d.w }; }
        const Vec3 v{ d.x, d.y, d.z };
        const float s = length(v);
        if (s < 1e-7f || dt <= 0) { return zero3(); }
        const float angle = 2.0f * std::atan2(s, d.w);
        return v * (angle / (s * dt));
    }

    // ---- World calls between steps (src/world.cpp:1743-2210), on the host mirrors ----
    //
    // Every such call brings the device's state into the mirrors, changes them as the reference's call changes
    // its world, and marks what the next step must send back. The reference's helpers they use are restated
    // below on the mirrors: the links between bodies (contacts with points, unbroken joints), the wake flood,
    // and the marking of contacts for the next step to drop.

    // Impl::Link (src/world.cpp:650-678): a body's contact pairs (once per key) and joints, in that order.
    struct Link {
        uint64_t key;
        uint32_t other;
        uint32_t joint;  // UINT32_MAX for a contact pair
    };

    static std::vector<std::vector<Link>> linksOf(const HostWorld& W) {
        std::vector<std::vector<Link>> links(W.bodies.size());
        for (size_t ci = 0; ci < W.contacts.size(); ++ci) {
            const DContact& c = W.contacts[ci];
            if (ci > 0 && W.contacts[ci - 1].key == c.key) { continue; }
            links[c.bodyA].push_back({ c.key, c.bodyB, UINT32_MAX });
            links[c.bodyB].push_back({ c.key, c.bodyA, UINT32_MAX });
        }
        for (uint32_t ji = 0; ji < W.joints.size(); ++ji) {
            const DJoint& j = W.joints[ji].d;
            if (!j.alive || j.bodyA == kWorldEnd) { continue; }
            links[j.bodyA].push_back({ 0, j.bodyB, ji });
            links[j.bodyB].push_back({ 0, j.bodyA, ji });
        }
        return links;
    }

    // The first contact of a pair in the mirrors' (key, part) order, or the end.
    static size_t firstOf(const HostWorld& W, uint64_t key) {
        return (size_t)(std::lower_bound(W.contacts.begin(), W.contacts.end(), key,
                                         [](const DContact& x, uint64_t k) { return x.key < k; }) -
                        W.contacts.begin());
    }

    // Impl::linked (src/world.cpp:681-689): a joint while unbroken, a contact pair while one of its contacts has
    // points.
    static bool linked(const HostWorld& W, const Link& l) {
        if (l.joint != UINT32_MAX) { return W.joints[l.joint].d.alive && !W.joints[l.joint].d.broken; }
        for (size_t ci = firstOf(W, l.key); ci < W.contacts.size() && W.contacts[ci].key == l.key; ++ci) {
            if (W.contacts[ci].count > 0) { return true; }
        }
        return false;
    }

    static void pushLinked(const HostWorld& W, const std::vector<std::vector<Link>>& links, uint32_t i,
                           std::vector<uint32_t>& stack) {
        for (const Link& l : links[i]) {
            const DBody& o = W.bodies[l.other].d;
            if (o.type == kDynamic && !o.awake && linked(W, l)) { stack.push_back(l.other); }
        }
    }

    // Impl::meshTouches (src/world.cpp:552-563): whether a triangle of the mesh shape lies in the box, the box
    // taken into the mesh's frame as boundsInMesh does (src/mesh.cpp).
    bool meshTouches(const HostShape& s, const Transform& xm, const Vec3& lo, const Vec3& hi) const {
        if (s.d.mesh < 0 || (size_t)s.d.mesh >= meshes.size()) { return false; }
        const HostMesh& m = meshes[(size_t)s.d.mesh];
        if (m.nodes.empty()) { return false; }
        const Vec3 c = applyInverse(xm, (lo + hi) * 0.5f);
        const Vec3 e = (hi - lo) * 0.5f;
        const Mat3 r = toMat3(conjugate(xm.q));
        Vec3 reach;
        for (int i = 0; i < 3; ++i) {
            setComp(reach, i, std::fabs(r.r[i].x) * e.x + std::fabs(r.r[i].y) * e.y + std::fabs(r.r[i].z) * e.z);
        }
        const Vec3 mlo = c - reach, mhi = c + reach;
        for (size_t t = 0; t < m.normals.size(); ++t) {
            Vec3 k[3];
            m.corners((int)t, k);
            if (boxesOverlap(minVec(minVec(k[0], k[1]), k[2]), maxVec(maxVec(k[0], k[1]), k[2]), mlo, mhi)) { return true; }
        }
        return false;
    }

    // Impl::pushOverlapping (src/world.cpp:620-647): sleeping dynamic bodies whose shapes an anchor's shapes
    // reach, per anchor shape in order, each shape's finds sorted and unique. The reference finds candidates in
    // its tree, whose fat leaves hold every shape the exact test below passes; here every shape is tested.
    void pushOverlapping(const HostWorld& W, uint32_t anchor, std::vector<uint32_t>& stack) const {
        const float g = tolerances().speculative;
        const Vec3 grow{ g, g, g };
        const HostBody& A = W.bodies[anchor];
        std::vector<uint32_t> found;
        for (uint32_t ai : A.shapes) {
            const HostShape& sa = W.shapes[ai];
            if (sa.d.sensor) { continue; }
            const Transform xa = A.d.xf * sa.d.local;
            const Vec3 n = rotate(xa.q, Vec3{ 0, 0, 1 });
            found.clear();
            for (const HostShape& sb : W.shapes) {
                if (!sb.d.alive || sb.d.sensor) { continue; }
                const DBody& b = W.bodies[sb.d.body].d;
                if (!b.alive || b.type != kDynamic || b.awake) { continue; }
                if (!(sa.d.category & sb.d.mask) || !(sb.d.category & sa.d.mask)) { continue; }
                const Vec3 blo = sb.d.lo - grow, bhi = sb.d.hi + grow;
                if (!boxesOverlap(sa.d.lo, sa.d.hi, blo, bhi)) { continue; }
                if (sa.d.kind == kHalfSpace) {
                    const Vec3 c = (blo + bhi) * 0.5f, e = (bhi - blo) * 0.5f;
                    const float reach = e.x * std::fabs(n.x) + e.y * std::fabs(n.y) + e.z * std::fabs(n.z);
                    if (dot(c - xa.p, n) > reach) { continue; }
                }
                if (sa.d.kind == kMesh && !meshTouches(sa, xa, blo, bhi)) { continue; }
                found.push_back(sb.d.body);
            }
            std::sort(found.begin(), found.end());
            found.erase(std::unique(found.begin(), found.end()), found.end());
            stack.insert(stack.end(), found.begin(), found.end());
        }
    }

    // Impl::wakeBodies (src/world.cpp:705-735): a sleeping dynamic start wakes its island through contacts with
    // points and unbroken joints; a static or kinematic start wakes the dynamic bodies touching or overlapping
    // it, without spreading past them.
    void wakeBodies(HostWorld& W, const std::vector<uint32_t>& start) {
        std::vector<uint32_t> stack;
        bool anchors = false;
        for (uint32_t i : start) {
            const DBody& b = W.bodies[i].d;
            if (!b.alive) { continue; }
            if (b.type != kDynamic) {
                anchors = true;
            } else if (!b.awake) {
                stack.push_back(i);
            }
        }
        if (stack.empty() && !anchors) { return; }
        const std::vector<std::vector<Link>> links = linksOf(W);
        for (uint32_t i : start) {
            if (!W.bodies[i].d.alive || W.bodies[i].d.type == kDynamic) { continue; }
            pushLinked(W, links, i, stack);
            pushOverlapping(W, i, stack);
        }
        while (!stack.empty()) {
            const uint32_t i = stack.back();
            stack.pop_back();
            DBody& b = W.bodies[i].d;
            if (b.awake) { continue; }
            b.awake = 1;
            b.sleepTime = 0.0f;
            updateInverseMass(b);
            pushLinked(W, links, i, stack);
        }
    }

    tf_contact_event endEvent(const HostWorld& W, const DContact& c) const {
        tf_contact_event e{};
        e.shape_a = c.shapeA;
        e.shape_b = c.shapeB;
        e.body_a = c.bodyA;
        e.body_b = c.bodyB;
        e.begin = 0;
        return e;
    }

    // Impl::dropContacts (src/world.cpp:565-593): marks the body's contact pairs that pick accepts as removed
    // (no points, not reusable) for the next step to drop, and returns the dynamic bodies on their other side.
    // When their shapes are going away (`ending`), pairs that touched end now, their event queued.
    template <class Pick>
    std::vector<uint32_t> dropContacts(HostWorld& W, uint32_t body, bool ending, Pick&& pick) {
        std::vector<uint32_t> touched;
        const std::vector<std::vector<Link>> links = linksOf(W);
        for (const Link& l : links[body]) {
            if (l.joint != UINT32_MAX || !pick(l)) { continue; }
            bool hit = false;
            size_t ci = firstOf(W, l.key);
            if (ending && ci < W.contacts.size() && W.contacts[ci].key == l.key && (W.contacts[ci].flags & kCTouched)) {
                W.queued.push_back(endEvent(W, W.contacts[ci]));
            }
            for (; ci < W.contacts.size() && W.contacts[ci].key == l.key; ++ci) {
                DContact& c = W.contacts[ci];
                if (ending) { c.flags &= ~kCTouched; }
                if (c.flags & kCRemoved) { continue; }
                c.flags |= kCRemoved;
                c.flags &= ~kCReusable;
                c.count = 0;
                hit = true;
            }
            if (hit && W.bodies[l.other].d.type == kDynamic) { touched.push_back(l.other); }
        }
        return touched;
    }

    // Impl::removeContacts (src/world.cpp:595-600): a body's pairs, or one shape's.
    void removeContacts(HostWorld& W, uint32_t body, int shape, bool ending) {
        wakeBodies(W, dropContacts(W, body, ending, [&](const Link& l) {
            return shape < 0 || (uint32_t)(l.key >> 32) == (uint32_t)shape || (uint32_t)l.key == (uint32_t)shape;
        }));
    }

    HostShape* shapeRef(int w, tf_id id) {
        if (w < 0 || w >= (int)worlds.size()) { return nullptr; }
        HostWorld& W = worlds[(size_t)w];
        if (id.index >= W.shapes.size()) { return nullptr; }
        HostShape& s = W.shapes[id.index];
        return (s.d.alive && s.generation == id.generation) ? &s : nullptr;
    }

    // The other calls' common start: the device's state in the mirrors, and the body named (nullptr for an
    // invalid handle, which the reference's setters take as a no-op).
    int hostBody(int w, tf_id id, HostBody** out) {
        *out = nullptr;
        const int rc = pull();
        if (rc != TF_OK) { return rc; }
        *out = body(w, id);
        return TF_OK;
    }

    // World::destroyBody (src/world.cpp:1784-1808).
    int destroyBody(int w, tf_id id) {
        HostBody* hb = nullptr;
        int rc = hostBody(w, id, &hb);
        if (rc != TF_OK || !hb) { return rc; }
        HostWorld& W = worlds[(size_t)w];
        const uint32_t bi = id.index;
        removeContacts(W, bi, -1, true);
        for (uint32_t ji = 0; ji < W.joints.size(); ++ji) {
            const DJoint& j = W.joints[ji].d;
            if (j.alive && (j.bodyA == bi || j.bodyB == bi)) { killJoint(W, ji); }
        }
        for (uint32_t si : W.bodies[bi].shapes) {
            HostShape& s = W.shapes[si];
            untrack(W, si);
            s.d.alive = 0;
            ++s.generation;
            W.freeShapes.push_back(si);
        }
        HostBody& b = W.bodies[bi];
        b.shapes.clear();
        b.d.alive = 0;
        b.d.hasBounds = 0;
        ++b.generation;
        W.freeBodies.push_back(bi);
        layoutDirty = true;
        return TF_OK;
    }

    static void untrack(HostWorld& W, uint32_t si) {
        if (W.shapes[si].d.kind == kHalfSpace) { W.planes.erase(std::remove(W.planes.begin(), W.planes.end(), si), W.planes.end()); }
    }

    // Impl::destroyJoint (src/world.cpp:399-406): the joint's dynamic ends woken, its slot freed.
    void killJoint(HostWorld& W, uint32_t ji) {
        HostJoint& hj = W.joints[ji];
        wakeJoint(W, hj.d);
        hj.d.alive = 0;
        hj.d.brokeNow = 0;
        ++hj.generation;
        W.freeJoints.push_back(ji);
        layoutDirty = true;
    }

    // Impl::wakeJoint (src/world.cpp:391-397).
    void wakeJoint(HostWorld& W, const DJoint& j) {
        std::vector<uint32_t> start;
        for (uint32_t i : { j.bodyA, j.bodyB }) {
            if (i != kWorldEnd && W.bodies[i].d.type == kDynamic) { start.push_back(i); }
        }
        wakeBodies(W, start);
    }

    // World::removeShape (src/world.cpp:1859-1876).
    int removeShape(int w, tf_id id) {
        const int rc = pull();
        if (rc != TF_OK) { return rc; }
        HostShape* s = shapeRef(w, id);
        if (!s) { return TF_OK; }
        HostWorld& W = worlds[(size_t)w];
        const uint32_t bi = s->d.body;
        removeContacts(W, bi, (int)id.index, true);
        HostBody& b = W.bodies[bi];
        b.shapes.erase(std::remove(b.shapes.begin(), b.shapes.end(), id.index), b.shapes.end());
        untrack(W, id.index);
        s->d.alive = 0;
        ++s->generation;
        W.freeShapes.push_back(id.index);
        bound(W, b);
        updateMass(W, b);
        wakeBodies(W, { bi });
        layoutDirty = true;
        return TF_OK;
    }

    // World::setFriction, setRestitution, setRollingResistance (src/world.cpp:1958-1968) and setFilter
    // (:1970-1978), which drops the shape's contact pairs without ending them.
    int setShapeValue(int w, tf_id id, int what, float value, uint32_t category, uint32_t mask) {
        const int rc = pull();
        if (rc != TF_OK) { return rc; }
        HostShape* s = shapeRef(w, id);
        if (!s) { return TF_OK; }
        switch (what) {
            case 0: s->d.friction = value; break;
            case 1: s->d.restitution = value; break;
            case 2: s->d.rollingResistance = value; break;
            case 3:
                s->d.category = category;
                s->d.mask = mask;
                removeContacts(worlds[(size_t)w], s->d.body, (int)id.index, false);
                break;
            default: return fail(TF_E_INVALID, "shape setter: unknown value");
        }
        layoutDirty = true;
        return TF_OK;
    }

    // World::setTransform (src/world.cpp:1993-2003): the pose, its bounds, and the bodies it wakes.
    int setTransform(int w, tf_id id, const Vec3& p, const Quat& q) {
        HostBody* hb = nullptr;
        int rc = hostBody(w, id, &hb);
        if (rc != TF_OK || !hb) { return rc; }
        HostWorld& W = worlds[(size_t)w];
        DBody& b = hb->d;
        b.xf = { p, normalize(q) };
        b.com = apply(b.xf, b.localCenter);
        b.hasTarget = 0;
        bound(W, *hb);
        wakeBodies(W, { id.index });
        layoutDirty = true;
        return TF_OK;
    }

    // World::setKinematicTarget (src/world.cpp:2031-2040).
    int setKinematicTarget(int w, tf_id id, const Vec3& p, const Quat& rotation, float dt) {
        HostBody* hb = nullptr;
        int rc = hostBody(w, id, &hb);
        if (rc != TF_OK || !hb || hb->d.type != kKinematic || !(dt > 0.0f)) { return rc; }
        DBody& b = hb->d;
        const Quat q = normalize(rotation);
        const Vec3 com = p + rotate(q, b.localCenter);
        b.v = (com - b.com) / dt;
        b.w = angularVelocityBetween(b.xf.q, q, dt);
        b.target = { p, q };
        b.hasTarget = 1;
        bodiesDirty = true;
        return TF_OK;
    }

    // World::setMotionType (src/world.cpp:2047-2062).
    int setMotionType(int w, tf_id id, int type) {
        if (type < 0 || type > 2) { return fail(TF_E_INVALID, "setMotionType: bad motion type"); }
        HostBody* hb = nullptr;
        int rc = hostBody(w, id, &hb);
        if (rc != TF_OK || !hb || (int)hb->d.type == type) { return rc; }
        HostWorld& W = worlds[(size_t)w];
        if (type == kDynamic) {
            for (uint32_t si : hb->shapes) {
                if (W.shapes[si].d.kind == kMesh || W.shapes[si].d.kind == kHalfSpace) {
                    return fail(TF_E_UNSUPPORTED, "setMotionType: meshes and half-spaces belong to bodies that are not dynamic");
                }
            }
        }
        DBody& b = hb->d;
        b.type = (uint32_t)type;
        b.hasTarget = 0;
        if (type == kStatic) {
            b.v = zero3();
            b.w = zero3();
        }
        if (type == kDynamic) { b.awake = 1; }
        if (type != kDynamic) {
            // Impl::removeAnchoredContacts (src/world.cpp:602-605).
            dropContacts(W, id.index, false, [&](const Link& l) { return W.bodies[l.other].d.type != kDynamic; });
        }
        updateMass(W, *hb);
        wakeBodies(W, { id.index });
        layoutDirty = true;
        return TF_OK;
    }

    // World::addForce, addForceAtPoint, addTorque, addImpulse, addImpulseAtPoint (src/world.cpp:2064-2112):
    // dynamic bodies, woken first when asked; a body still asleep takes nothing.
    int push(int w, tf_id id, int what, const Vec3& v, const Vec3* point, bool wake) {
        HostBody* hb = nullptr;
        int rc = hostBody(w, id, &hb);
        if (rc != TF_OK || !hb || hb->d.type != kDynamic) { return rc; }
        if (wake) { wakeBodies(worlds[(size_t)w], { id.index }); }
        DBody& b = hb->d;
        if (!b.awake) {
            bodiesDirty = true;
            return TF_OK;
        }
        switch (what) {
            case 0:
                b.force += v;
                if (point) { b.torque += cross(*point - b.com, v); }
                break;
            case 1: b.torque += v; break;
            case 2:
                b.v += b.invMassWorld * v;
                if (point) { b.w += b.invInertiaWorld * cross(*point - b.com, v); }
                break;
            default: return fail(TF_E_INVALID, "push: unknown kind");
        }
        bodiesDirty = true;
        return TF_OK;
    }

    // World::setLinearVelocity, setAngularVelocity (src/world.cpp:2015-2029): projected on the free axes, and
    // the body woken.
    int setVelocity(int w, tf_id id, const float* v, const float* av) {
        HostBody* hb = nullptr;
        int rc = hostBody(w, id, &hb);
        if (rc != TF_OK || !hb || hb->d.type == kStatic) { return rc; }
        if (v) {
            hb->d.v = hb->d.linearProj * v3of(v);
            wakeBodies(worlds[(size_t)w], { id.index });
        }
        if (av) {
            hb->d.w = hb->d.angularProj * v3of(av);
            wakeBodies(worlds[(size_t)w], { id.index });
        }
        bodiesDirty = true;
        return TF_OK;
    }

    // World::setDamping, setGravityScale, setCanSleep, wake, sleep (src/world.cpp:2163-2207).
    int setBodyValue(int w, tf_id id, int what, float a, float b) {
        HostBody* hb = nullptr;
        int rc = hostBody(w, id, &hb);
        if (rc != TF_OK || !hb) { return rc; }
        HostWorld& W = worlds[(size_t)w];
        DBody& d = hb->d;
        switch (what) {
            case 0:
                d.linearDamping = a;
                d.angularDamping = b;
                break;
            case 1: d.gravityScale = a; break;
            case 2:
                d.canSleep = a != 0.0f ? 1u : 0u;
                if (!d.canSleep) { wakeBodies(W, { id.index }); }
                break;
            case 3: wakeBodies(W, { id.index }); break;
            case 4:
                if (d.type != kDynamic) { return TF_OK; }
                d.awake = 0;
                d.v = zero3();
                d.w = zero3();
                d.sleepTime = 0.0f;
                updateInverseMass(d);
                break;
            default: return fail(TF_E_INVALID, "body setter: unknown value");
        }
        bodiesDirty = true;
        return TF_OK;
    }

    // ---- layout and transfer ----

    // World::createJoint (src/world.cpp:2221-2333): the joint's frames in each body at their current poses.
    int createJoint(int w, const tf_joint_desc* d, tf_id* out) {
        if (w < 0 || w >= (int)worlds.size() || !d) { return fail(TF_E_INVALID, "createJoint: bad world or desc"); }
        if (d->type < TF_JOINT_POINT || d->type > TF_JOINT_SWING_TWIST) { return fail(TF_E_INVALID, "createJoint: bad type"); }
        int rc = pull();
        if (rc != TF_OK) { return rc; }
        HostWorld& W = worlds[(size_t)w];
        auto valid = [&](tf_id id) {
            return id.index < W.bodies.size() && W.bodies[id.index].d.alive && W.bodies[id.index].generation == id.generation;
        };
        if (!valid(d->body_b)) { return fail(TF_E_INVALID, "createJoint: invalid body B"); }
        uint32_t ai = kWorldEnd;
        if (d->body_a.index != UINT32_MAX) {
            if (!valid(d->body_a) || d->body_a.index == d->body_b.index) { return fail(TF_E_INVALID, "createJoint: invalid body A"); }
            ai = d->body_a.index;
        }
        const uint32_t bi = d->body_b.index;
        HostJoint hj;
        DJoint& j = hj.d;
        j.alive = 1;
        j.type = (uint32_t)d->type;
        j.bodyA = ai;
        j.bodyB = bi;
        j.collideConnected = d->collide_connected ? 1u : 0u;
        j.breakForce = d->break_force;
        j.breakTorque = d->break_torque;
        const JBody worldBody = worldEnd();
        const Transform xa = ai == kWorldEnd ? worldBody.xf : W.bodies[ai].d.xf;
        const Transform xb = W.bodies[bi].d.xf;
        const Vec3 anchor = v3of(d->anchor);
        Vec3 anchorA = anchor, anchorB = anchor, axis{ 1, 0, 0 }, normal = zero3();
        // The cone's half-angle sine, correctly rounded like every transcendental the device evaluates
        // (src/world.cpp:21-24).
        auto coneSine = [](float swing) {
            if (swing >= kJointPi) { return 1.0f; }
            return (float)std::sin((double)(0.5f * maxf(swing, 1e-3f)));
        };
        switch (d->type) {
            case TF_JOINT_HINGE:
            case TF_JOINT_SLIDER:
                axis = normalize(v3of(d->axis));
                j.limited = d->limited ? 1u : 0u;
                j.lower = d->lower;
                j.upper = d->upper;
                j.motorSpeed = d->motor_speed;
                j.maxMotor = d->max_motor;
                j.maxFriction = d->friction;
                break;
            case TF_JOINT_DISTANCE:
                anchorB = v3of(d->anchor_b);
                j.length = d->length < 0.0f ? length(anchorB - anchorA) : d->length;
                j.hertz = d->hertz;
                j.dampingRatio = d->damping_ratio;
                j.limited = d->limited ? 1u : 0u;
                j.lower = d->lower;
                j.upper = d->upper;
                break;
            case TF_JOINT_SWING_TWIST:
                axis = normalize(v3of(d->axis));
                normal = v3of(d->normal);
                j.limited = d->upper - d->lower < 2.0f * kJointPi ? 1u : 0u;
                j.lower = d->lower;
                j.upper = d->upper;
                j.swingY = coneSine(d->swing_y);
                j.swingZ = coneSine(d->swing_z);
                j.maxFriction = d->friction;
                break;
            default:
                break;
        }
        if (d->type != TF_JOINT_SWING_TWIST) {
            j.swingY = 1.0f;
            j.swingZ = 1.0f;
        }
        const Vec3 ref = perpendicular(axis);
        j.localA = applyInverse(xa, anchorA);
        j.localB = applyInverse(xb, anchorB);
        j.axisA = unrotate(xa.q, axis);
        j.axisB = unrotate(xb.q, axis);
        j.refA = unrotate(xa.q, ref);
        j.refB = unrotate(xb.q, ref);
        j.restTurn = conjugate(xa.q) * xb.q;
        j.frameA = qid();
        j.frameB = qid();
        if (d->type == TF_JOINT_SWING_TWIST) {
            Vec3 y = normal - axis * dot(normal, axis);
            y = lengthSquared(y) > 1e-12f ? normalize(y) : ref;
            const Vec3 z = cross(axis, y);
            Mat3 m;
            m.r[0] = { axis.x, y.x, z.x };
            m.r[1] = { axis.y, y.y, z.y };
            m.r[2] = { axis.z, y.z, z.z };
            const Quat frame = quatOfMat3(m);
            j.frameA = normalize(conjugate(xa.q) * frame);
            j.frameB = normalize(conjugate(xb.q) * frame);
        }
        uint32_t index = (uint32_t)W.joints.size();
        if (!W.freeJoints.empty()) {
            index = W.freeJoints.back();
            W.freeJoints.pop_back();
            hj.generation = W.joints[index].generation;
            W.joints[index] = hj;
        } else {
            W.joints.push_back(hj);
        }
        // The joined bodies' contacts go, touching pairs ending now (src/world.cpp:2317-2327); the joint's
        // dynamic ends wake.
        if (!d->collide_connected && ai != kWorldEnd) {
            auto between = [&](const DContact& c) {
                return (c.bodyA == ai && c.bodyB == bi) || (c.bodyA == bi && c.bodyB == ai);
            };
            for (size_t ci = 0; ci < W.contacts.size(); ++ci) {
                const DContact& c = W.contacts[ci];
                if ((c.flags & kCTouched) && between(c) && (ci == 0 || W.contacts[ci - 1].key != c.key)) {
                    W.queued.push_back(endEvent(W, c));
                }
            }
            W.contacts.erase(std::remove_if(W.contacts.begin(), W.contacts.end(), between), W.contacts.end());
        }
        wakeJoint(W, W.joints[index].d);
        layoutDirty = true;
        if (out) { *out = { index, hj.generation }; }
        return TF_OK;
    }

    // The joint's host record for a change through the API, or null for an invalid id (the reference's
    // setters then do nothing). Changes other than the break limits wake the joint's dynamic ends after they
    // are made (src/world.cpp:2341-2397).
    int jointForChange(int w, tf_id id, bool wakes, HostJoint** out) {
        *out = nullptr;
        if (w < 0 || w >= (int)worlds.size()) { return fail(TF_E_INVALID, "joint: bad world"); }
        int rc = pull();
        if (rc != TF_OK) { return rc; }
        HostWorld& W = worlds[(size_t)w];
        if (id.index >= W.joints.size() || !W.joints[id.index].d.alive || W.joints[id.index].generation != id.generation) {
            return TF_OK;
        }
        HostJoint& j = W.joints[id.index];
        (void)wakes;
        *out = &j;
        return TF_OK;
    }

    // World::setJointLimits, setJointMotor, setJointSpring, setJointFriction, setJointSwing, setJointBreakLimits
    // (src/world.cpp:2341-2397) and destroyJoint (:399-406).
    int jointSet(int w, tf_id id, int what, const float* v) {
        HostJoint* hj = nullptr;
        const int rc = jointForChange(w, id, what != 5, &hj);
        if (rc != TF_OK || !hj) { return rc; }
        DJoint& j = hj->d;
        switch (what) {
            case 0:  // limits: limited, lower, upper
                j.limited = (v[0] != 0.0f && (j.type != kJointSwingTwist || v[2] - v[1] < 2.0f * kJointPi)) ? 1u : 0u;
                j.lower = v[1];
                j.upper = v[2];
                j.lowerImpulse = 0.0f;
                j.upperImpulse = 0.0f;
                break;
            case 1:  // motor: speed, max force or torque
                j.motorSpeed = v[0];
                j.maxMotor = v[1];
                break;
            case 2:  // spring: hertz, damping ratio
                j.hertz = v[0];
                j.dampingRatio = v[1];
                break;
            case 3:  // friction
                j.maxFriction = v[0];
                if (!(v[0] > 0.0f)) {
                    j.frictionImpulse = 0.0f;
                    j.frictionTurn = zero3();
                }
                break;
            case 4:  // swing cone, as sines of the half angles
                j.swingY = v[0] >= kJointPi ? 1.0f : (float)std::sin((double)(0.5f * maxf(v[0], 1e-3f)));
                j.swingZ = v[1] >= kJointPi ? 1.0f : (float)std::sin((double)(0.5f * maxf(v[1], 1e-3f)));
                j.swingImpulse = 0.0f;
                break;
            case 5:  // break limits
                j.breakForce = v[0];
                j.breakTorque = v[1];
                break;
            default:
                return fail(TF_E_INVALID, "joint: unknown change");
        }
        if (what != 5) { wakeJoint(worlds[(size_t)w], j); }
        layoutDirty = true;
        return TF_OK;
    }

    int destroyJoint(int w, tf_id id) {
        HostJoint* hj = nullptr;
        const int rc = jointForChange(w, id, true, &hj);
        if (rc != TF_OK || !hj) { return rc; }
        killJoint(worlds[(size_t)w], id.index);
        return TF_OK;
    }

    // World::jointInfo (src/world.cpp:410-425) from the host mirrors.
    int jointInfo(int w, tf_id id, tf_joint_info* out) {
        if (w < 0 || w >= (int)worlds.size() || !out) { return fail(TF_E_INVALID, "jointInfo: bad world"); }
        int rc = pull();
        if (rc != TF_OK) { return rc; }
        const HostWorld& W = worlds[(size_t)w];
        std::memset(out, 0, sizeof(*out));
        out->body_a = UINT32_MAX;
        if (id.index >= W.joints.size() || W.joints[id.index].generation != id.generation || !W.joints[id.index].d.alive) {
            return TF_OK;  // an invalid id reads as defaults, as the reference's getters do
        }
        const DJoint& j = W.joints[id.index].d;
        const JBody a = j.bodyA == kWorldEnd ? worldEnd() : jointBodyOf(W.bodies[j.bodyA].d);
        const JBody b = jointBodyOf(W.bodies[j.bodyB].d);
        out->type = (int32_t)j.type;
        out->body_a = j.bodyA;
        out->body_b = j.bodyB;
        const Vec3 pa = apply(a.xf, j.localA), pb = apply(b.xf, j.localB), ax = rotate(a.xf.q, j.axisA);
        out->anchor_a[0] = pa.x, out->anchor_a[1] = pa.y, out->anchor_a[2] = pa.z;
        out->anchor_b[0] = pb.x, out->anchor_b[1] = pb.y, out->anchor_b[2] = pb.z;
        out->axis[0] = ax.x, out->axis[1] = ax.y, out->axis[2] = ax.z;
        out->value = jointValue(j, a, b);
        out->force[0] = j.force.x, out->force[1] = j.force.y, out->force[2] = j.force.z;
        out->torque[0] = j.torque.x, out->torque[1] = j.torque.y, out->torque[2] = j.torque.z;
        out->broken = j.broken ? 1 : 0;
        return TF_OK;
    }

    // World::brokenJoints (src/world.cpp:2413-2420): joints that broke in the last step, in index order.
    int brokenJoints(int w, tf_id* out, int cap, int* count) {
        if (w < 0 || w >= (int)worlds.size() || !count) { return fail(TF_E_INVALID, "brokenJoints: bad world"); }
        int rc = pull();
        if (rc != TF_OK) { return rc; }
        const HostWorld& W = worlds[(size_t)w];
        int n = 0;
        for (size_t k = 0; k < W.joints.size(); ++k) {
            if (!W.joints[k].d.brokeNow || !W.joints[k].d.alive) { continue; }
            if (out && n < cap) { out[n] = { (uint32_t)k, W.joints[k].generation }; }
            ++n;
        }
        *count = n;
        return TF_OK;
    }

    int pull() {
        if (!onDevice || hostFresh) { return TF_OK; }
        TF_CUDA(cudaStreamSynchronize(stream));
        std::vector<DBody> bodies(totalBodies);
        std::vector<DShape> shapes(totalShapes);
        std::vector<WorldCounts> counts(worlds.size());
        TF_CUDA(cudaMemcpy(bodies.data(), dBodies.ptr, totalBodies * sizeof(DBody), cudaMemcpyDeviceToHost));
        TF_CUDA(cudaMemcpy(shapes.data(), dShapes.ptr, totalShapes * sizeof(DShape), cudaMemcpyDeviceToHost));
        TF_CUDA(cudaMemcpy(counts.data(), dCounts.ptr, worlds.size() * sizeof(WorldCounts), cudaMemcpyDeviceToHost));
        minCandCap.resize(worlds.size(), 0);
        minContactCap.resize(worlds.size(), 0);
        for (size_t w = 0; w < worlds.size(); ++w) {
            HostWorld& W = worlds[w];
            const WorldInfo& wi = info[w];
            if (counts[w].candNeeded > wi.candCap) {
                minCandCap[w] = std::max(minCandCap[w], counts[w].candNeeded + counts[w].candNeeded / 4 + 64);
            }
            if (counts[w].contactNeeded > wi.contactCap) {
                minContactCap[w] = std::max(minContactCap[w], counts[w].contactNeeded + counts[w].contactNeeded / 4 + 64);
            }
            for (size_t i = 0; i < W.bodies.size(); ++i) {
                DBody d = bodies[wi.bodyFirst + i];
                // Keep the host's own bookkeeping fields.
                d.shapeFirst = W.bodies[i].d.shapeFirst;
                d.shapeCount = W.bodies[i].d.shapeCount;
                d.world = W.bodies[i].d.world;
                W.bodies[i].d = d;
            }
            for (size_t i = 0; i < W.shapes.size(); ++i) {
                W.shapes[i].d.lo = shapes[wi.shapeFirst + i].lo;
                W.shapes[i].d.hi = shapes[wi.shapeFirst + i].hi;
            }
            const uint32_t nc = std::min(counts[w].contactCount, wi.contactCap);
            W.contacts.resize(nc);
            if (nc) {
                TF_CUDA(cudaMemcpy(W.contacts.data(), dContacts[cur].ptr + wi.contactFirst, nc * sizeof(DContact),
                                   cudaMemcpyDeviceToHost));
            }
            for (DContact& c : W.contacts) {
                c.bodyA -= wi.bodyFirst;
                c.bodyB -= wi.bodyFirst;
                c.shapeA -= wi.shapeFirst;
                c.shapeB -= wi.shapeFirst;
            }
            if (!W.joints.empty() && wi.jointCount == W.joints.size()) {
                std::vector<DJoint> js(W.joints.size());
                TF_CUDA(cudaMemcpy(js.data(), dJoints.ptr + wi.jointFirst, js.size() * sizeof(DJoint), cudaMemcpyDeviceToHost));
                for (size_t k = 0; k < js.size(); ++k) {
                    DJoint j = js[k];
                    if (j.bodyA != kWorldEnd) { j.bodyA -= wi.bodyFirst; }
                    j.bodyB -= wi.bodyFirst;
                    W.joints[k].d = j;
                }
            }
        }
        hostFresh = true;
        return TF_OK;
    }

    int layout() {
        ++layoutGen;
        bodyStepsBase = bodyStepsTotal;
        dropGraphs();
        const size_t nw = worlds.size();
        info.assign(nw, WorldInfo{});
        size_t nb = 0, ns = 0, ncand = 0, ncon = 0, nplanes = 0, nparts = 0, nbounds = 0, njoints = 0;
        std::vector<DPoly> polys;
        std::vector<Vec3> verts, normals, arcs;
        std::vector<int32_t> indices;
        std::vector<DFace> faces;
        std::vector<float> offsets;
        std::vector<DEdge> edges;
        uint32_t maxCap = 0, maxBodies = 0, maxContacts = 0;
        minCandCap.resize(nw, 0);
        minContactCap.resize(nw, 0);
        for (size_t w = 0; w < nw; ++w) {
            const HostWorld& W = worlds[w];
            WorldInfo& wi = info[w];
            wi.bodyFirst = (uint32_t)nb;
            wi.bodyCount = (uint32_t)W.bodies.size();
            wi.shapeFirst = (uint32_t)ns;
            wi.shapeCount = (uint32_t)W.shapes.size();
            wi.planeFirst = (uint32_t)nplanes;
            wi.planeCount = (uint32_t)W.planes.size();
            wi.planeBody = UINT32_MAX;
            for (size_t i = 0; i < W.bodies.size(); ++i) {
                if (W.bodies[i].d.alive && isPlanar(W.bodies[i].d)) {
                    wi.planeBody = wi.bodyFirst + (uint32_t)i;
                    break;
                }
            }
            const uint32_t cap = std::max((uint32_t)std::ceil(capFactor * (float)W.shapes.size()) + 64u, minCandCap[w]);
            wi.candFirst = (uint32_t)ncand;
            wi.candCap = cap;
            wi.contactFirst = (uint32_t)ncon;
            wi.contactCap = std::max({ cap + 64u, (uint32_t)W.contacts.size() + 64u, minContactCap[w] });
            maxBodies = std::max(maxBodies, wi.bodyCount);
            maxContacts = std::max(maxContacts, wi.contactCap);
            bool hasMesh = false;
            for (const HostShape& hs : W.shapes) { hasMesh = hasMesh || (hs.d.alive && hs.d.kind == kMesh); }
            wi.partFirst = (uint32_t)nparts;
            wi.partCap = hasMesh ? cap : 0u;
            wi.boundsFirst = (uint32_t)nbounds;
            wi.boundsCap = hasMesh ? 16u * cap : 0u;
            nparts += wi.partCap;
            nbounds += wi.boundsCap;
            wi.jointFirst = (uint32_t)njoints;
            wi.jointCount = (uint32_t)W.joints.size();
            njoints += wi.jointCount;
            nb += wi.bodyCount;
            ns += wi.shapeCount;
            nplanes += wi.planeCount;
            ncand += wi.candCap;
            ncon += wi.contactCap;
            maxCap = std::max(maxCap, cap);
        }
        totalBodies = nb;
        totalShapes = ns;
        totalCand = ncand;
        totalContacts = ncon;
        std::vector<DBody> bodies(nb);
        std::vector<DShape> shapes(ns);
        std::vector<uint32_t> shapeList(ns), planeList(std::max<size_t>(nplanes, 1));
        std::vector<DJoint> joints(std::max<size_t>(njoints, 1));
        std::vector<uint64_t> joined(std::max<size_t>(njoints, 1));
        // Contacts carried over from the device: packed, with one (slot, first, count) run per world.
        std::vector<DContact> packed;
        std::vector<size_t> runSlot, runFirst, runCount;
        std::vector<WorldCounts> counts(nw);
        for (size_t w = 0; w < nw; ++w) {
            HostWorld& W = worlds[w];
            const WorldInfo& wi = info[w];
            uint32_t listPos = wi.shapeFirst;
            for (size_t i = 0; i < W.bodies.size(); ++i) {
                HostBody& hb = W.bodies[i];
                DBody d = hb.d;
                d.shapeFirst = listPos;
                d.shapeCount = (uint32_t)hb.shapes.size();
                d.world = (uint32_t)w;
                for (uint32_t si : hb.shapes) { shapeList[listPos++] = wi.shapeFirst + si; }
                hb.d.shapeFirst = d.shapeFirst;
                hb.d.shapeCount = d.shapeCount;
                hb.d.world = d.world;
                bodies[wi.bodyFirst + i] = d;
            }
            for (size_t i = 0; i < W.shapes.size(); ++i) {
                const HostShape& s = W.shapes[i];
                DShape d = s.d;
                d.body = wi.bodyFirst + s.d.body;
                d.poly = -1;
                if (s.hasPoly && s.d.alive) {
                    DPoly p{};
                    p.vFirst = (int32_t)verts.size();
                    p.vCount = (int32_t)s.poly.vertices.size();
                    p.fFirst = (int32_t)normals.size();
                    p.fCount = (int32_t)s.poly.faces.size();
                    p.eFirst = (int32_t)edges.size();
                    p.eCount = (int32_t)s.poly.edges.size();
                    p.iFirst = (int32_t)indices.size();
                    p.iCount = (int32_t)s.poly.indices.size();
                    p.centroid = s.poly.centroid;
                    p.lo = s.poly.lo;
                    p.hi = s.poly.hi;
                    verts.insert(verts.end(), s.poly.vertices.begin(), s.poly.vertices.end());
                    normals.insert(normals.end(), s.poly.normals.begin(), s.poly.normals.end());
                    offsets.insert(offsets.end(), s.poly.offsets.begin(), s.poly.offsets.end());
                    faces.insert(faces.end(), s.poly.faces.begin(), s.poly.faces.end());
                    edges.insert(edges.end(), s.poly.edges.begin(), s.poly.edges.end());
                    arcs.insert(arcs.end(), s.poly.arcs.begin(), s.poly.arcs.end());
                    indices.insert(indices.end(), s.poly.indices.begin(), s.poly.indices.end());
                    d.poly = (int32_t)polys.size();
                    polys.push_back(p);
                }
                shapes[wi.shapeFirst + i] = d;
            }
            for (size_t k = 0; k < W.planes.size(); ++k) { planeList[wi.planeFirst + k] = wi.shapeFirst + W.planes[k]; }
            // Joints with global ends, and the sorted pairs that joints keep from colliding
            // (src/world.cpp:375-383).
            std::vector<uint64_t> keys;
            for (size_t k = 0; k < W.joints.size(); ++k) {
                DJoint j = W.joints[k].d;
                if (j.alive && !j.collideConnected && j.bodyA != kWorldEnd) {
                    keys.push_back(((uint64_t)std::min(j.bodyA, j.bodyB) << 32) | (uint64_t)std::max(j.bodyA, j.bodyB));
                }
                if (j.bodyA != kWorldEnd) { j.bodyA += wi.bodyFirst; }
                j.bodyB += wi.bodyFirst;
                joints[wi.jointFirst + k] = j;
            }
            std::sort(keys.begin(), keys.end());
            info[w].joinedCount = (uint32_t)keys.size();
            for (size_t k = 0; k < keys.size(); ++k) { joined[wi.jointFirst + k] = keys[k]; }
            if (!W.contacts.empty()) {
                runSlot.push_back(wi.contactFirst);
                runFirst.push_back(packed.size());
                runCount.push_back(std::min<size_t>(W.contacts.size(), wi.contactCap));
            }
            for (size_t k = 0; k < W.contacts.size() && k < wi.contactCap; ++k) {
                DContact c = W.contacts[k];
                c.bodyA += wi.bodyFirst;
                c.bodyB += wi.bodyFirst;
                c.shapeA += wi.shapeFirst;
                c.shapeB += wi.shapeFirst;
                packed.push_back(c);
            }
            counts[w] = WorldCounts{};
            counts[w].contactCount = (uint32_t)std::min<size_t>(W.contacts.size(), wi.contactCap);
        }
        order.resize(nw);
        for (size_t w = 0; w < nw; ++w) { order[w] = (uint32_t)w; }
        std::stable_sort(order.begin(), order.end(),
                         [&](uint32_t a, uint32_t b) { return info[a].bodyCount > info[b].bodyCount; });
        maxWorldBodies = maxBodies;
        maxWorldContacts = maxContacts;
        {
            std::vector<uint32_t> sizes(nw);
            for (size_t w = 0; w < nw; ++w) { sizes[w] = info[w].bodyCount; }
            std::sort(sizes.begin(), sizes.end(), std::greater<uint32_t>());
            medianWorldBodies = nw ? sizes[nw / 2] : 0;
            sortedSizes = std::move(sizes);
        }
        hasJoints = njoints > 0;
        smallBatch = ncand <= kSmallBatchCandidates;
        laidOut = true;
        {
            const int rc0 = configureLaunches();
            if (rc0 != TF_OK) { return rc0; }
        }

        int rc;
#define TF_ALLOC(arr, count) \
    if ((rc = (arr).alloc(count)) != TF_OK) { return rc; }
        TF_ALLOC(dInfo, nw);
        TF_ALLOC(dCounts, nw);
        TF_ALLOC(dOrder, nw);
        TF_ALLOC(dBodies, nb);
        TF_ALLOC(dShapes, ns);
        TF_ALLOC(dShapeList, ns);
        TF_ALLOC(dPlaneList, planeList.size());
        TF_ALLOC(dPolys, polys.size());
        TF_ALLOC(dVerts, verts.size());
        TF_ALLOC(dNormals, normals.size());
        TF_ALLOC(dArcs, arcs.size());
        TF_ALLOC(dIndices, indices.size());
        TF_ALLOC(dFaces, faces.size());
        TF_ALLOC(dOffsets, offsets.size());
        TF_ALLOC(dEdges, edges.size());
        // The meshes, shared by every world: each mesh's arrays one after another.
        std::vector<DMesh> meshRecs(meshes.size());
        std::vector<Vec3> meshVerts, meshNormals;
        std::vector<uint32_t> meshIndices;
        std::vector<uint8_t> meshEdges;
        std::vector<MeshNode> meshNodes;
        for (size_t m = 0; m < meshes.size(); ++m) {
            const HostMesh& hm = meshes[m];
            meshRecs[m] = { (int32_t)meshVerts.size(), (int32_t)hm.vertices.size(), (int32_t)meshNormals.size(),
                            (int32_t)hm.normals.size(), (int32_t)meshNodes.size(), (int32_t)hm.nodes.size() };
            meshVerts.insert(meshVerts.end(), hm.vertices.begin(), hm.vertices.end());
            meshIndices.insert(meshIndices.end(), hm.indices.begin(), hm.indices.end());
            meshNormals.insert(meshNormals.end(), hm.normals.begin(), hm.normals.end());
            meshEdges.insert(meshEdges.end(), hm.edges.begin(), hm.edges.end());
            meshNodes.insert(meshNodes.end(), hm.nodes.begin(), hm.nodes.end());
        }
        TF_ALLOC(dMeshes, meshRecs.size());
        TF_ALLOC(dMeshVerts, meshVerts.size());
        TF_ALLOC(dMeshIndices, meshIndices.size());
        TF_ALLOC(dMeshNormals, meshNormals.size());
        TF_ALLOC(dMeshEdges, meshEdges.size());
        TF_ALLOC(dMeshNodes, meshNodes.size());
        TF_ALLOC(dGrow, nb);
        TF_ALLOC(dIslandTime, nb);
        TF_ALLOC(dBodyColors, nb);
        TF_ALLOC(dUnionParent, nb);
        TF_ALLOC(dStruck, nb);
        TF_ALLOC(dWakeMark, nb);
        TF_ALLOC(dCand, ncand);
        TF_ALLOC(dStage, ncand);
        TF_ALLOC(dStageUsed, ncand);
        TF_ALLOC(dStagePart, ncand);
        TF_ALLOC(dStageExtra, nparts);
        TF_ALLOC(dTriBounds, nbounds);
        TF_ALLOC(dContacts[0], ncon);
        TF_ALLOC(dContacts[1], ncon);
        TF_ALLOC(dActive, ncon);
        TF_ALLOC(dImpact, ncon);
        TF_ALLOC(dColored, ncon);
        TF_ALLOC(dImpactColored, ncon);
        TF_ALLOC(dRest, ncon);
        TF_ALLOC(dImpactRest, ncon);
        TF_ALLOC(dRestLevel, ncon);
        TF_ALLOC(dImpactRestLevel, ncon);
        TF_ALLOC(dColor, ncon);
        TF_ALLOC(dCflags, ncon);
        TF_ALLOC(dAxes, ncon * kAxesPerContact);
        TF_ALLOC(dRows, ncon * kRowWords);
        TF_ALLOC(dSlotOf, ncon);
        TF_ALLOC(dFlatBodies, nb * kFlatBodyWords);
        TF_ALLOC(dFlatPose, nb * kFlatPoseWords);
        TF_ALLOC(dFlatMotion, nb * kFlatMotionWords);
        TF_ALLOC(dFlatColored, ncon);
        TF_ALLOC(dFlatImpact, ncon);
        TF_ALLOC(dMergeKeyA, ncon);
        TF_ALLOC(dMergeKeyB, ncon);
        TF_ALLOC(dMergePartA, ncon);
        TF_ALLOC(dMergePartB, ncon);
        TF_ALLOC(dMergeIdxA, ncon);
        TF_ALLOC(dMergeIdxB, ncon);
        TF_ALLOC(dJoints, joints.size());
        TF_ALLOC(dJoined, joined.size());
        TF_ALLOC(dTouchEvents, 2 * ncon);
        TF_ALLOC(dHitEvents, ncon);
        TF_ALLOC(dWork, kSlotCount);
        TF_ALLOC(dCandItems, ncand * kPairClasses);
        TF_ALLOC(dContactItems, ncon * (kPairClasses + 1));
        TF_ALLOC(dRowScratch, ns);
        TF_ALLOC(dRowLong, ns);
        TF_ALLOC(dRowCount, ns);
        bigWorlds.clear();
        bigBodyStart.assign(1, 0u);
        for (uint32_t w : order) {
            if (info[w].bodyCount > kSweepBodies) {
                bigWorlds.push_back(w);
                bigBodyStart.push_back(bigBodyStart.back() + info[w].bodyCount);
            }
        }
        TF_ALLOC(dSweepLo, nb);
        TF_ALLOC(dSweepHi, nb);
        TF_ALLOC(dSweepOrder, nb);
        TF_ALLOC(dSweepRecs, nb);
        TF_ALLOC(dSweepStart, nb + nw);
        TF_ALLOC(dBigWorlds, bigWorlds.size());
        TF_ALLOC(dBigBodyStart, bigBodyStart.size());
        TF_ALLOC(dSweptLo, ns);
        TF_ALLOC(dSweptHi, ns);
        TF_ALLOC(dSweepList, ns);
        TF_ALLOC(dHitParent, nb);
        TF_ALLOC(dHitKey, nb);
        TF_ALLOC(dGroupKey, nb);
        TF_ALLOC(dAbort, 1);
        TF_ALLOC(dDebug, 4);
        nPolys = polys.size();
#undef TF_ALLOC
        auto up = [&](void* dst, const void* src, size_t bytes) -> int {
            if (bytes == 0) { return TF_OK; }
            cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) { return fail(TF_E_CUDA, std::string("upload: ") + cudaGetErrorString(e)); }
            return TF_OK;
        };
        cur = 0;
        if ((rc = up(dInfo.ptr, info.data(), nw * sizeof(WorldInfo))) != TF_OK) { return rc; }
        if ((rc = up(dCounts.ptr, counts.data(), nw * sizeof(WorldCounts))) != TF_OK) { return rc; }
        if ((rc = up(dOrder.ptr, order.data(), nw * sizeof(uint32_t))) != TF_OK) { return rc; }
        if ((rc = up(dBodies.ptr, bodies.data(), nb * sizeof(DBody))) != TF_OK) { return rc; }
        if ((rc = up(dShapes.ptr, shapes.data(), ns * sizeof(DShape))) != TF_OK) { return rc; }
        if ((rc = up(dShapeList.ptr, shapeList.data(), ns * sizeof(uint32_t))) != TF_OK) { return rc; }
        if ((rc = up(dPlaneList.ptr, planeList.data(), planeList.size() * sizeof(uint32_t))) != TF_OK) { return rc; }
        if ((rc = up(dJoints.ptr, joints.data(), joints.size() * sizeof(DJoint))) != TF_OK) { return rc; }
        if ((rc = up(dJoined.ptr, joined.data(), joined.size() * sizeof(uint64_t))) != TF_OK) { return rc; }
        if ((rc = up(dPolys.ptr, polys.data(), polys.size() * sizeof(DPoly))) != TF_OK) { return rc; }
        if ((rc = up(dVerts.ptr, verts.data(), verts.size() * sizeof(Vec3))) != TF_OK) { return rc; }
        if ((rc = up(dNormals.ptr, normals.data(), normals.size() * sizeof(Vec3))) != TF_OK) { return rc; }
        if ((rc = up(dArcs.ptr, arcs.data(), arcs.size() * sizeof(Vec3))) != TF_OK) { return rc; }
        if ((rc = up(dIndices.ptr, indices.data(), indices.size() * sizeof(int32_t))) != TF_OK) { return rc; }
        if ((rc = up(dFaces.ptr, faces.data(), faces.size() * sizeof(DFace))) != TF_OK) { return rc; }
        if ((rc = up(dOffsets.ptr, offsets.data(), offsets.size() * sizeof(float))) != TF_OK) { return rc; }
        if ((rc = up(dEdges.ptr, edges.data(), edges.size() * sizeof(DEdge))) != TF_OK) { return rc; }
        if ((rc = up(dBigWorlds.ptr, bigWorlds.data(), bigWorlds.size() * sizeof(uint32_t))) != TF_OK) { return rc; }
        if ((rc = up(dBigBodyStart.ptr, bigBodyStart.data(), bigBodyStart.size() * sizeof(uint32_t))) != TF_OK) { return rc; }
        if ((rc = up(dMeshes.ptr, meshRecs.data(), meshRecs.size() * sizeof(DMesh))) != TF_OK) { return rc; }
        if ((rc = up(dMeshVerts.ptr, meshVerts.data(), meshVerts.size() * sizeof(Vec3))) != TF_OK) { return rc; }
        if ((rc = up(dMeshIndices.ptr, meshIndices.data(), meshIndices.size() * sizeof(uint32_t))) != TF_OK) { return rc; }
        if ((rc = up(dMeshNormals.ptr, meshNormals.data(), meshNormals.size() * sizeof(Vec3))) != TF_OK) { return rc; }
        if ((rc = up(dMeshEdges.ptr, meshEdges.data(), meshEdges.size() * sizeof(uint8_t))) != TF_OK) { return rc; }
        if ((rc = up(dMeshNodes.ptr, meshNodes.data(), meshNodes.size() * sizeof(MeshNode))) != TF_OK) { return rc; }
        for (size_t r = 0; r < runSlot.size(); ++r) {
            if ((rc = up(dContacts[0].ptr + runSlot[r], packed.data() + runFirst[r], runCount[r] * sizeof(DContact))) != TF_OK) {
                return rc;
            }
        }
        TF_CUDA(cudaMemset(dWakeMark.ptr, 0, nb));
        TF_CUDA(cudaMemset(dDebug.ptr, 0, 4 * sizeof(uint32_t)));
        layoutDirty = false;
        bodiesDirty = false;
        onDevice = true;
        hostFresh = true;
        return TF_OK;
    }

    // Pushes host body state (after a setter) without changing the layout.
    int pushBodies() {
        std::vector<DBody> bodies(totalBodies);
        for (size_t w = 0; w < worlds.size(); ++w) {
            for (size_t i = 0; i < worlds[w].bodies.size(); ++i) { bodies[info[w].bodyFirst + i] = worlds[w].bodies[i].d; }
        }
        TF_CUDA(cudaMemcpy(dBodies.ptr, bodies.data(), totalBodies * sizeof(DBody), cudaMemcpyHostToDevice));
        bodiesDirty = false;
        return TF_OK;
    }

    int prepareDevice() {
        const int rc0 = ensureDevice();
        if (rc0 != TF_OK) { return rc0; }
        if (layoutDirty) {
            int rc = pull();
            if (rc != TF_OK) { return rc; }
            return layout();
        }
        if (bodiesDirty) { return pushBodies(); }
        return TF_OK;
    }

    StepParams params(float dt) const {
        StepParams P{};
        const tf_settings& s = settings;
        const int n = std::min(kMaxSubsteps, std::max(1, (int)s.substeps));
        P.gravity = v3of(s.gravity);
        P.lengthUnit = s.length_unit;
        P.substeps = n;
        P.dt = dt;
        P.h = dt / (float)n;
        P.invH = 1.0f / P.h;
        const float hertz = minf(s.contact_hertz, 0.25f * P.invH);
        P.contactSoft = makeSoft(hertz, s.contact_damping_ratio, P.h);
        P.staticSoft = makeSoft(2.0f * hertz, s.contact_damping_ratio, P.h);
        P.maxPushout = s.max_pushout_speed * s.length_unit;
        P.restitutionThreshold = s.restitution_threshold * s.length_unit;
        P.maxLinearSpeed = s.max_linear_speed * s.length_unit;
        P.maxAngularSpeed = s.max_angular_speed;
        P.sleepThreshold = s.sleep_threshold * s.length_unit;
        P.timeToSleep = s.time_to_sleep;
        P.reuseDistance = s.contact_reuse_distance * s.length_unit;
        P.reuseCos = std::cos(0.5f * s.contact_reuse_angle);
        P.featureTurnCos = std::cos(0.5f * kFeatureTurn);
        P.treeMargin = kTreeMargin * s.length_unit;
        P.tol.linearSlop = 0.005f * s.length_unit;
        P.tol.speculative = 4.0f * P.tol.linearSlop;
        P.continuous = s.continuous;
        P.hitThreshold = s.hit_threshold * s.length_unit;
        P.jointSoft = makeSoft(minf(s.joint_hertz, 0.5f * P.invH), s.joint_damping_ratio, P.h);
        return P;
    }

    Batch batch(int cur_) {
        Batch B{};
        B.nWorlds = (int)worlds.size();
        B.order = dOrder.ptr;
        B.abortStep = dAbort.ptr;
        B.info = dInfo.ptr;
        B.counts = dCounts.ptr;
        B.bodies = dBodies.ptr;
        B.shapes = dShapes.ptr;
        B.shapeList = dShapeList.ptr;
        B.planeList = dPlaneList.ptr;
        B.cx.pt = { dPolys.ptr, dVerts.ptr, dIndices.ptr, dFaces.ptr, dNormals.ptr, dOffsets.ptr, dEdges.ptr, dArcs.ptr };
        B.cx.boxes = boxTopology;
        // The cap circle and the turn between its points, from the host's C library as the reference takes
        // them (src/collide3d.cpp:724-731, 1161-1164).
        for (int k = 0; k < kCapPoints; ++k) {
            const float t = 2.0f * 3.14159265358979f * (float)k / (float)kCapPoints;
            B.cx.cap.cos[k] = std::cos(t);
            B.cx.cap.sin[k] = std::sin(t);
        }
        {
            const float t = 2.0f * 3.14159265358979f / (float)kCapPoints;
            B.cx.cap.turnCos = std::cos(t);
            B.cx.cap.turnSin = std::sin(t);
        }
        B.cx.mt = { dMeshes.ptr, dMeshVerts.ptr, dMeshIndices.ptr, dMeshNormals.ptr, dMeshEdges.ptr, dMeshNodes.ptr };
        B.grow = dGrow.ptr;
        B.bodyColors = dBodyColors.ptr;
        B.struck = dStruck.ptr;
        B.wakeMark = dWakeMark.ptr;
        B.unionParent = dUnionParent.ptr;
        B.islandTime = dIslandTime.ptr;
        B.cand = dCand.ptr;
        B.stage = dStage.ptr;
        B.stageUsed = dStageUsed.ptr;
        B.stagePart = dStagePart.ptr;
        B.stageExtra = dStageExtra.ptr;
        B.triBounds = dTriBounds.ptr;
        B.contacts = dContacts[cur_].ptr;
        B.previous = dContacts[1 - cur_].ptr;
        B.active = dActive.ptr;
        B.impact = dImpact.ptr;
        B.colored = dColored.ptr;
        B.impactColored = dImpactColored.ptr;
        B.rest = dRest.ptr;
        B.impactRest = dImpactRest.ptr;
        B.restLevel = dRestLevel.ptr;
        B.impactRestLevel = dImpactRestLevel.ptr;
        B.color = dColor.ptr;
        B.cflags = dCflags.ptr;
        B.axes = dAxes.ptr;
        B.rows = dRows.ptr;
        B.rowStride = dContacts[0].n;
        B.slotOf = dSlotOf.ptr;
        B.flatBodies = dFlatBodies.ptr;
        B.flatPose = dFlatPose.ptr;
        B.flatMotion = dFlatMotion.ptr;
        B.flatColored = dFlatColored.ptr;
        B.flatImpact = dFlatImpact.ptr;
        B.mergeKeyA = dMergeKeyA.ptr;
        B.mergePartA = dMergePartA.ptr;
        B.mergeIdxA = dMergeIdxA.ptr;
        B.mergeKeyB = dMergeKeyB.ptr;
        B.mergePartB = dMergePartB.ptr;
        B.mergeIdxB = dMergeIdxB.ptr;
        B.joints = dJoints.ptr;
        B.joined = dJoined.ptr;
        B.touchEvents = dTouchEvents.ptr;
        B.hitEvents = dHitEvents.ptr;
        B.work = dWork.ptr;
        B.candItems = dCandItems.ptr;
        B.contactItems = dContactItems.ptr;
        B.candItemStride = (uint32_t)(dCandItems.n / kPairClasses);
        B.contactItemStride = (uint32_t)(dContactItems.n / (kPairClasses + 1));
        B.rowScratch = dRowScratch.ptr;
        B.rowLong = dRowLong.ptr;
        B.rowCount = dRowCount.ptr;
        B.sweepLo = dSweepLo.ptr;
        B.sweepHi = dSweepHi.ptr;
        B.sweepOrder = dSweepOrder.ptr;
        B.sweepRecs = dSweepRecs.ptr;
        B.sweepStart = dSweepStart.ptr;
        B.bigWorlds = dBigWorlds.ptr;
        B.bigBodyStart = dBigBodyStart.ptr;
        B.nBigWorlds = (uint32_t)bigWorlds.size();
        B.sweptLo = dSweptLo.ptr;
        B.sweptHi = dSweptHi.ptr;
        B.sweepList = dSweepList.ptr;
        B.hitParent = dHitParent.ptr;
        B.hitKey = dHitKey.ptr;
        B.groupKey = dGroupKey.ptr;
        B.debug = dDebug.ptr;
        B.nPolys = (uint32_t)nPolys;
        B.totalBodies = (uint32_t)totalBodies;
        return B;
    }

    // Issues one step on the stream: the new contact list goes into buffer `into`, the old one is read from
    // the other buffer.
    int enqueueStep(float dt, int into, int serial, cudaEvent_t* marks, bool capturing = false) {
        const StepParams P = params(dt);
        Batch B = batch(into);
        B.cx.tol = P.tol;
        const bool rec = profiling && !capturing;
        auto threads = [&](int k) { return (int)shapes[k].threads; };
        auto smem = [&](int k) { return (size_t)splits[k].smemBytes; };
        cudaMemsetAsync(dWork.ptr, 0, kSlotCount * sizeof(uint32_t), stream);
        if (marks) { cudaEventRecord(marks[0], stream); }
        timed(0, rec, [&] {
            launch(kKBroadphase, grids[0], threads(0), smem(0), B, P, splits[0], serial);
            if (!bigWorlds.empty()) {
                launch(kKBroadPairs, smCount * 8, 256, 0, B, serial);
                launch(kKBroadFinish, grids[0], threads(0), 0, B, splits[0], serial);
            }
        });
        if (marks) { cudaEventRecord(marks[1], stream); }
        timed(7, rec, [&] {
            if (smallBatch) {
                launch(kKCollideAll, *std::max_element(flatGrids, flatGrids + kPairClasses), threads(7), 0, B, P, serial);
                return;
            }
            for (int c = 0; c < kPairClasses; ++c) { launch(kKCollide + c, flatGrids[c], flatThreads(c), 0, B, P, serial); }
        });
        timed(1, rec, [&] { launch(kKNarrowphase, grids[1], threads(1), 0, B, P, splits[1], serial); });
        timed(2, rec, [&] { launch(kKWake, grids[2], threads(2), 0, B, splits[2], serial); });
        if (marks) { cudaEventRecord(marks[2], stream); }
        timed(3, rec, [&] { launch(kKPrepare, grids[3], threads(3), smem(3), B, P, splits[3], serial); });
        if (recording && !capturing) {
            const int rc = recordStep(B, serial);
            if (rc != TF_OK) { return rc; }
        }
        for (int i = 0; i < P.substeps; ++i) {
            if (i > 0) {
                timed(4, rec, [&] {
                    if (smallBatch) {
                        launch(kKRefreshAll, flatGrids[6], threads(4), 0, B, P, i, serial);
                        return;
                    }
                    launch(kKRefresh + kPairClasses, flatGrids[6], threads(4), 0, B, P, i, serial);
                    for (int c = 0; c < kPairClasses; ++c) {
                        launch(kKRefresh + c, flatGrids[7 + c], flatThreads(7 + c), 0, B, P, i, serial);
                    }
                });
            }
            timed(5, rec, [&] {
                if (shapes[5].flat) {
                    launchCooperative(hasJoints ? kKSubstepFlatJoints : kKSubstepFlat, grids[5], threads(5), B, P, i, serial);
                } else {
                    launch(hasJoints ? kKSubstepJoints : kKSubstep, grids[5], threads(5), smem(5), B, P, splits[5], i, serial);
                }
            });
        }
        timed(6, rec, [&] {
            launch(hasJoints ? kKFinishJoints : kKFinish, grids[6], threads(6), smem(6), B, P, splits[6], serial);
        });
        if (marks) { cudaEventRecord(marks[3], stream); }
        launches += smallBatch ? 5 + 1 + P.substeps + (P.substeps - 1) + (bigWorlds.empty() ? 0 : 2)
                               : 5 + kPairClasses + P.substeps + (kPairClasses + 1) * (P.substeps - 1) +
                                     (bigWorlds.empty() ? 0 : 2);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { return fail(TF_E_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e)); }
        return TF_OK;
    }

    int configureKernels() {
        if (kernelsConfigured) { return TF_OK; }
        bool& done = kernelsConfigured;
        int maxSmem = 0;
        TF_CUDA(cudaDeviceGetAttribute(&maxSmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
        // Dynamic shared memory may use what the kernel's static shared variables leave.
        auto allow = [&](const void* fn) -> int {
            cudaFuncAttributes a{};
            TF_CUDA(cudaFuncGetAttributes(&a, fn));
            TF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, maxSmem - (int)a.sharedSizeBytes));
            dynSmemLimit[fn] = (size_t)(maxSmem - (int)a.sharedSizeBytes);
            return TF_OK;
        };
        int rc;
        for (int id : { kKBroadphase, kKSubstep, kKSubstepJoints, kKPrepare, kKFinish, kKFinishJoints }) {
            if ((rc = allow(kernelEntry(id))) != TF_OK) { return rc; }
        }
        done = true;
        return TF_OK;
    }

    static bool flatKernel(int k) { return k == 4 || k == 7; }
    static constexpr uint32_t kMaxFlatBlock = 256;

    // Default launch shapes: batches of few worlds give every world a whole CTA (512 threads when a world
    // has more than 512 bodies); batches of many worlds give worlds of up to 96 bodies a warp each and the
    // larger ones the CTA. 64 KB of staging per CTA leaves room for three CTAs on an SM.
    LaunchShape defaultShape(int k) const {
        LaunchShape s;
        const bool many = worlds.size() >= (size_t)smCount * 4;
        s.threads = !many && maxWorldBodies > 512 && !flatKernel(k) ? 512u : 256u;
        s.bigBodies = many ? 96u : 0u;
        const bool stages = k == 0 || k == 3 || k == 5 || k == 6;
        s.smemBytes = stages ? 64u * 1024u : 0u;
        if (k == 5 && many) {
            // Batches of many worlds solve flat (k_substep_flat).
            s.threads = 256u;
            s.bigBodies = 0u;
            s.smemBytes = 0u;
            s.flat = true;
        }
        return s;
    }

    // Bodies (and active contacts) one staging slice of `bytes` holds, for the kernels that stage.
    static StageSizes stageFor(int k, uint32_t bytes) {
        StageSizes st{ 0, 0 };
        switch (k) {
            case 0:  // broadphase: a PairBody per body
                st.bodies = bytes / (uint32_t)sizeof(PairBody);
                break;
            case 3:  // prepare: a color mask and a mark per body, two endpoints per active contact, ~3 contacts per body
                st.bodies = bytes > 512 ? (bytes - 512) / 32 : 0;
                st.contacts = 3 * st.bodies + 64;
                break;
            case 5:  // substep: the solver state of each body
                st.bodies = bytes / (uint32_t)(kSBodyWords * sizeof(float));
                break;
            case 6:  // finish: parent and island time per body, a union pair per contact
                st.bodies = bytes > 512 ? (bytes - 512) / 32 : 0;
                st.contacts = 3 * st.bodies + 64;
                break;
            default:
                break;
        }
        if (st.contacts == 64 && st.bodies == 0) { st.contacts = 0; }
        return st;
    }

    // Threads per CTA of flat grid f (the pair collisions by class, then the refreshes: the other active contacts
    // and each class): the collide or refresh shape's, at most kMeshWarps warps for the mesh pairs, which a warp
    // each collides with the warp's shared room.
    static bool meshGrid(int f) { return f == kClassMesh || f == 7 + kClassMesh; }
    int flatThreads(int f) const {
        const int t = (int)shapes[f < kPairClasses ? 7 : 4].threads;
        return meshGrid(f) ? std::min(t, 32 * kMeshWarps) : t;
    }

    // Turns the launch shapes into kernel arguments and grid sizes for the current layout.
    int configureLaunches() {
        int rc = configureKernels();
        if (rc != TF_OK) { return rc; }
        for (int k = 0; k < kKernels; ++k) {
            LaunchShape& sh = shapes[k];
            if (!sh.chosen) { sh = defaultShape(k); }
            if (k == 5 && sh.flat) {
                // The flat solve: as many CTAs as are resident at once, all in one cooperative launch.
                int perSm = 0;
                TF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &perSm, kernelEntry(hasJoints ? kKSubstepFlatJoints : kKSubstepFlat), (int)sh.threads, 0));
                if (perSm < 1) { return fail(TF_E_INVALID, "launch shape does not fit on an SM"); }
                splits[k] = Split{};
                grids[k] = smCount * perSm;
                continue;
            }
            const void* fns[kKernels] = { kernelEntry(kKBroadphase), kernelEntry(kKNarrowphase), kernelEntry(kKWake),
                                          kernelEntry(kKPrepare),    kernelEntry(kKRefresh + kPairClasses),
                                          kernelEntry(hasJoints ? kKSubstepJoints : kKSubstep),
                                          kernelEntry(hasJoints ? kKFinishJoints : kKFinish),
                                          kernelEntry(kKCollide + kClassConvex) };
            const uint32_t warps = sh.threads / 32;
            auto lim = dynSmemLimit.find(fns[k]);
            const uint32_t limit = lim == dynSmemLimit.end() ? 0u : (uint32_t)lim->second;
            const uint32_t bytes = std::min(sh.smemBytes, limit) / (16 * warps) * (16 * warps);
            Split& sp = splits[k];
            sp.bigBodies = sh.bigBodies;
            sp.smemBytes = bytes;
            sp.big = stageFor(k, bytes);
            sp.small = stageFor(k, bytes / warps);
            int perSm = 0;
            TF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fns[k], (int)sh.threads, bytes));
            if (perSm < 1) { return fail(TF_E_INVALID, "launch shape does not fit on an SM"); }
            const size_t big = (size_t)(std::upper_bound(sortedSizes.begin(), sortedSizes.end(), sh.bigBodies,
                                                         std::greater<uint32_t>()) -
                                        sortedSizes.begin());
            const size_t needed = big + (sortedSizes.size() - big + warps - 1) / warps;
            grids[k] = flatKernel(k) ? smCount * perSm
                                     : (int)std::max<size_t>(1, std::min<size_t>(needed, (size_t)smCount * perSm));
        }
        // The flat kernels, one grid per instantiation: as many CTAs as fit on the device at once.
        const void* flat[kFlatGrids] = {
            kernelEntry(kKCollide + kClassSpheres),  kernelEntry(kKCollide + kClassSpherePoly),
            kernelEntry(kKCollide + kClassPlane),    kernelEntry(kKCollide + kClassConvex),
            kernelEntry(kKCollide + kClassPlanar),   kernelEntry(kKCollide + kClassMesh),
            kernelEntry(kKRefresh + kPairClasses),   kernelEntry(kKRefresh + kClassSpheres),
            kernelEntry(kKRefresh + kClassSpherePoly), kernelEntry(kKRefresh + kClassPlane),
            kernelEntry(kKRefresh + kClassConvex),   kernelEntry(kKRefresh + kClassPlanar),
            kernelEntry(kKRefresh + kClassMesh) };
        for (int f = 0; f < kFlatGrids; ++f) {
            int perSm = 0;
            const int threads = flatThreads(f);
            TF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, flat[f], threads, 0));
            if (perSm < 1) { return fail(TF_E_INVALID, "launch shape does not fit on an SM"); }
            // No more CTAs than the class list can ever fill: its capacity is the batch's candidate slots (pair
            // collisions) or contact slots (refreshes), an item a thread (a warp for mesh pairs). A small batch
            // then launches a handful of CTAs rather than a full device's worth that find no work.
            const size_t cap = f < kPairClasses ? totalCand : totalContacts;
            const size_t perCta = meshGrid(f) ? (size_t)std::min(threads / 32, kMeshWarps) : (size_t)threads;
            const size_t needed = std::max<size_t>(1, (cap + perCta - 1) / perCta);
            flatGrids[f] = (int)std::min<size_t>((size_t)smCount * (size_t)perSm, needed);
        }
        return TF_OK;
    }

    // Chooses how a kernel (or every kernel, k < 0) is launched; takes effect at the next step.
    int setLaunch(int k, uint32_t threads, uint32_t bigBodies, uint32_t smemBytes) {
        if (k >= kKernels || threads < 32 || threads > (uint32_t)kMaxBlock || threads % 32 != 0) {
            return fail(TF_E_INVALID, "launch shape: kernel index or thread count out of range");
        }
        if (threads > kMaxFlatBlock && (k < 0 || flatKernel(k))) {
            return fail(TF_E_INVALID, "launch shape: the refresh and collide kernels take at most 256 threads");
        }
        const bool flat = bigBodies == kFlatShape;
        if (flat && (k != 5 || threads > 256)) {
            return fail(TF_E_INVALID, "launch shape: the flat solve is a substep shape of at most 256 threads");
        }
        for (int i = 0; i < kKernels; ++i) {
            if (k >= 0 && i != k) { continue; }
            shapes[i] = LaunchShape{ threads, flat ? 0u : bigBodies, flat ? 0u : smemBytes, true, flat };
        }
        dropGraphs();
        if (laidOut) { return configureLaunches(); }
        return TF_OK;
    }

    int getLaunch(int k, uint32_t* out) const {
        if (k < 0 || k >= kKernels) { return TF_E_INVALID; }
        out[0] = shapes[k].threads;
        out[1] = shapes[k].flat ? kFlatShape : shapes[k].bigBodies;
        out[2] = splits[k].smemBytes;
        out[3] = (uint32_t)grids[k];
        out[4] = splits[k].big.bodies;
        out[5] = splits[k].small.bodies;
        return TF_OK;
    }

    // ---- Recording for the adjoint: what each step's solve saw (twofold_b200/csrc/tf_tape.h) ----

    struct TapeBuffers {
        DevArray<TapeWorld> worlds;
        DevArray<TapeContact> contacts;
        DevArray<uint32_t> colored, impactColored, rest, impactRest;
        DevArray<uint8_t> awake;
    };
    std::vector<std::unique_ptr<TapeBuffers>> tape;
    int tapeCursor = 0;     // the step being recorded
    bool recording = false;
    DevArray<TapeStep> dTapeSteps;
    DevArray<uint32_t> dTBodyFirst, dTBodyCount, dTShapeFirst;
    DevArray<uint8_t> dTDynamic;
    DevArray<float> dTGravityScale, dTLinDamp, dTAngDamp, dTMass, dTInvIL, dTCom0, dTQ0, dTV0, dTW0, dTFriction;
    AdjointSetup adjoint{};
    bool taped = false;
    void* adjRun = nullptr;

    // Launched after k_prepare while recording; sizes the step's buffers to the current layout first.
    int recordStep(const Batch& B, int serial) {
        if (tapeCursor >= (int)tape.size()) { return fail(TF_E_INVALID, "recording: more steps than the tape holds"); }
        TapeBuffers& T = *tape[(size_t)tapeCursor];
        const size_t ncon = dContacts[0].n;
        int rc;
        if ((rc = T.worlds.alloc(worlds.size())) != TF_OK || (rc = T.contacts.alloc(ncon)) != TF_OK ||
            (rc = T.colored.alloc(ncon)) != TF_OK || (rc = T.impactColored.alloc(ncon)) != TF_OK ||
            (rc = T.rest.alloc(ncon)) != TF_OK || (rc = T.impactRest.alloc(ncon)) != TF_OK ||
            (rc = T.awake.alloc(totalBodies)) != TF_OK) {
            return rc;
        }
        const TapeStep ts{ T.worlds.ptr, T.contacts.ptr, T.colored.ptr, T.impactColored.ptr, T.rest.ptr, T.impactRest.ptr,
                           T.awake.ptr };
        launch(kKTapeRecord, grids[3], shapes[3].threads, 0, B, splits[3], ts, serial);
        return TF_OK;
    }

    // Records n steps of dt from the current state (stepping the batch), for the adjoint to replay.
    int tapeRecord(float dt, int nSteps) {
        if (!(dt > 0.0f) || !std::isfinite(dt) || nSteps <= 0) { return fail(TF_E_INVALID, "tape: bad dt or steps"); }
        TF_CUDA(cudaSetDevice(device));
        int rc = prepareDevice();
        if (rc != TF_OK) { return rc; }
        if ((rc = pull()) != TF_OK) { return rc; }
        // Constants and the initial state, from the host mirrors.
        const size_t nw = worlds.size();
        std::vector<uint32_t> bodyFirst(nw), bodyCount(nw), shapeFirst(nw);
        std::vector<uint8_t> dyn(totalBodies);
        std::vector<float> gs(totalBodies), ld(totalBodies), ad(totalBodies), mass(totalBodies), invIL(9 * totalBodies);
        std::vector<float> com(3 * totalBodies), q(4 * totalBodies), v(3 * totalBodies), w(3 * totalBodies);
        std::vector<float> friction(totalShapes);
        for (size_t k = 0; k < nw; ++k) {
            const HostWorld& W = worlds[k];
            bodyFirst[k] = info[k].bodyFirst;
            bodyCount[k] = info[k].bodyCount;
            shapeFirst[k] = info[k].shapeFirst;
            for (size_t i = 0; i < W.bodies.size(); ++i) {
                const DBody& d = W.bodies[i].d;
                const size_t g = info[k].bodyFirst + i;
                if (d.alive && d.locks != 0) { return fail(TF_E_UNSUPPORTED, "tape: locked bodies are not differentiated"); }
                if (!W.joints.empty()) { return fail(TF_E_UNSUPPORTED, "tape: joints are not differentiated"); }
                dyn[g] = d.alive && d.type == kDynamic ? 1 : 0;
                gs[g] = d.gravityScale;
                ld[g] = d.linearDamping;
                ad[g] = d.angularDamping;
                mass[g] = d.mass;
                const Mat3 ii = dyn[g] ? inverse(d.inertia) : mzero();
                for (int r = 0; r < 3; ++r) {
                    invIL[9 * g + 3 * r] = ii.r[r].x, invIL[9 * g + 3 * r + 1] = ii.r[r].y, invIL[9 * g + 3 * r + 2] = ii.r[r].z;
                }
                com[3 * g] = d.com.x, com[3 * g + 1] = d.com.y, com[3 * g + 2] = d.com.z;
                q[4 * g] = d.xf.q.x, q[4 * g + 1] = d.xf.q.y, q[4 * g + 2] = d.xf.q.z, q[4 * g + 3] = d.xf.q.w;
                v[3 * g] = d.v.x, v[3 * g + 1] = d.v.y, v[3 * g + 2] = d.v.z;
                w[3 * g] = d.w.x, w[3 * g + 1] = d.w.y, w[3 * g + 2] = d.w.z;
            }
            for (size_t i = 0; i < W.shapes.size(); ++i) {
                const DShape& sd = W.shapes[i].d;
                if (sd.rollingResistance > 0.0f) { return fail(TF_E_UNSUPPORTED, "tape: rolling resistance is not differentiated"); }
                friction[info[k].shapeFirst + i] = sd.friction;
            }
        }
        auto up = [&](auto& arr, const auto& host) -> int {
            int r = arr.alloc(host.size());
            if (r != TF_OK) { return r; }
            TF_CUDA(cudaMemcpy(arr.ptr, host.data(), host.size() * sizeof(host[0]), cudaMemcpyHostToDevice));
            return TF_OK;
        };
        if ((rc = up(dTBodyFirst, bodyFirst)) || (rc = up(dTBodyCount, bodyCount)) || (rc = up(dTShapeFirst, shapeFirst)) ||
            (rc = up(dTDynamic, dyn)) || (rc = up(dTGravityScale, gs)) || (rc = up(dTLinDamp, ld)) ||
            (rc = up(dTAngDamp, ad)) || (rc = up(dTMass, mass)) || (rc = up(dTInvIL, invIL)) || (rc = up(dTCom0, com)) ||
            (rc = up(dTQ0, q)) || (rc = up(dTV0, v)) || (rc = up(dTW0, w)) || (rc = up(dTFriction, friction))) {
            return rc;
        }
        tape.clear();
        for (int k = 0; k < nSteps; ++k) { tape.emplace_back(new TapeBuffers()); }
        taped = false;
        recording = true;
        for (tapeCursor = 0; tapeCursor < nSteps && rc == TF_OK; ++tapeCursor) { rc = step(dt, 1); }
        recording = false;
        if (rc != TF_OK) { return rc; }
        std::vector<TapeStep> steps;
        size_t slots = 0;
        for (auto& T : tape) {
            steps.push_back(TapeStep{ T->worlds.ptr, T->contacts.ptr, T->colored.ptr, T->impactColored.ptr, T->rest.ptr,
                                      T->impactRest.ptr, T->awake.ptr });
            slots = std::max(slots, T->contacts.n);
        }
        if ((rc = up(dTapeSteps, steps)) != TF_OK) { return rc; }
        const StepParams P = params(dt);
        AdjointSetup& A = adjoint;
        A.nWorlds = (int)nw;
        A.nSteps = nSteps;
        A.totalBodies = (uint32_t)totalBodies;
        A.totalShapes = (uint32_t)totalShapes;
        A.contactSlots = (uint32_t)slots;
        A.bodyFirst = dTBodyFirst.ptr;
        A.bodyCount = dTBodyCount.ptr;
        A.shapeFirst = dTShapeFirst.ptr;
        A.steps = dTapeSteps.ptr;
        A.dynamic = dTDynamic.ptr;
        A.gravityScale = dTGravityScale.ptr;
        A.linearDamping = dTLinDamp.ptr;
        A.angularDamping = dTAngDamp.ptr;
        A.mass = dTMass.ptr;
        A.invInertiaLocal = dTInvIL.ptr;
        A.com0 = dTCom0.ptr;
        A.q0 = dTQ0.ptr;
        A.v0 = dTV0.ptr;
        A.w0 = dTW0.ptr;
        A.friction = dTFriction.ptr;
        A.gravity[0] = P.gravity.x, A.gravity[1] = P.gravity.y, A.gravity[2] = P.gravity.z;
        A.dt = dt;
        A.substeps = P.substeps;
        A.contactSoft[0] = P.contactSoft.biasRate, A.contactSoft[1] = P.contactSoft.massScale,
        A.contactSoft[2] = P.contactSoft.impulseScale;
        A.staticSoft[0] = P.staticSoft.biasRate, A.staticSoft[1] = P.staticSoft.massScale,
        A.staticSoft[2] = P.staticSoft.impulseScale;
        A.maxPushout = P.maxPushout;
        A.restitutionThreshold = P.restitutionThreshold;
        taped = true;
        return TF_OK;
    }

    template <class T>
    int copyArray(DevArray<T>& to, const DevArray<T>& from) {
        int rc = to.alloc(from.n);
        if (rc != TF_OK) { return rc; }
        TF_CUDA(cudaMemcpyAsync(to.ptr, from.ptr, from.n * sizeof(T), cudaMemcpyDeviceToDevice, stream));
        return TF_OK;
    }

    // Copies the dynamic device state into snapshot `slot` (stream-ordered; nothing waits).
    int saveState(int slot) {
        TF_CUDA(cudaSetDevice(device));
        int rc = prepareDevice();
        if (rc != TF_OK) { return rc; }
        std::unique_ptr<Snapshot>& sp = snapshots[slot];
        if (!sp) { sp.reset(new Snapshot()); }
        Snapshot& S = *sp;
        if ((rc = copyArray(S.bodies, dBodies)) != TF_OK) { return rc; }
        if ((rc = copyArray(S.shapes, dShapes)) != TF_OK) { return rc; }
        if ((rc = copyArray(S.contacts, dContacts[cur])) != TF_OK) { return rc; }
        if ((rc = copyArray(S.counts, dCounts)) != TF_OK) { return rc; }
        if ((rc = copyArray(S.struck, dStruck)) != TF_OK) { return rc; }
        if ((rc = copyArray(S.wakeMark, dWakeMark)) != TF_OK) { return rc; }
        if ((rc = copyArray(S.joints, dJoints)) != TF_OK) { return rc; }
        S.cur = cur;
        S.layoutGen = layoutGen;
        S.bodyStepsTotal = bodyStepsTotal;
        S.bodyStepsBase = bodyStepsBase;
        return TF_OK;
    }

    // Puts snapshot `slot` back. Refused when the batch was laid out again since (a list grew, or a body or
    // shape was added): the snapshot's arrays no longer match the device's.
    int restoreState(int slot) {
        TF_CUDA(cudaSetDevice(device));
        auto it = snapshots.find(slot);
        if (it == snapshots.end()) { return fail(TF_E_INVALID, "restore: no snapshot in that slot"); }
        Snapshot& S = *it->second;
        if (S.layoutGen != layoutGen || layoutDirty) {
            return fail(TF_E_INVALID, "restore: the batch was laid out again since the snapshot was taken");
        }
        cur = S.cur;
        int rc;
        if ((rc = copyArray(dBodies, S.bodies)) != TF_OK) { return rc; }
        if ((rc = copyArray(dShapes, S.shapes)) != TF_OK) { return rc; }
        if ((rc = copyArray(dContacts[cur], S.contacts)) != TF_OK) { return rc; }
        if ((rc = copyArray(dCounts, S.counts)) != TF_OK) { return rc; }
        if ((rc = copyArray(dStruck, S.struck)) != TF_OK) { return rc; }
        if ((rc = copyArray(dWakeMark, S.wakeMark)) != TF_OK) { return rc; }
        if ((rc = copyArray(dJoints, S.joints)) != TF_OK) { return rc; }
        bodyStepsTotal = S.bodyStepsTotal;
        bodyStepsBase = S.bodyStepsBase;
        hostFresh = false;
        onDevice = true;
        bodiesDirty = false;
        eventsValid = false;  // the event rooms hold the last step run, not the restored one's
        return TF_OK;
    }

    // The contact events and hits of world w's last step, in the reference's order: by shape pair, and for
    // one pair the narrowphase's before the end-of-step report's (src/world.cpp:1694-1700).
    bool eventsValid = false;
    int events(size_t w, std::vector<TouchEvent>* touch, std::vector<HitRecord>* hits) {
        if (touch) { touch->clear(); }
        if (hits) { hits->clear(); }
        if (!eventsValid) { return TF_OK; }
        int rc = refreshCounts();
        if (rc != TF_OK) { return rc; }
        if (w >= lastCounts.size() || w >= info.size()) { return TF_OK; }
        TF_CUDA(cudaSetDevice(device));
        TF_CUDA(cudaStreamSynchronize(stream));
        const WorldInfo& wi = info[w];
        if (touch && lastCounts[w].touchEvents > 0) {
            touch->resize(std::min<size_t>(lastCounts[w].touchEvents, 2 * (size_t)wi.contactCap));
            TF_CUDA(cudaMemcpy(touch->data(), dTouchEvents.ptr + 2 * (size_t)wi.contactFirst,
                               touch->size() * sizeof(TouchEvent), cudaMemcpyDeviceToHost));
            std::sort(touch->begin(), touch->end(), [](const TouchEvent& a, const TouchEvent& b) {
                return a.key != b.key ? a.key < b.key : a.late < b.late;
            });
        }
        if (hits && lastCounts[w].hitEvents > 0) {
            hits->resize(std::min<size_t>(lastCounts[w].hitEvents, (size_t)wi.contactCap));
            TF_CUDA(cudaMemcpy(hits->data(), dHitEvents.ptr + wi.contactFirst, hits->size() * sizeof(HitRecord),
                               cudaMemcpyDeviceToHost));
            std::sort(hits->begin(), hits->end(), [](const HitRecord& a, const HitRecord& b) { return a.key < b.key; });
        }
        return TF_OK;
    }

    // Times candidate launch shapes on the batch's current state and keeps the fastest per kernel. Every
    // candidate gives the same results (the pipeline's output does not depend on launch shapes), so each
    // trial runs every kernel with its own next candidate and reads all kernel times at once. The state is
    // put back after every trial and at the end. out (8 x 3: threads, big-world threshold, shared bytes per
    // kernel) receives the choice when non-null.
    int autotune(float dt, int trialSteps, uint32_t* out) {
        if (!(dt > 0.0f) || !std::isfinite(dt) || trialSteps <= 0) { return fail(TF_E_INVALID, "autotune: bad dt or steps"); }
        TF_CUDA(cudaSetDevice(device));
        int rc = prepareDevice();
        if (rc != TF_OK) { return rc; }
        if ((rc = pull()) != TF_OK) { return rc; }
        const std::vector<HostWorld> saved = worlds;  // for a trial that grows a list and lays out again
        const int64_t savedTotal = bodyStepsTotal, savedBase = bodyStepsBase;
        const int kSlot = -1;
        if ((rc = saveState(kSlot)) != TF_OK) { return rc; }
        std::vector<LaunchShape> cands[kKernels];
        for (int k = 0; k < kKernels; ++k) {
            if (flatKernel(k)) {
                for (uint32_t t : { 64u, 128u, 256u }) { cands[k].push_back(LaunchShape{ t, 0u, 0u, true }); }
                continue;
            }
            const bool stages = k == 0 || k == 3 || k == 5 || k == 6;
            if (k == 5) {
                for (uint32_t t : { 128u, 256u }) { cands[k].push_back(LaunchShape{ t, 0u, 0u, true, true }); }
            }
            for (uint32_t t : { 128u, 256u, 512u }) {
                for (uint32_t big : { 0u, 32u, 64u, 128u, 256u }) {
                    if (stages) {
                        for (uint32_t sm : { 32u * 1024u, 48u * 1024u, 96u * 1024u }) {
                            cands[k].push_back(LaunchShape{ t, big, sm, true });
                        }
                    } else {
                        cands[k].push_back(LaunchShape{ t, big, 0u, true });
                    }
                }
            }
        }
        size_t trials = 0;
        for (auto& c : cands) { trials = std::max(trials, c.size()); }
        double best[kKernels];
        LaunchShape chosen[kKernels];
        for (int k = 0; k < kKernels; ++k) {
            best[k] = 1e300;
            chosen[k] = shapes[k];
        }
        const bool wasProfiling = profiling;
        profiling = true;
        for (size_t t = 0; t < trials && rc == TF_OK; ++t) {
            for (int k = 0; k < kKernels; ++k) { shapes[k] = cands[k][t % cands[k].size()]; }
            dropGraphs();
            if ((rc = configureLaunches()) != TF_OK) { break; }
            if (restoreState(kSlot) != TF_OK) {
                // A trial grew a list: lay the saved state out again and take the snapshot anew.
                worlds = saved;
                hostFresh = true;
                layoutDirty = true;
                if ((rc = prepareDevice()) != TF_OK || (rc = saveState(kSlot)) != TF_OK) { break; }
            }
            if ((rc = step(dt, 1)) != TF_OK) { break; }
            for (int k = 0; k < kKernelKinds; ++k) {
                kernelMs[k] = 0.0;
                kernelLaunches[k] = 0;
            }
            if ((rc = step(dt, trialSteps)) != TF_OK) { break; }
            for (int k = 0; k < kKernels; ++k) {
                if (t < cands[k].size() && kernelMs[k] < best[k]) {
                    best[k] = kernelMs[k];
                    chosen[k] = shapes[k];
                }
            }
        }
        profiling = wasProfiling;
        for (int k = 0; k < kKernels; ++k) { shapes[k] = chosen[k]; }
        dropGraphs();
        const int rcShape = configureLaunches();
        if (restoreState(kSlot) != TF_OK) {
            worlds = saved;
            hostFresh = true;
            layoutDirty = true;
        }
        bodyStepsTotal = savedTotal;
        bodyStepsBase = savedBase;
        snapshots.erase(kSlot);
        if (rc != TF_OK) { return rc; }
        if (rcShape != TF_OK) { return rcShape; }
        if (out) {
            for (int k = 0; k < kKernels; ++k) {
                out[3 * k] = shapes[k].threads;
                out[3 * k + 1] = shapes[k].flat ? kFlatShape : shapes[k].bigBodies;
                out[3 * k + 2] = shapes[k].smemBytes;
            }
        }
        return TF_OK;
    }

    // Reads how many of the steps just issued completed: all of them, or those before the first one that
    // overflowed a list (it and every later step did nothing).
    int completedSteps(int issued, int* completed) {
        uint32_t abort = 0;
        TF_CUDA(cudaMemcpy(&abort, dAbort.ptr, sizeof(abort), cudaMemcpyDeviceToHost));
        *completed = abort == 0xffffffffu ? issued : (int)abort;
        return TF_OK;
    }

    // Grows the lists of the worlds that overflowed and lays the batch out again from the device state
    // the completed steps left.
    int growAfterAbort() {
        if (std::getenv("TWOFOLD_B200_TRACE")) { std::fprintf(stderr, "twofold_b200: list overflow, growing and laying out again\n"); }
        hostFresh = false;
        onDevice = true;
        int rc = pull();
        if (rc != TF_OK) { return rc; }
        return layout();
    }

    // The events that calls since the last step queued belong to the next step; after a call of several steps
    // the last one's events are read, which had none.
    void takeQueuedEvents(int nSteps) {
        for (HostWorld& W : worlds) {
            W.stepQueued.clear();
            if (nSteps == 1) { W.stepQueued.swap(W.queued); }
            W.queued.clear();
        }
    }

    int step(float dt, int nSteps) {
        if (!(dt > 0.0f) || !std::isfinite(dt) || nSteps <= 0) { return TF_OK; }
        TF_CUDA(cudaSetDevice(device));
        int rc = prepareDevice();
        if (rc != TF_OK) { return rc; }
        rc = configureKernels();
        if (rc != TF_OK) { return rc; }
        cudaEvent_t marks[4];
        for (cudaEvent_t& e : marks) { TF_CUDA(cudaEventCreate(&e)); }
        int done = 0;
        TF_CUDA(cudaEventRecord(callStart, stream));
        for (int attempt = 0; done < nSteps && attempt < 8; ++attempt) {
            TF_CUDA(cudaMemsetAsync(dAbort.ptr, 0xff, sizeof(uint32_t), stream));
            const int start = cur;
            const int issue = nSteps - done;
            int c = cur;
            for (int s = 0; s < issue && rc == TF_OK; ++s) {
                rc = enqueueStep(dt, 1 - c, s, s == issue - 1 ? marks : nullptr);
                c = 1 - c;
            }
            cudaEventRecord(callStop, stream);
            cudaError_t e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) { rc = fail(TF_E_CUDA, std::string("step: ") + cudaGetErrorString(e)); }
            if (rc != TF_OK) { break; }
            cudaEventElapsedTime(&lastElapsedMs, callStart, callStop);
            collectKernelTimes();
            int completed = 0;
            if ((rc = completedSteps(issue, &completed)) != TF_OK) { break; }
            cur = (completed % 2) ? 1 - start : start;
            done += completed;
            hostFresh = false;
            if (completed == issue) {
                float bp = 0, np = 0, sv = 0;
                cudaEventElapsedTime(&bp, marks[0], marks[1]);
                cudaEventElapsedTime(&np, marks[1], marks[2]);
                cudaEventElapsedTime(&sv, marks[2], marks[3]);
                for (tf_profile& p : profiles) {
                    p.broadphase = bp;
                    p.narrowphase = np;
                    p.solver = sv;
                    p.total = bp + np + sv;
                }
                break;
            }
            if ((rc = growAfterAbort()) != TF_OK) { break; }
        }
        for (cudaEvent_t& ev : marks) { cudaEventDestroy(ev); }
        if (rc != TF_OK) { return rc; }
        if (done < nSteps) { return fail(TF_E_CAPACITY, "device lists kept overflowing"); }
        return checkFlags();
    }

    // Records n steps into a CUDA graph on first use (the contact buffers alternate, so n even keeps the
    // same buffer at the end), then replays it.
    int stepGraph(float dt, int nSteps) {
        if (!(dt > 0.0f) || !std::isfinite(dt) || nSteps <= 0) { return TF_OK; }
        TF_CUDA(cudaSetDevice(device));
        int rc = prepareDevice();
        if (rc != TF_OK) { return rc; }
        rc = configureKernels();
        if (rc != TF_OK) { return rc; }
        if (graphSteps != nSteps || graphDt != dt || graphProfiled != profiling) { dropGraphs(); }
        cudaGraphExec_t& graphExec = graphs[cur];
        const int startBuffer = cur;
        if (!graphExec) {
            cudaGraph_t graph;
            if (profiling) {
                // One event pair per kernel group of every step: 6 groups and 2 per substep cover them all.
                const size_t pairs = (size_t)nSteps * (6 + 2 * (size_t)std::max(1, (int)settings.substeps));
                for (size_t k = graphTimers[cur].size(); k < pairs; ++k) {
                    KernelTimer t{ 0, nullptr, nullptr };
                    TF_CUDA(cudaEventCreate(&t.start));
                    TF_CUDA(cudaEventCreate(&t.stop));
                    graphTimers[cur].push_back(t);
                }
            }
            TF_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            captureTimers = profiling ? &graphTimers[cur] : nullptr;
            captureUsed = 0;
            int c = cur;
            for (int s = 0; s < nSteps; ++s) {
                const int into = 1 - c;
                rc = enqueueStep(dt, into, s, nullptr, true);
                if (rc != TF_OK) { break; }
                c = into;
            }
            captureTimers = nullptr;
            graphTimersUsed[cur] = captureUsed;
            cudaError_t e = cudaStreamEndCapture(stream, &graph);
            if (rc != TF_OK) { return rc; }
            if (e != cudaSuccess) { return fail(TF_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e)); }
            e = cudaGraphInstantiate(&graphExec, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) { return fail(TF_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)); }
            graphSteps = nSteps;
            graphDt = dt;
            graphProfiled = profiling;
        }
        TF_CUDA(cudaMemsetAsync(dAbort.ptr, 0xff, sizeof(uint32_t), stream));
        TF_CUDA(cudaEventRecord(callStart, stream));
        TF_CUDA(cudaGraphLaunch(graphExec, stream));
        TF_CUDA(cudaEventRecord(callStop, stream));
        launches += (int64_t)nSteps * (4 + 2 * std::max(1, (int)settings.substeps));
        TF_CUDA(cudaStreamSynchronize(stream));
        TF_CUDA(cudaEventElapsedTime(&lastElapsedMs, callStart, callStop));
        if (graphProfiled) {
            for (size_t k = 0; k < graphTimersUsed[startBuffer]; ++k) {
                const KernelTimer& t = graphTimers[startBuffer][k];
                float ms = 0.0f;
                if (cudaEventElapsedTime(&ms, t.start, t.stop) == cudaSuccess) {
                    kernelMs[t.kind] += ms;
                    kernelLaunches[t.kind] += 1;
                }
            }
        }
        int completed = 0;
        if ((rc = completedSteps(nSteps, &completed)) != TF_OK) { return rc; }
        const int start = cur;
        cur = (completed % 2) ? 1 - start : start;
        hostFresh = false;
        if (completed < nSteps) {
            // A list overflowed: grow it and finish the remaining steps with direct launches. The call's device
            // time is the aborted graph launch's plus the retry's.
            const float graphMs = lastElapsedMs;
            if ((rc = growAfterAbort()) != TF_OK) { return rc; }
            rc = step(dt, nSteps - completed);
            lastElapsedMs += graphMs;
            return rc;
        }
        return checkFlags();
    }

    int checkFlags() {
#if defined(TF_DEVICE_CHECKS)
        uint32_t dbg[4] = { 0, 0, 0, 0 };
        TF_CUDA(cudaMemcpy(dbg, dDebug.ptr, sizeof(dbg), cudaMemcpyDeviceToHost));
        if (dbg[0] != 0) {
            char msg[160];
            snprintf(msg, sizeof(msg), "device index check %u failed (world/base %u, value %u)", dbg[0], dbg[1], dbg[2]);
            return fail(TF_E_INVALID, msg);
        }
#endif
        // Every step: the worlds' flags and body steps, summed on the device (16 bytes back). The worlds' own
        // counts come back only when something asks for them (refreshCounts).
        int rc = dSummary.alloc(4);
        if (rc != TF_OK) { return rc; }
        if (!hostSummary) { TF_CUDA(cudaMallocHost(&hostSummary, 4 * sizeof(uint32_t))); }
        launch(kKStepSummary, 1u, 256u, 0, (const WorldCounts*)dCounts.ptr, (uint32_t)worlds.size(), dSummary.ptr);
        ++launches;
        TF_CUDA(cudaGetLastError());
        TF_CUDA(cudaMemcpyAsync(hostSummary, dSummary.ptr, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        TF_CUDA(cudaStreamSynchronize(stream));
        const uint32_t flags = hostSummary[0];
        const int64_t bodySteps = (int64_t)((uint64_t)hostSummary[1] | (uint64_t)hostSummary[2] << 32);
        countsStale = true;
        eventsValid = true;
        deviceFlags = flags;
        bodyStepsTotal = bodyStepsBase + bodySteps;
        if (flags & kDevUnsupported) { return fail(TF_E_UNSUPPORTED, "the step met a pair this build cannot collide"); }
        if (flags & kDevNonFinite) { return fail(TF_E_NUMERIC, "a body state became non-finite"); }
        if (flags & kDevTimeout) { return fail(TF_E_TIMEOUT, "a bounded device wait gave up"); }
        return TF_OK;
    }

    // Every world's counts of the last step (lastCounts) and the step profiles' counts, read back on demand.
    int refreshCounts() {
        if (!countsStale) { return TF_OK; }
        TF_CUDA(cudaSetDevice(device));
        TF_CUDA(cudaStreamSynchronize(stream));
        std::vector<WorldCounts> counts(worlds.size());
        TF_CUDA(cudaMemcpy(counts.data(), dCounts.ptr, worlds.size() * sizeof(WorldCounts), cudaMemcpyDeviceToHost));
        for (size_t w = 0; w < worlds.size(); ++w) {
            tf_profile& p = profiles[w];
            p.candidate_pairs = (int32_t)counts[w].candCount;
            p.manifolds = (int32_t)counts[w].contactCount;
            p.awake_bodies = (int32_t)counts[w].awakeBodies;
            p.awake_islands = (int32_t)counts[w].awakeIslands;
            p.swept_pairs = (int32_t)counts[w].sweptPairs;
            p.impacts = (int32_t)counts[w].impacts;
            p.touching_contacts = (int32_t)counts[w].touching;
        }
        lastCounts = counts;
        countsStale = false;
        return TF_OK;
    }
    std::vector<WorldCounts> lastCounts;
    bool countsStale = false;
    DevArray<uint32_t> dSummary;
    uint32_t* hostSummary = nullptr;  // pinned
    uint32_t deviceFlags = 0;
    int64_t bodyStepsBase = 0;  // body steps of layouts before the current one

    int addForces(const float* f, const float* t) {
        int rc = ensureDevice();
        if (rc != TF_OK) { return rc; }
        if ((rc = prepareDevice()) != TF_OK) { return rc; }
        const size_t n = totalBodies;
        if ((rc = dHostIn.alloc(6 * n)) != TF_OK) { return rc; }
        if (f) { TF_CUDA(cudaMemcpyAsync(dHostIn.ptr, f, 3 * n * sizeof(float), cudaMemcpyHostToDevice, stream)); }
        if (t) { TF_CUDA(cudaMemcpyAsync(dHostIn.ptr + 3 * n, t, 3 * n * sizeof(float), cudaMemcpyHostToDevice, stream)); }
        launch(kKAddForces, (unsigned)((n + 255) / 256), 256, 0, dBodies.ptr, (uint32_t)n,
               (const float*)(f ? dHostIn.ptr : nullptr), (const float*)(t ? dHostIn.ptr + 3 * n : nullptr));
        ++launches;
        TF_CUDA(cudaGetLastError());
        hostFresh = false;
        return TF_OK;
    }

    int readPoses(float* p, float* q) {
        if (!onDevice || layoutDirty) {
            // Nothing stepped yet: the host mirrors are current.
            size_t k = 0;
            for (const auto& W : worlds) {
                for (const auto& hb : W.bodies) {
                    if (p) { p[3 * k] = hb.d.xf.p.x, p[3 * k + 1] = hb.d.xf.p.y, p[3 * k + 2] = hb.d.xf.p.z; }
                    if (q) { q[4 * k] = hb.d.xf.q.x, q[4 * k + 1] = hb.d.xf.q.y, q[4 * k + 2] = hb.d.xf.q.z, q[4 * k + 3] = hb.d.xf.q.w; }
                    ++k;
                }
            }
            return TF_OK;
        }
        const size_t n = totalBodies;
        int rc = dHostOut.alloc(7 * n);
        if (rc != TF_OK) { return rc; }
        launch(kKPackPoses, (unsigned)((n + 255) / 256), 256, 0, (const DBody*)dBodies.ptr, (uint32_t)n, dHostOut.ptr,
               dHostOut.ptr + 3 * n);
        ++launches;
        TF_CUDA(cudaGetLastError());
        if (p) { TF_CUDA(cudaMemcpyAsync(p, dHostOut.ptr, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, stream)); }
        if (q) { TF_CUDA(cudaMemcpyAsync(q, dHostOut.ptr + 3 * n, 4 * n * sizeof(float), cudaMemcpyDeviceToHost, stream)); }
        TF_CUDA(cudaStreamSynchronize(stream));
        return TF_OK;
    }

    // readPoses queued: the pack on the world's stream into a staging buffer, the copy on the copy stream after
    // it, so the copy runs beside the world's next launches. A staging buffer is packed again only after its
    // last copy has read it (a wait on the device, not the host).
    int readPosesAsync(float* p, float* q) {
        if (!onDevice || layoutDirty) { return readPoses(p, q); }
        const size_t n = totalBodies;
        if (!copyStream) {
            TF_CUDA(cudaStreamCreateWithFlags(&copyStream, cudaStreamNonBlocking));
            for (cudaEvent_t* e : { &posePacked[0], &posePacked[1], &poseCopied[0], &poseCopied[1] }) {
                TF_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
            }
        }
        const int slot = poseSlot;
        poseSlot ^= 1;
        DevArray<float>& buf = dPoseStage[slot];
        if (!buf.ptr || buf.n < 7 * n) {
            int rc = posesWait();
            if (rc == TF_OK) { rc = buf.alloc(7 * n); }
            if (rc != TF_OK) { return rc; }
        }
        if (poseCopyPending[slot]) { TF_CUDA(cudaStreamWaitEvent(stream, poseCopied[slot], 0)); }
        launch(kKPackPoses, (unsigned)((n + 255) / 256), 256, 0, (const DBody*)dBodies.ptr, (uint32_t)n, buf.ptr,
               buf.ptr + 3 * n);
        ++launches;
        TF_CUDA(cudaGetLastError());
        TF_CUDA(cudaEventRecord(posePacked[slot], stream));
        TF_CUDA(cudaStreamWaitEvent(copyStream, posePacked[slot], 0));
        if (p) { TF_CUDA(cudaMemcpyAsync(p, buf.ptr, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, copyStream)); }
        if (q) { TF_CUDA(cudaMemcpyAsync(q, buf.ptr + 3 * n, 4 * n * sizeof(float), cudaMemcpyDeviceToHost, copyStream)); }
        TF_CUDA(cudaEventRecord(poseCopied[slot], copyStream));
        poseCopyPending[slot] = true;
        return TF_OK;
    }

    int posesWait() {
        for (int k = 0; k < 2; ++k) {
            if (!poseCopyPending[k]) { continue; }
            TF_CUDA(cudaEventSynchronize(poseCopied[k]));
            poseCopyPending[k] = false;
        }
        return TF_OK;
    }
};

}  // namespace tfb

using tfb::Engine;

namespace {
Engine* E(void* h) { return static_cast<Engine*>(h); }
}

extern "C" {

TF_API int tf_abi_version(void) { return TF_ABI_VERSION; }

TF_API const char* tf_last_error(void) { return tfb::g_error.c_str(); }

TF_API void tf_default_settings(tf_settings* s) {
    if (!s) { return; }
    *s = tf_settings{};
    s->gravity[0] = 0.0f;
    s->gravity[1] = -9.81f;
    s->gravity[2] = 0.0f;
    s->length_unit = 1.0f;
    s->substeps = 4;
    s->contact_hertz = 30.0f;
    s->contact_damping_ratio = 10.0f;
    s->max_pushout_speed = 3.0f;
    s->max_linear_speed = 1000.0f;
    s->max_angular_speed = 1000.0f;
    s->restitution_threshold = 1.0f;
    s->hit_threshold = 1.0f;
    s->sleep_threshold = 0.05f;
    s->time_to_sleep = 0.5f;
    s->contact_reuse_distance = 0.0005f;
    s->contact_reuse_angle = 0.035f;
    s->joint_hertz = 60.0f;
    s->joint_damping_ratio = 2.0f;
    s->continuous = 1;
}

TF_API int tf_world_create(const tf_settings* settings, int32_t n_worlds, int32_t device, void** out) {
    if (!out || n_worlds <= 0) { return tfb::fail(TF_E_INVALID, "tf_world_create: bad arguments"); }
    *out = nullptr;
    tf_settings s;
    if (settings) {
        s = *settings;
    } else {
        tf_default_settings(&s);
    }
    std::unique_ptr<Engine> e(new Engine());
    const int rc = e->init(&s, n_worlds, device);
    if (rc != TF_OK) { return rc; }
    *out = e.release();
    return TF_OK;
}

TF_API int tf_world_destroy(void* h) {
    delete E(h);
    return TF_OK;
}

TF_API int tf_world_count(void* h, int32_t* n) {
    if (!h || !n) { return tfb::fail(TF_E_INVALID, "tf_world_count: null"); }
    *n = (int32_t)E(h)->worlds.size();
    return TF_OK;
}

TF_API int tf_world_set_settings(void* h, const tf_settings* s) {
    if (!h || !s) { return tfb::fail(TF_E_INVALID, "tf_world_set_settings: null"); }
    E(h)->settings = *s;
    return TF_OK;
}

TF_API int tf_mesh_create(void* h, const float* vertices, int32_t vertex_count, const uint32_t* indices,
                          int32_t index_count, int32_t* out_mesh) {
    if (!h || !out_mesh) { return tfb::fail(TF_E_INVALID, "tf_mesh_create: null"); }
    if (vertex_count < 0 || index_count < 0 || (vertex_count > 0 && !vertices) || (index_count > 0 && !indices)) {
        return tfb::fail(TF_E_INVALID, "tf_mesh_create: bad arrays");
    }
    std::vector<tfb::Vec3> v((size_t)vertex_count);
    for (int32_t i = 0; i < vertex_count; ++i) { v[(size_t)i] = { vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2] }; }
    std::vector<uint32_t> idx(indices, indices + index_count);
    Engine* e = E(h);
    *out_mesh = (int32_t)e->meshes.size();
    e->meshes.push_back(tfb::buildMesh(v, idx));
    e->layoutDirty = true;
    return TF_OK;
}

TF_API int tf_mesh_read(void* h, int32_t mesh, int32_t counts[3], float* vertices, uint32_t* indices, float* normals,
                        uint8_t* edges, float* node_bounds, int32_t* node_ranges) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_mesh_read: null world"); }
    Engine* e = E(h);
    if (mesh < 0 || (size_t)mesh >= e->meshes.size()) { return tfb::fail(TF_E_INVALID, "tf_mesh_read: unknown mesh"); }
    const tfb::HostMesh& m = e->meshes[(size_t)mesh];
    if (counts) {
        counts[0] = (int32_t)m.vertices.size();
        counts[1] = (int32_t)m.normals.size();
        counts[2] = (int32_t)m.nodes.size();
    }
    for (size_t i = 0; i < m.vertices.size(); ++i) {
        if (vertices) { vertices[3 * i] = m.vertices[i].x, vertices[3 * i + 1] = m.vertices[i].y, vertices[3 * i + 2] = m.vertices[i].z; }
    }
    if (indices) { std::copy(m.indices.begin(), m.indices.end(), indices); }
    for (size_t t = 0; t < m.normals.size(); ++t) {
        if (normals) { normals[3 * t] = m.normals[t].x, normals[3 * t + 1] = m.normals[t].y, normals[3 * t + 2] = m.normals[t].z; }
        if (edges) { edges[t] = m.edges[t]; }
    }
    for (size_t n = 0; n < m.nodes.size(); ++n) {
        const tfb::MeshNode& x = m.nodes[n];
        if (node_bounds) {
            const float b[6] = { x.lo.x, x.lo.y, x.lo.z, x.hi.x, x.hi.y, x.hi.z };
            std::copy(b, b + 6, node_bounds + 6 * n);
        }
        if (node_ranges) {
            node_ranges[2 * n] = x.first;
            node_ranges[2 * n + 1] = x.count;
        }
    }
    return TF_OK;
}

TF_API int tf_hull_compute(const float* points, int32_t count, int32_t max_vertices, int32_t counts[2], float* vertices,
                           int32_t vertex_capacity, int32_t* faces, int32_t face_capacity) {
    if (count < 0 || !counts || (count > 0 && !points)) { return tfb::fail(TF_E_INVALID, "tf_hull_compute: bad arguments"); }
    std::vector<tfb::Vec3> cloud((size_t)count);
    for (int32_t i = 0; i < count; ++i) { cloud[i] = { points[3 * i], points[3 * i + 1], points[3 * i + 2] }; }
    const tfb::HullResult h = tfb::computeHull(cloud, max_vertices);
    int32_t words = 0;
    for (const auto& f : h.faces) { words += 1 + (int32_t)f.size(); }
    counts[0] = (int32_t)h.vertices.size();
    counts[1] = words;
    if (vertices && vertex_capacity >= counts[0]) {
        for (size_t i = 0; i < h.vertices.size(); ++i) {
            vertices[3 * i] = h.vertices[i].x, vertices[3 * i + 1] = h.vertices[i].y, vertices[3 * i + 2] = h.vertices[i].z;
        }
    }
    if (faces && face_capacity >= words) {
        int32_t at = 0;
        for (const auto& f : h.faces) {
            faces[at++] = (int32_t)f.size();
            for (int v : f) { faces[at++] = v; }
        }
    }
    return TF_OK;
}

TF_API int tf_body_create(void* h, int32_t w, const tf_body_desc* d, tf_id* out) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_body_create: null world"); }
    return E(h)->createBody(w, d, out);
}

TF_API int tf_shape_add(void* h, int32_t w, tf_id body, const tf_shape_desc* d, tf_id* out) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_shape_add: null world"); }
    return E(h)->addShape(w, body, d, out);
}

TF_API int tf_bodies_create(void* h, int32_t n, const int32_t* world_of, const tf_body_desc* descs, tf_id* out) {
    if (!h || (n > 0 && (!world_of || !descs))) { return tfb::fail(TF_E_INVALID, "tf_bodies_create: null"); }
    for (int32_t i = 0; i < n; ++i) {
        const int rc = E(h)->createBody(world_of[i], &descs[i], out ? &out[i] : nullptr);
        if (rc != TF_OK) { return rc; }
    }
    return TF_OK;
}

TF_API int tf_shapes_add(void* h, int32_t n, const int32_t* world_of, const uint32_t* body_of,
                         const tf_shape_desc* descs, tf_id* out) {
    if (!h || (n > 0 && (!world_of || !body_of || !descs))) { return tfb::fail(TF_E_INVALID, "tf_shapes_add: null"); }
    Engine* e = E(h);
    for (int32_t i = 0; i < n; ++i) {
        const int w = world_of[i];
        if (w < 0 || w >= (int)e->worlds.size() || body_of[i] >= e->worlds[(size_t)w].bodies.size()) {
            return tfb::fail(TF_E_INVALID, "tf_shapes_add: bad body");
        }
        const tf_id body{ body_of[i], e->worlds[(size_t)w].bodies[body_of[i]].generation };
        const int rc = e->addShape(w, body, &descs[i], out ? &out[i] : nullptr);
        if (rc != TF_OK) { return rc; }
    }
    return TF_OK;
}

TF_API int tf_world_step(void* h, float dt, int32_t n) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_step: null world"); }
    if (dt > 0.0f && std::isfinite(dt) && n > 0) { E(h)->takeQueuedEvents(n); }
    return E(h)->step(dt, n);
}

TF_API int tf_world_step_graph(void* h, float dt, int32_t n) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_step_graph: null world"); }
    if (dt > 0.0f && std::isfinite(dt) && n > 0) { E(h)->takeQueuedEvents(n); }
    return E(h)->stepGraph(dt, n);
}

TF_API int tf_world_synchronize(void* h) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_synchronize: null world"); }
    if (!E(h)->stream) { return TF_OK; }
    cudaError_t e = cudaStreamSynchronize(E(h)->stream);
    return e == cudaSuccess ? TF_OK : tfb::fail(TF_E_CUDA, cudaGetErrorString(e));
}

TF_API int tf_world_device_status(void* h, uint32_t* flags) {
    if (!h || !flags) { return tfb::fail(TF_E_INVALID, "tf_world_device_status: null"); }
    *flags = E(h)->deviceFlags;
    return TF_OK;
}

TF_API int tf_body_get_state(void* h, int32_t w, tf_id id, float p[3], float q[4], float v[3], float av[3]) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_body_get_state: null world"); }
    Engine* e = E(h);
    const int rc = e->pull();
    if (rc != TF_OK) { return rc; }
    tfb::HostBody* b = e->body(w, id);
    const tfb::DBody zero{};
    const tfb::DBody& d = b ? b->d : zero;
    if (p) { p[0] = d.xf.p.x, p[1] = d.xf.p.y, p[2] = d.xf.p.z; }
    if (q) { q[0] = b ? d.xf.q.x : 0.0f, q[1] = b ? d.xf.q.y : 0.0f, q[2] = b ? d.xf.q.z : 0.0f, q[3] = b ? d.xf.q.w : 1.0f; }
    if (v) { v[0] = d.v.x, v[1] = d.v.y, v[2] = d.v.z; }
    if (av) { av[0] = d.w.x, av[1] = d.w.y, av[2] = d.w.z; }
    return TF_OK;
}

TF_API int tf_body_set_velocity(void* h, int32_t w, tf_id id, const float v[3], const float av[3]) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_body_set_velocity: null world"); }
    return E(h)->setVelocity(w, id, v, av);
}

TF_API int tf_body_destroy(void* h, int32_t w, tf_id id) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_body_destroy: null world"); }
    return E(h)->destroyBody(w, id);
}

TF_API int tf_shape_remove(void* h, int32_t w, tf_id id) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_shape_remove: null world"); }
    return E(h)->removeShape(w, id);
}

TF_API int tf_shape_set_friction(void* h, int32_t w, tf_id id, float v) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_shape_set_friction: null world"); }
    return E(h)->setShapeValue(w, id, 0, v, 0, 0);
}

TF_API int tf_shape_set_restitution(void* h, int32_t w, tf_id id, float v) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_shape_set_restitution: null world"); }
    return E(h)->setShapeValue(w, id, 1, v, 0, 0);
}

TF_API int tf_shape_set_rolling_resistance(void* h, int32_t w, tf_id id, float v) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_shape_set_rolling_resistance: null world"); }
    return E(h)->setShapeValue(w, id, 2, v, 0, 0);
}

TF_API int tf_shape_set_filter(void* h, int32_t w, tf_id id, uint32_t category, uint32_t mask) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_shape_set_filter: null world"); }
    return E(h)->setShapeValue(w, id, 3, 0.0f, category, mask);
}

TF_API int tf_body_set_transform(void* h, int32_t w, tf_id id, const float p[3], const float q[4]) {
    if (!h || !p || !q) { return tfb::fail(TF_E_INVALID, "tf_body_set_transform: null"); }
    return E(h)->setTransform(w, id, tfb::v3of(p), tfb::q4of(q));
}

TF_API int tf_body_set_kinematic_target(void* h, int32_t w, tf_id id, const float p[3], const float q[4], float dt) {
    if (!h || !p || !q) { return tfb::fail(TF_E_INVALID, "tf_body_set_kinematic_target: null"); }
    return E(h)->setKinematicTarget(w, id, tfb::v3of(p), tfb::q4of(q), dt);
}

TF_API int tf_body_set_motion_type(void* h, int32_t w, tf_id id, int32_t type) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_body_set_motion_type: null world"); }
    return E(h)->setMotionType(w, id, type);
}

TF_API int tf_body_add_force(void* h, int32_t w, tf_id id, const float f[3], const float* point, int32_t wake) {
    if (!h || !f) { return tfb::fail(TF_E_INVALID, "tf_body_add_force: null"); }
    const tfb::Vec3 at = point ? tfb::v3of(point) : tfb::zero3();
    return E(h)->push(w, id, 0, tfb::v3of(f), point ? &at : nullptr, wake != 0);
}

TF_API int tf_body_add_torque(void* h, int32_t w, tf_id id, const float t[3], int32_t wake) {
    if (!h || !t) { return tfb::fail(TF_E_INVALID, "tf_body_add_torque: null"); }
    return E(h)->push(w, id, 1, tfb::v3of(t), nullptr, wake != 0);
}

TF_API int tf_body_add_impulse(void* h, int32_t w, tf_id id, const float j[3], const float* point, int32_t wake) {
    if (!h || !j) { return tfb::fail(TF_E_INVALID, "tf_body_add_impulse: null"); }
    const tfb::Vec3 at = point ? tfb::v3of(point) : tfb::zero3();
    return E(h)->push(w, id, 2, tfb::v3of(j), point ? &at : nullptr, wake != 0);
}

TF_API int tf_body_set_damping(void* h, int32_t w, tf_id id, float linear, float angular) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_body_set_damping: null world"); }
    return E(h)->setBodyValue(w, id, 0, linear, angular);
}

TF_API int tf_body_set_gravity_scale(void* h, int32_t w, tf_id id, float scale) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_body_set_gravity_scale: null world"); }
    return E(h)->setBodyValue(w, id, 1, scale, 0.0f);
}

TF_API int tf_body_set_can_sleep(void* h, int32_t w, tf_id id, int32_t can_sleep) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_body_set_can_sleep: null world"); }
    return E(h)->setBodyValue(w, id, 2, can_sleep ? 1.0f : 0.0f, 0.0f);
}

TF_API int tf_body_wake(void* h, int32_t w, tf_id id) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_body_wake: null world"); }
    return E(h)->setBodyValue(w, id, 3, 0.0f, 0.0f);
}

TF_API int tf_body_sleep(void* h, int32_t w, tf_id id) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_body_sleep: null world"); }
    return E(h)->setBodyValue(w, id, 4, 0.0f, 0.0f);
}

TF_API int tf_world_set_mix(void* h, int32_t which, int32_t mix) {
    if (!h || which < 0 || which > 1) { return tfb::fail(TF_E_INVALID, "tf_world_set_mix: bad arguments"); }
    if (mix != 0) {
        return tfb::fail(TF_E_UNSUPPORTED, "tf_world_set_mix: only the default mixes run on the device");
    }
    return TF_OK;
}

TF_API int tf_body_get_mass(void* h, int32_t w, tf_id id, float* mass, float center[3], float inertia[9]) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_body_get_mass: null world"); }
    tfb::HostBody* b = E(h)->body(w, id);
    const tfb::DBody zero{};
    const tfb::DBody& d = b ? b->d : zero;
    if (mass) { *mass = d.mass; }
    if (center) { center[0] = d.localCenter.x, center[1] = d.localCenter.y, center[2] = d.localCenter.z; }
    if (inertia) {
        for (int r = 0; r < 3; ++r) {
            inertia[3 * r + 0] = d.inertia.r[r].x;
            inertia[3 * r + 1] = d.inertia.r[r].y;
            inertia[3 * r + 2] = d.inertia.r[r].z;
        }
    }
    return TF_OK;
}

TF_API int tf_body_is_awake(void* h, int32_t w, tf_id id, int32_t* awake) {
    if (!h || !awake) { return tfb::fail(TF_E_INVALID, "tf_body_is_awake: null"); }
    Engine* e = E(h);
    const int rc = e->pull();
    if (rc != TF_OK) { return rc; }
    tfb::HostBody* b = e->body(w, id);
    *awake = (b && b->d.awake) ? 1 : 0;
    return TF_OK;
}

TF_API int tf_world_body_count(void* h, int64_t* total) {
    if (!h || !total) { return tfb::fail(TF_E_INVALID, "tf_world_body_count: null"); }
    int64_t n = 0;
    for (const auto& W : E(h)->worlds) { n += (int64_t)W.bodies.size(); }
    *total = n;
    return TF_OK;
}

TF_API int tf_world_get_states(void* h, float* p, float* q, float* v, float* w, int32_t* awake) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_get_states: null world"); }
    Engine* e = E(h);
    const int rc = e->pull();
    if (rc != TF_OK) { return rc; }
    size_t k = 0;
    for (const auto& W : e->worlds) {
        for (const auto& hb : W.bodies) {
            const tfb::DBody& d = hb.d;
            if (p) { p[3 * k] = d.xf.p.x, p[3 * k + 1] = d.xf.p.y, p[3 * k + 2] = d.xf.p.z; }
            if (q) { q[4 * k] = d.xf.q.x, q[4 * k + 1] = d.xf.q.y, q[4 * k + 2] = d.xf.q.z, q[4 * k + 3] = d.xf.q.w; }
            if (v) { v[3 * k] = d.v.x, v[3 * k + 1] = d.v.y, v[3 * k + 2] = d.v.z; }
            if (w) { w[3 * k] = d.w.x, w[3 * k + 1] = d.w.y, w[3 * k + 2] = d.w.z; }
            if (awake) { awake[k] = d.awake ? 1 : 0; }
            ++k;
        }
    }
    return TF_OK;
}

TF_API int tf_world_contacts(void* h, int32_t w, int32_t mode, tf_contact* out, int32_t cap, int32_t* count) {
    if (!h || !count) { return tfb::fail(TF_E_INVALID, "tf_world_contacts: null"); }
    Engine* e = E(h);
    if (w < 0 || w >= (int)e->worlds.size()) { return tfb::fail(TF_E_INVALID, "tf_world_contacts: bad world"); }
    const int rc = e->pull();
    if (rc != TF_OK) { return rc; }
    const auto& W = e->worlds[(size_t)w];
    int32_t n = 0;
    for (const tfb::DContact& c : W.contacts) {
        bool touching = false;
        for (int i = 0; i < c.count; ++i) {
            touching = touching || c.points[i].separation < 0.0f || c.points[i].normalImpulse > 0.0f;
        }
        if (mode < 2 && ((c.flags & tfb::kCRemoved) || (mode == 0 && !touching))) { continue; }
        if (out && n < cap) {
            tf_contact& o = out[n];
            std::memset(&o, 0, sizeof(o));
            o.key = c.key;
            o.part = c.part;
            o.shape_a = c.shapeA;
            o.shape_b = c.shapeB;
            o.body_a = c.bodyA;
            o.body_b = c.bodyB;
            o.point_count = c.count;
            o.feature_kind = c.featKind;
            o.feature_a = c.featA;
            o.feature_b = c.featB;
            o.normal[0] = c.normal.x, o.normal[1] = c.normal.y, o.normal[2] = c.normal.z;
            o.friction = c.friction;
            o.restitution = c.restitution;
            o.rolling_resistance = c.rollingResistance;
            o.rolling_impulse[0] = c.rollingImpulse.x, o.rolling_impulse[1] = c.rollingImpulse.y,
            o.rolling_impulse[2] = c.rollingImpulse.z;
            const tfb::Transform xa = W.bodies[c.bodyA].d.xf;
            for (int i = 0; i < c.count; ++i) {
                const tfb::Vec3 pw = tfb::apply(xa, c.points[i].localA);
                o.points[i][0] = pw.x, o.points[i][1] = pw.y, o.points[i][2] = pw.z;
                o.separations[i] = c.points[i].separation;
                o.normal_impulses[i] = c.points[i].normalImpulse;
                o.tangent_impulses[i][0] = c.points[i].tangentImpulse.x;
                o.tangent_impulses[i][1] = c.points[i].tangentImpulse.y;
                o.tangent_impulses[i][2] = c.points[i].tangentImpulse.z;
            }
        }
        ++n;
    }
    *count = n;
    return TF_OK;
}

// The bodies of a pair's shapes, world-local; shape indices come from the key (lower index first).
static void pairOf(const tfb::HostWorld& W, uint64_t key, uint32_t* sa, uint32_t* sb, uint32_t* ba, uint32_t* bb) {
    *sa = (uint32_t)(key >> 32);
    *sb = (uint32_t)key;
    *ba = *sa < W.shapes.size() ? W.shapes[*sa].d.body : UINT32_MAX;
    *bb = *sb < W.shapes.size() ? W.shapes[*sb].d.body : UINT32_MAX;
}

TF_API int tf_world_contact_events(void* h, int32_t w, tf_contact_event* out, int32_t cap, int32_t* count) {
    if (!h || !count) { return tfb::fail(TF_E_INVALID, "tf_world_contact_events: null"); }
    Engine* e = E(h);
    if (w < 0 || w >= (int)e->worlds.size()) { return tfb::fail(TF_E_INVALID, "tf_world_contact_events: bad world"); }
    std::vector<tfb::TouchEvent> ev;
    const int rc = e->events((size_t)w, &ev, nullptr);
    if (rc != TF_OK) { return rc; }
    const tfb::HostWorld& W = e->worlds[(size_t)w];
    // Events queued by calls before the step come first, as the reference reports them (src/world.cpp:1570).
    const size_t q = W.stepQueued.size();
    for (size_t i = 0; out && i < q && (int32_t)i < cap; ++i) { out[i] = W.stepQueued[i]; }
    for (size_t i = 0; out && i < ev.size() && (int32_t)(q + i) < cap; ++i) {
        tf_contact_event& o = out[q + i];
        pairOf(W, ev[i].key, &o.shape_a, &o.shape_b, &o.body_a, &o.body_b);
        o.begin = (int32_t)ev[i].begin;
    }
    *count = (int32_t)(q + ev.size());
    return TF_OK;
}

TF_API int tf_world_hit_events(void* h, int32_t w, tf_hit_event* out, int32_t cap, int32_t* count) {
    if (!h || !count) { return tfb::fail(TF_E_INVALID, "tf_world_hit_events: null"); }
    Engine* e = E(h);
    if (w < 0 || w >= (int)e->worlds.size()) { return tfb::fail(TF_E_INVALID, "tf_world_hit_events: bad world"); }
    std::vector<tfb::HitRecord> ev;
    const int rc = e->events((size_t)w, nullptr, &ev);
    if (rc != TF_OK) { return rc; }
    const tfb::HostWorld& W = e->worlds[(size_t)w];
    for (size_t i = 0; out && i < ev.size() && (int32_t)i < cap; ++i) {
        tf_hit_event& o = out[i];
        pairOf(W, ev[i].key, &o.shape_a, &o.shape_b, &o.body_a, &o.body_b);
        o.point[0] = ev[i].point.x, o.point[1] = ev[i].point.y, o.point[2] = ev[i].point.z;
        o.normal[0] = ev[i].normal.x, o.normal[1] = ev[i].normal.y, o.normal[2] = ev[i].normal.z;
        o.speed = ev[i].speed;
    }
    *count = (int32_t)ev.size();
    return TF_OK;
}

TF_API int tf_joint_create(void* h, int32_t w, const tf_joint_desc* desc, tf_id* out) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_joint_create: null world"); }
    return E(h)->createJoint(w, desc, out);
}

TF_API int tf_joint_get_info(void* h, int32_t w, tf_id joint, tf_joint_info* out) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_joint_get_info: null world"); }
    return E(h)->jointInfo(w, joint, out);
}

TF_API int tf_joint_set_limits(void* h, int32_t w, tf_id joint, int32_t limited, float lower, float upper) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_joint_set_limits: null world"); }
    const float v[3] = { limited ? 1.0f : 0.0f, lower, upper };
    return E(h)->jointSet(w, joint, 0, v);
}

TF_API int tf_joint_set_motor(void* h, int32_t w, tf_id joint, float speed, float max_force) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_joint_set_motor: null world"); }
    const float v[3] = { speed, max_force, 0.0f };
    return E(h)->jointSet(w, joint, 1, v);
}

TF_API int tf_joint_set_spring(void* h, int32_t w, tf_id joint, float hertz, float damping_ratio) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_joint_set_spring: null world"); }
    const float v[3] = { hertz, damping_ratio, 0.0f };
    return E(h)->jointSet(w, joint, 2, v);
}

TF_API int tf_joint_set_friction(void* h, int32_t w, tf_id joint, float max_friction) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_joint_set_friction: null world"); }
    const float v[3] = { max_friction, 0.0f, 0.0f };
    return E(h)->jointSet(w, joint, 3, v);
}

TF_API int tf_joint_set_swing(void* h, int32_t w, tf_id joint, float swing_y, float swing_z) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_joint_set_swing: null world"); }
    const float v[3] = { swing_y, swing_z, 0.0f };
    return E(h)->jointSet(w, joint, 4, v);
}

TF_API int tf_joint_set_break_limits(void* h, int32_t w, tf_id joint, float force, float torque) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_joint_set_break_limits: null world"); }
    const float v[3] = { force, torque, 0.0f };
    return E(h)->jointSet(w, joint, 5, v);
}

TF_API int tf_joint_destroy(void* h, int32_t w, tf_id joint) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_joint_destroy: null world"); }
    return E(h)->destroyJoint(w, joint);
}

TF_API int tf_world_broken_joints(void* h, int32_t w, tf_id* out, int32_t cap, int32_t* count) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_broken_joints: null world"); }
    return E(h)->brokenJoints(w, out, cap, count);
}

TF_API int tf_world_candidates(void* h, int32_t w, uint64_t* out, int32_t cap, int32_t* count) {
    if (!h || !count) { return tfb::fail(TF_E_INVALID, "tf_world_candidates: null"); }
    Engine* e = E(h);
    if (w < 0 || w >= (int)e->worlds.size()) { return tfb::fail(TF_E_INVALID, "tf_world_candidates: bad world"); }
    if (!e->layoutDirty) {
        const int rc = e->refreshCounts();
        if (rc != TF_OK) { return rc; }
    }
    if (e->lastCounts.empty() || e->layoutDirty) {
        *count = 0;
        return TF_OK;
    }
    const uint32_t n = e->lastCounts[(size_t)w].candCount;
    *count = (int32_t)n;
    if (out && cap > 0) {
        const size_t m = std::min<size_t>(n, (size_t)cap);
        cudaError_t err = cudaMemcpy(out, e->dCand.ptr + e->info[(size_t)w].candFirst, m * sizeof(uint64_t), cudaMemcpyDeviceToHost);
        if (err != cudaSuccess) { return tfb::fail(TF_E_CUDA, cudaGetErrorString(err)); }
    }
    return TF_OK;
}

TF_API int tf_world_profile(void* h, int32_t w, tf_profile* out) {
    if (!h || !out) { return tfb::fail(TF_E_INVALID, "tf_world_profile: null"); }
    Engine* e = E(h);
    if (w < 0 || w >= (int)e->worlds.size()) { return tfb::fail(TF_E_INVALID, "tf_world_profile: bad world"); }
    const int rc = e->refreshCounts();
    if (rc != TF_OK) { return rc; }
    *out = e->profiles[(size_t)w];
    return TF_OK;
}

TF_API int tf_world_awake_bodies(void* h, int64_t* count) {
    if (!h || !count) { return tfb::fail(TF_E_INVALID, "tf_world_awake_bodies: null"); }
    int64_t n = 0;
    const int rc = E(h)->refreshCounts();
    if (rc != TF_OK) { return rc; }
    for (const auto& c : E(h)->lastCounts) { n += c.awakeBodies; }
    *count = n;
    return TF_OK;
}

TF_API int tf_world_elapsed_ms(void* h, float* ms) {
    if (!h || !ms) { return tfb::fail(TF_E_INVALID, "tf_world_elapsed_ms: null"); }
    *ms = E(h)->lastElapsedMs;
    return TF_OK;
}

TF_API int tf_world_body_steps(void* h, int64_t* n) {
    if (!h || !n) { return tfb::fail(TF_E_INVALID, "tf_world_body_steps: null"); }
    *n = E(h)->bodyStepsTotal;
    return TF_OK;
}

TF_API int tf_world_add_forces(void* h, const float* forces, const float* torques) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_add_forces: null world"); }
    return E(h)->addForces(forces, torques);
}

TF_API int tf_world_read_poses(void* h, float* positions, float* rotations) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_read_poses: null world"); }
    return E(h)->readPoses(positions, rotations);
}

TF_API int tf_world_read_poses_async(void* h, float* positions, float* rotations) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_read_poses_async: null world"); }
    return E(h)->readPosesAsync(positions, rotations);
}

TF_API int tf_world_poses_wait(void* h) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_poses_wait: null world"); }
    return E(h)->posesWait();
}

TF_API int tf_world_set_profiling(void* h, int32_t on) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_set_profiling: null world"); }
    Engine* e = E(h);
    e->profiling = on != 0;
    for (int k = 0; k < Engine::kKernelKinds; ++k) {
        e->kernelMs[k] = 0.0;
        e->kernelLaunches[k] = 0;
    }
    return TF_OK;
}

TF_API int tf_world_kernel_times(void* h, float* ms, int64_t* launches, int32_t capacity, int32_t* count) {
    if (!h || !count) { return tfb::fail(TF_E_INVALID, "tf_world_kernel_times: null"); }
    Engine* e = E(h);
    *count = Engine::kKernelKinds;
    for (int k = 0; k < Engine::kKernelKinds && k < capacity; ++k) {
        if (ms) { ms[k] = (float)e->kernelMs[k]; }
        if (launches) { launches[k] = e->kernelLaunches[k]; }
    }
    return TF_OK;
}

TF_API const char* tf_kernel_name(int32_t k) {
    static const char* names[] = { "k_broadphase", "k_narrowphase", "k_wake", "k_prepare",
                                   "k_refresh",    "k_substep",     "k_finish", "k_collide" };
    return (k >= 0 && k < 8) ? names[k] : "";
}

TF_API int tf_world_work_counts(void* h, int64_t out[6]) {
    if (!h || !out) { return tfb::fail(TF_E_INVALID, "tf_world_work_counts: null"); }
    Engine* e = E(h);
    for (int k = 0; k < 6; ++k) { out[k] = 0; }
    out[0] = (int64_t)e->totalBodies;
    const int rc = e->refreshCounts();
    if (rc != TF_OK) { return rc; }
    for (const auto& c : e->lastCounts) {
        out[1] += c.awakeBodies;
        out[2] += c.candCount;
        out[3] += c.contactCount;
        out[4] += c.activeCount;
        out[5] += c.activePoints;
    }
    return TF_OK;
}

TF_API int tf_world_launch_count(void* h, int64_t* launches) {
    if (!h || !launches) { return tfb::fail(TF_E_INVALID, "tf_world_launch_count: null"); }
    *launches = E(h)->launches;
    return TF_OK;
}

TF_API int tf_tape_record(void* h, float dt, int32_t n_steps) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_tape_record: null"); }
    return E(h)->tapeRecord(dt, n_steps);
}

TF_API int tf_adjoint_forward(void* h, int32_t precision, const double* initial_state, const double* mass,
                              const double* friction, double* final_state) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_adjoint_forward: null"); }
    Engine* e = E(h);
    if (!e->taped) { return tfb::fail(TF_E_INVALID, "tf_adjoint_forward: record a run with tf_tape_record first"); }
    if (cudaSetDevice(e->device) != cudaSuccess) { return tfb::fail(TF_E_CUDA, "tf_adjoint_forward: cudaSetDevice"); }
    if (!e->adjRun) { e->adjRun = tfb::adjointCreate(); }
    return tfb::adjointForward(e->adjRun, e->adjoint, e->stream, precision, initial_state, mass, friction, final_state);
}

TF_API int tf_adjoint_backward(void* h, const double* grad_final, double* grad_initial, double* grad_mass,
                               double* grad_friction) {
    if (!h || !grad_final) { return tfb::fail(TF_E_INVALID, "tf_adjoint_backward: null"); }
    Engine* e = E(h);
    if (!e->adjRun) { return tfb::fail(TF_E_INVALID, "tf_adjoint_backward: run tf_adjoint_forward first"); }
    if (cudaSetDevice(e->device) != cudaSuccess) { return tfb::fail(TF_E_CUDA, "tf_adjoint_backward: cudaSetDevice"); }
    return tfb::adjointBackward(e->adjRun, e->adjoint, e->stream, grad_final, grad_initial, grad_mass, grad_friction);
}

TF_API int tf_adjoint_elapsed_ms(void* h, float ms[2]) {
    if (!h || !ms) { return tfb::fail(TF_E_INVALID, "tf_adjoint_elapsed_ms: null"); }
    Engine* e = E(h);
    ms[0] = ms[1] = 0.0f;
    if (e->adjRun) {
        float all[4];
        tfb::adjointTimes(e->adjRun, all);
        ms[0] = all[0];
        ms[1] = all[1];
    }
    return TF_OK;
}

TF_API int tf_adjoint_backward_ms(void* h, float ms[2]) {
    if (!h || !ms) { return tfb::fail(TF_E_INVALID, "tf_adjoint_backward_ms: null"); }
    Engine* e = E(h);
    ms[0] = ms[1] = 0.0f;
    if (e->adjRun) {
        float all[4];
        tfb::adjointTimes(e->adjRun, all);
        ms[0] = all[2];
        ms[1] = all[3];
    }
    return TF_OK;
}

TF_API int tf_adjoint_branches(void* h, uint64_t* per_world) {
    if (!h || !per_world) { return tfb::fail(TF_E_INVALID, "tf_adjoint_branches: null"); }
    Engine* e = E(h);
    if (!e->adjRun) { return tfb::fail(TF_E_INVALID, "tf_adjoint_branches: run tf_adjoint_forward first"); }
    if (cudaSetDevice(e->device) != cudaSuccess) { return tfb::fail(TF_E_CUDA, "tf_adjoint_branches: cudaSetDevice"); }
    return tfb::adjointBranches(e->adjRun, (int)e->worlds.size(), per_world);
}

TF_API int tf_world_save_state(void* h, int32_t slot) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_save_state: null"); }
    if (slot < 0) { return tfb::fail(TF_E_INVALID, "tf_world_save_state: negative slot"); }
    return E(h)->saveState(slot);
}

TF_API int tf_world_restore_state(void* h, int32_t slot) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_restore_state: null"); }
    if (slot < 0) { return tfb::fail(TF_E_INVALID, "tf_world_restore_state: negative slot"); }
    return E(h)->restoreState(slot);
}

TF_API int tf_world_autotune(void* h, float dt, int32_t trial_steps, uint32_t* out) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_autotune: null"); }
    return E(h)->autotune(dt, trial_steps, out);
}

TF_API int tf_world_solver_counts(void* h, int32_t w, int32_t out[8]) {
    if (!h || !out) { return tfb::fail(TF_E_INVALID, "tf_world_solver_counts: null"); }
    Engine* e = E(h);
    if (w < 0 || w >= (int)e->worlds.size()) { return tfb::fail(TF_E_INVALID, "tf_world_solver_counts: bad world"); }
    for (int k = 0; k < 8; ++k) { out[k] = 0; }
    const int rc = e->refreshCounts();
    if (rc != TF_OK) { return rc; }
    if (e->lastCounts.size() != e->worlds.size()) { return TF_OK; }
    const tfb::WorldCounts& c = e->lastCounts[(size_t)w];
    out[0] = (int32_t)c.activeCount;
    out[1] = (int32_t)c.colorCount;
    out[2] = (int32_t)c.restCount;
    out[3] = (int32_t)c.impactCount;
    out[4] = (int32_t)c.impactColorCount;
    out[5] = (int32_t)c.impactRestCount;
    out[6] = (int32_t)c.fastCount;
    out[7] = (int32_t)c.fastSolidCount;
    return TF_OK;
}

TF_API int tf_world_set_launch(void* h, int32_t kernel, int32_t threads, int32_t big_bodies, int32_t smem_bytes) {
    if (!h) { return tfb::fail(TF_E_INVALID, "tf_world_set_launch: null"); }
    if ((big_bodies < 0 && !(kernel == 5 && big_bodies == -1)) || smem_bytes < 0) {
        return tfb::fail(TF_E_INVALID, "tf_world_set_launch: negative size");
    }
    Engine* e = E(h);
    if (cudaSetDevice(e->device) != cudaSuccess) { return tfb::fail(TF_E_CUDA, "tf_world_set_launch: cudaSetDevice"); }
    return e->setLaunch(kernel, (uint32_t)threads, (uint32_t)big_bodies, (uint32_t)smem_bytes);
}

TF_API int tf_world_get_launch(void* h, int32_t kernel, uint32_t out[6]) {
    if (!h || !out) { return tfb::fail(TF_E_INVALID, "tf_world_get_launch: null"); }
    const int rc = E(h)->getLaunch(kernel, out);
    if (rc != TF_OK) { return tfb::fail(rc, "tf_world_get_launch: bad kernel index"); }
    return TF_OK;
}

}
