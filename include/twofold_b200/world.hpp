// twofold::World over the B200 contact pipeline: the drop-in C++ surface for World::step.
//
// Code written against the reference's include/twofold/world.h (World, BodyDesc, ShapeDesc, WorldSettings,
// StepProfile, ContactInfo, the id types and geometry alternatives) compiles against this header for the
// part of the API the contact pipeline covers: building bodies and shapes, step(), reading poses,
// velocities, mass, sleep state, contacts, contact and hit events and the step profile, setting velocities
// and adding forces, and joints (creating them, their info, the joints that broke).
// Every call forwards to the C ABI in twofold_b200.h; the library owns the device state.
//
// Same conventions as the reference (include/twofold/world.h:362-510, src/world.cpp:352-371): invalid ids
// make getters return defaults and setters do nothing; step() ignores dt <= 0 or non-finite dt; nothing
// throws. What the reference reports by silence this header also records: status() is the last C ABI
// status (TF_OK or a negative TF_E* code) and statusMessage() its text.
//
// Differences a caller can see:
//   - Geometry: spheres, boxes, prisms, hulls, half-spaces and meshes (on static and kinematic bodies) run on
//     the device. Cylinders are refused by addShape (an invalid ShapeId, status TF_E_UNSUPPORTED), as are
//     sensors and meshes on dynamic bodies. Bodies locked to
//     a plane run when every such body of the world is locked to the same plane; createBody refuses a
//     second plane (an invalid BodyId, status TF_E_UNSUPPORTED).
//   - addForce/addTorque queue the force for the next step and act on awake bodies only (wake = false).
//   - Copying a World is not provided; move it instead.
//   - The math types carry the reference's fields and a few operators, not all of math.h.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <variant>
#include <vector>

#include "../twofold_b200.h"

namespace twofold {

struct Vec2 {
    float x = 0, y = 0;
    Vec2() = default;
    constexpr Vec2(float x_, float y_) : x(x_), y(y_) {}
};

struct Vec3 {
    float x = 0, y = 0, z = 0;
    Vec3() = default;
    constexpr Vec3(float x_, float y_, float z_) : x(x_), y(y_), z(z_) {}
    Vec3 operator+(const Vec3& b) const { return { x + b.x, y + b.y, z + b.z }; }
    Vec3 operator-(const Vec3& b) const { return { x - b.x, y - b.y, z - b.z }; }
    Vec3 operator-() const { return { -x, -y, -z }; }
    Vec3 operator*(float s) const { return { x * s, y * s, z * s }; }
};

inline float dot(const Vec3& a, const Vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec3 cross(const Vec3& a, const Vec3& b) { return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x }; }
inline float length(const Vec3& v) { return std::sqrt(dot(v, v)); }

struct Mat3 {
    Vec3 r[3] = { { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } };
    static Mat3 zero() {
        Mat3 m;
        m.r[0] = m.r[1] = m.r[2] = Vec3{};
        return m;
    }
};

struct Quat {
    float x = 0, y = 0, z = 0, w = 1;
    Quat() = default;
    constexpr Quat(float x_, float y_, float z_, float w_) : x(x_), y(y_), z(z_), w(w_) {}
    // v + 2w (u x v) + 2 u x (u x v), u the vector part.
    Vec3 rotate(const Vec3& v) const {
        const Vec3 u{ x, y, z };
        const Vec3 t = cross(u, v) * 2.0f;
        return v + t * w + cross(u, t);
    }
};

struct Transform {
    Vec3 p;
    Quat q;
    Vec3 apply(const Vec3& v) const { return p + q.rotate(v); }
};

struct BodyId {
    uint32_t index = UINT32_MAX;
    uint32_t generation = 0;
    bool operator==(const BodyId& b) const { return index == b.index && generation == b.generation; }
    bool operator!=(const BodyId& b) const { return !(*this == b); }
};

struct ShapeId {
    uint32_t index = UINT32_MAX;
    uint32_t generation = 0;
    bool operator==(const ShapeId& b) const { return index == b.index && generation == b.generation; }
    bool operator!=(const ShapeId& b) const { return !(*this == b); }
};

enum class MotionType : uint8_t { Static, Kinematic, Dynamic };

enum LockFlags : uint8_t {
    LockTranslationX = TF_LOCK_TRANSLATION_X,
    LockTranslationY = TF_LOCK_TRANSLATION_Y,
    LockTranslationZ = TF_LOCK_TRANSLATION_Z,
    LockRotationX = TF_LOCK_ROTATION_X,
    LockRotationY = TF_LOCK_ROTATION_Y,
    LockRotationZ = TF_LOCK_ROTATION_Z,
    LockPlanar = TF_LOCK_PLANAR,
};

struct Sphere {
    float radius = 0.5f;
};
struct Box {
    Vec3 halfExtents{ 0.5f, 0.5f, 0.5f };
};
struct Cylinder {
    float radius = 0.5f;
    float halfHeight = 0.5f;
};
struct Prism {
    std::vector<Vec2> polygon;
    float zMin = -0.5f;
    float zMax = 0.5f;
};
struct Hull {
    std::vector<Vec3> points;
    int maxVertices = 64;
};
struct HalfSpace {};
// TriangleMesh (include/twofold/mesh.h:13-30): triangles indexed three to a face; vertices at the same position
// are merged and degenerate triangles dropped when it is built. A World sends it to its device the first time
// one of its shapes uses it.
class TriangleMesh {
public:
    TriangleMesh(const std::vector<Vec3>& vertices, const std::vector<uint32_t>& indices) : inputIndices_(indices) {
        for (const Vec3& v : vertices) { input_.insert(input_.end(), { v.x, v.y, v.z }); }
        // The built mesh is read back from a handle that holds only it (no device is touched).
        void* h = nullptr;
        if (tf_world_create(nullptr, 1, 0, &h) != TF_OK) { return; }
        int32_t id = -1;
        int32_t counts[3] = { 0, 0, 0 };
        if (tf_mesh_create(h, input_.data(), (int32_t)vertices.size(), indices.data(), (int32_t)indices.size(), &id) == TF_OK &&
            tf_mesh_read(h, id, counts, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr) == TF_OK) {
            std::vector<float> v(3 * (size_t)counts[0]);
            indices_.resize(3 * (size_t)counts[1]);
            tf_mesh_read(h, id, counts, v.data(), indices_.data(), nullptr, nullptr, nullptr, nullptr);
            for (int32_t i = 0; i < counts[0]; ++i) { vertices_.push_back({ v[3 * i], v[3 * i + 1], v[3 * i + 2] }); }
        }
        tf_world_destroy(h);
    }
    TriangleMesh(const TriangleMesh&) = delete;
    TriangleMesh& operator=(const TriangleMesh&) = delete;

    const std::vector<Vec3>& vertices() const { return vertices_; }
    // Three per triangle, in the mesh's own order.
    const std::vector<uint32_t>& indices() const { return indices_; }
    int triangleCount() const { return (int)(indices_.size() / 3); }

    // What it was built from, for a World to build it again on its device.
    const std::vector<float>& input() const { return input_; }
    const std::vector<uint32_t>& inputIndices() const { return inputIndices_; }

private:
    std::vector<float> input_;
    std::vector<uint32_t> inputIndices_;
    std::vector<Vec3> vertices_;
    std::vector<uint32_t> indices_;
};
struct Mesh {
    std::shared_ptr<const TriangleMesh> mesh;
};
using Geometry = std::variant<Sphere, Box, Cylinder, Prism, Hull, HalfSpace, Mesh>;

struct ShapeDesc {
    Geometry geometry = Box{};
    Vec3 position;
    Quat rotation;
    float density = 1.0f;
    float friction = 0.5f;
    float restitution = 0.0f;
    float rollingResistance = 0.0f;
    uint32_t category = 1;
    uint32_t mask = 0xffffffffu;
    bool sensor = false;
    void* userData = nullptr;
};

struct BodyDesc {
    MotionType type = MotionType::Dynamic;
    Vec3 position;
    Quat rotation;
    Vec3 linearVelocity;
    Vec3 angularVelocity;
    float linearDamping = 0.0f;
    float angularDamping = 0.0f;
    float gravityScale = 1.0f;
    uint8_t locks = 0;
    Quat lockFrame;
    bool awake = true;
    bool canSleep = true;
    void* userData = nullptr;
};

struct MassProperties {
    float mass = 0.0f;
    Vec3 center;
    Mat3 inertia = Mat3::zero();
};

struct WorldSettings {
    Vec3 gravity{ 0.0f, -9.81f, 0.0f };
    float lengthUnit = 1.0f;
    int substeps = 4;
    float contactHertz = 30.0f;
    float contactDampingRatio = 10.0f;
    float maxPushoutSpeed = 3.0f;
    float maxLinearSpeed = 1000.0f;
    float maxAngularSpeed = 1000.0f;
    float restitutionThreshold = 1.0f;
    float hitThreshold = 1.0f;
    float sleepThreshold = 0.05f;
    float timeToSleep = 0.5f;
    float contactReuseDistance = 0.0005f;
    float contactReuseAngle = 0.035f;
    float jointHertz = 60.0f;
    float jointDampingRatio = 2.0f;
    bool continuous = true;
};

// WorldSettings-side material mixing (include/twofold/world.h:243-248). Mixing runs on the device, where a host
// function cannot be called: only the reference's default mixes run, and a World given any other function
// records TF_E_UNSUPPORTED (status()).
struct MaterialInput {
    float value;
    MotionType type;
};

using MixFunction = float (*)(const MaterialInput& a, const MaterialInput& b);

struct ContactInfo {
    BodyId bodyA;
    BodyId bodyB;
    ShapeId shapeA;
    ShapeId shapeB;
    Vec3 normal;
    float friction = 0.0f;
    float restitution = 0.0f;
    float rollingResistance = 0.0f;
    Vec3 rollingImpulse;
    int pointCount = 0;
    Vec3 points[4];
    float separations[4] = {};
    float normalImpulses[4] = {};
    Vec3 tangentImpulses[4];
};

struct JointId {
    uint32_t index = UINT32_MAX;
    uint32_t generation = 0;
    bool operator==(const JointId& b) const { return index == b.index && generation == b.generation; }
    bool operator!=(const JointId& b) const { return !(*this == b); }
};

// Anchors and axes are in world space, at the poses the bodies have when the joint is made.
struct PointJoint {
    Vec3 anchor;
};
struct FixedJoint {
    Vec3 anchor;
};
struct HingeJoint {
    Vec3 anchor;
    Vec3 axis{ 0, 0, 1 };
    bool limited = false;
    float lowerAngle = 0.0f;
    float upperAngle = 0.0f;
    float motorSpeed = 0.0f;
    float maxMotorTorque = 0.0f;
    float frictionTorque = 0.0f;
};
struct SliderJoint {
    Vec3 anchor;
    Vec3 axis{ 1, 0, 0 };
    bool limited = false;
    float lowerTranslation = 0.0f;
    float upperTranslation = 0.0f;
    float motorSpeed = 0.0f;
    float maxMotorForce = 0.0f;
    float frictionForce = 0.0f;
};
struct DistanceJoint {
    Vec3 anchorA;
    Vec3 anchorB;
    float length = -1.0f;
    float hertz = 0.0f;
    float dampingRatio = 0.0f;
    bool limited = false;
    float minDistance = 0.0f;
    float maxDistance = 0.0f;
};
struct SwingTwistJoint {
    Vec3 anchor;
    Vec3 axis{ 1, 0, 0 };
    Vec3 normal{ 0, 1, 0 };
    float swingY = 3.14159265f;
    float swingZ = 3.14159265f;
    float lowerTwist = -3.14159265f;
    float upperTwist = 3.14159265f;
    float frictionTorque = 0.0f;
};

using JointKind = std::variant<PointJoint, FixedJoint, HingeJoint, SliderJoint, DistanceJoint, SwingTwistJoint>;
enum class JointType : uint8_t { Point, Fixed, Hinge, Slider, Distance, SwingTwist };

struct JointDesc {
    // Left unset, body B is joined to the world.
    BodyId bodyA;
    BodyId bodyB;
    JointKind kind = PointJoint{};
    bool collideConnected = false;
    float breakForce = INFINITY;
    float breakTorque = INFINITY;
    void* userData = nullptr;
};

struct JointInfo {
    JointId joint;
    JointType type = JointType::Point;
    BodyId bodyA;
    BodyId bodyB;
    Vec3 anchorA;
    Vec3 anchorB;
    Vec3 axis;
    // The hinge angle, slider translation, distance or twist. Zero for point and fixed joints.
    float value = 0.0f;
    // Force and torque on body B in the last step the joint was active, the torque about anchor B.
    Vec3 force;
    Vec3 torque;
    bool broken = false;
};

// Two shapes that started or stopped touching. Shape A has the lower index.
struct ContactEvent {
    BodyId bodyA;
    BodyId bodyB;
    ShapeId shapeA;
    ShapeId shapeB;
    // False when they stopped.
    bool begin = true;
};

// The fastest approaching point of a touching pair, when faster than WorldSettings::hitThreshold.
struct HitEvent {
    BodyId bodyA;
    BodyId bodyB;
    ShapeId shapeA;
    ShapeId shapeB;
    Vec3 point;
    // Points from shape A to shape B.
    Vec3 normal;
    float speed = 0.0f;
};

struct StepProfile {
    float total = 0.0f;
    float broadphase = 0.0f;
    float narrowphase = 0.0f;
    float solver = 0.0f;
    float continuous = 0.0f;
    float sleep = 0.0f;
    int candidatePairs = 0;
    int sweptPairs = 0;
    int impacts = 0;
    int manifolds = 0;
    int touchingContacts = 0;
    int awakeBodies = 0;
    int awakeIslands = 0;
};

class World {
public:
    explicit World(const WorldSettings& settings = {}, int device = 0) : settings_(settings) {
        const tf_settings s = toC(settings);
        void* h = nullptr;
        status_ = tf_world_create(&s, 1, device, &h);
        handle_ = h;
    }
    ~World() {
        if (handle_) { tf_world_destroy(handle_); }
    }
    World(const World&) = delete;
    World& operator=(const World&) = delete;
    World(World&& o) noexcept { *this = std::move(o); }
    World& operator=(World&& o) noexcept {
        if (this != &o) {
            if (handle_) { tf_world_destroy(handle_); }
            handle_ = o.handle_;
            o.handle_ = nullptr;
            settings_ = o.settings_;
            profile_ = o.profile_;
            bodies_ = std::move(o.bodies_);
            shapes_ = std::move(o.shapes_);
            meshIds_ = std::move(o.meshIds_);
            meshes_ = std::move(o.meshes_);
            shapeOwner_ = std::move(o.shapeOwner_);
            jointEnds_ = std::move(o.jointEnds_);
            status_ = o.status_;
        }
        return *this;
    }

    const WorldSettings& settings() const { return settings_; }
    void setSettings(const WorldSettings& settings) {
        settings_ = settings;
        const tf_settings s = toC(settings);
        note(tf_world_set_settings(handle_, &s));
    }
    void setGravity(const Vec3& gravity) {
        WorldSettings s = settings_;
        s.gravity = gravity;
        setSettings(s);
    }

    void step(float dt) {
        if (!(dt > 0.0f) || !std::isfinite(dt) || !handle_) { return; }
        if (!note(tf_world_step(handle_, dt, 1))) { return; }
        tf_profile p{};
        if (note(tf_world_profile(handle_, 0, &p))) {
            profile_.total = p.total;
            profile_.broadphase = p.broadphase;
            profile_.narrowphase = p.narrowphase;
            profile_.solver = p.solver;
            profile_.continuous = p.continuous;
            profile_.sleep = p.sleep;
            profile_.candidatePairs = p.candidate_pairs;
            profile_.sweptPairs = p.swept_pairs;
            profile_.impacts = p.impacts;
            profile_.manifolds = p.manifolds;
            profile_.touchingContacts = p.touching_contacts;
            profile_.awakeBodies = p.awake_bodies;
            profile_.awakeIslands = p.awake_islands;
        }
    }
    const StepProfile& profile() const { return profile_; }

    BodyId createBody(const BodyDesc& d) {
        tf_body_desc c{};
        c.type = d.type == MotionType::Static ? TF_STATIC : d.type == MotionType::Kinematic ? TF_KINEMATIC : TF_DYNAMIC;
        put3(c.position, d.position);
        put4(c.rotation, d.rotation);
        put3(c.linear_velocity, d.linearVelocity);
        put3(c.angular_velocity, d.angularVelocity);
        c.linear_damping = d.linearDamping;
        c.angular_damping = d.angularDamping;
        c.gravity_scale = d.gravityScale;
        c.locks = d.locks;
        put4(c.lock_frame, d.lockFrame);
        c.awake = d.awake ? 1 : 0;
        c.can_sleep = d.canSleep ? 1 : 0;
        tf_id id{ UINT32_MAX, 0 };
        if (!note(tf_body_create(handle_, 0, &c, &id))) { return {}; }
        if (id.index >= bodies_.size()) { bodies_.resize(id.index + 1, BodyId{}); }
        bodies_[id.index] = BodyId{ id.index, id.generation };
        return bodies_[id.index];
    }

    ShapeId addShape(BodyId body, const ShapeDesc& d) {
        if (!isValid(body)) { return {}; }
        tf_shape_desc c{};
        std::vector<float> points;
        if (const Sphere* s = std::get_if<Sphere>(&d.geometry)) {
            c.geometry = TF_SPHERE;
            c.radius = s->radius;
        } else if (const Box* b = std::get_if<Box>(&d.geometry)) {
            c.geometry = TF_BOX;
            put3(c.half_extents, b->halfExtents);
        } else if (const Cylinder* y = std::get_if<Cylinder>(&d.geometry)) {
            c.geometry = TF_CYLINDER;
            c.radius = y->radius;
            c.half_height = y->halfHeight;
        } else if (const Prism* p = std::get_if<Prism>(&d.geometry)) {
            c.geometry = TF_PRISM;
            for (const Vec2& v : p->polygon) { points.insert(points.end(), { v.x, v.y }); }
            c.point_count = (int32_t)p->polygon.size();
            c.z_min = p->zMin;
            c.z_max = p->zMax;
        } else if (const Hull* hl = std::get_if<Hull>(&d.geometry)) {
            c.geometry = TF_HULL;
            for (const Vec3& v : hl->points) { points.insert(points.end(), { v.x, v.y, v.z }); }
            c.point_count = (int32_t)hl->points.size();
            c.max_vertices = hl->maxVertices;
        } else if (std::holds_alternative<HalfSpace>(d.geometry)) {
            c.geometry = TF_HALFSPACE;
        } else {
            c.geometry = TF_MESH;
            const Mesh& m = std::get<Mesh>(d.geometry);
            if (!m.mesh) { return {}; }
            auto found = meshIds_.find(m.mesh.get());
            if (found == meshIds_.end()) {
                int32_t id = -1;
                const std::vector<float>& v = m.mesh->input();
                const std::vector<uint32_t>& i = m.mesh->inputIndices();
                if (!note(tf_mesh_create(handle_, v.data(), (int32_t)(v.size() / 3), i.data(), (int32_t)i.size(), &id))) {
                    return {};
                }
                found = meshIds_.emplace(m.mesh.get(), id).first;
                meshes_.push_back(m.mesh);
            }
            c.mesh = found->second;
        }
        c.points = points.empty() ? nullptr : points.data();
        put3(c.position, d.position);
        put4(c.rotation, d.rotation);
        c.density = d.density;
        c.friction = d.friction;
        c.restitution = d.restitution;
        c.rolling_resistance = d.rollingResistance;
        c.category = d.category;
        c.mask = d.mask;
        c.sensor = d.sensor ? 1 : 0;
        tf_id id{ UINT32_MAX, 0 };
        if (!note(tf_shape_add(handle_, 0, tf_id{ body.index, body.generation }, &c, &id))) { return {}; }
        if (id.index >= shapes_.size()) {
            shapes_.resize(id.index + 1, ShapeId{});
            shapeOwner_.resize(id.index + 1, UINT32_MAX);
        }
        shapes_[id.index] = ShapeId{ id.index, id.generation };
        shapeOwner_[id.index] = body.index;
        return shapes_[id.index];
    }

    // ---- Calls between steps (include/twofold/world.h:375-463) ----

    void setFrictionMix(MixFunction mix) { note(tf_world_set_mix(handle_, 0, mix ? 1 : 0)); }
    void setRestitutionMix(MixFunction mix) { note(tf_world_set_mix(handle_, 1, mix ? 1 : 0)); }

    void destroyBody(BodyId body) {
        if (!isValid(body) || !note(tf_body_destroy(handle_, 0, cid(body)))) { return; }
        bodies_[body.index] = BodyId{ UINT32_MAX, body.generation + 1 };
        for (size_t i = 0; i < shapes_.size(); ++i) {
            if (shapeOwner_[i] == body.index && shapes_[i].index != UINT32_MAX) {
                shapes_[i] = ShapeId{ UINT32_MAX, shapes_[i].generation + 1 };
            }
        }
        for (size_t k = 0; k < joints_.size(); ++k) {
            if (joints_[k].index != UINT32_MAX && (jointEnds_[2 * k] == body.index || jointEnds_[2 * k + 1] == body.index)) {
                joints_[k] = JointId{ UINT32_MAX, joints_[k].generation + 1 };
            }
        }
    }
    void removeShape(ShapeId shape) {
        if (!isValid(shape) || !note(tf_shape_remove(handle_, 0, cid(shape)))) { return; }
        shapes_[shape.index] = ShapeId{ UINT32_MAX, shape.generation + 1 };
    }
    void setFriction(ShapeId shape, float friction) {
        if (isValid(shape)) { note(tf_shape_set_friction(handle_, 0, cid(shape), friction)); }
    }
    void setRestitution(ShapeId shape, float restitution) {
        if (isValid(shape)) { note(tf_shape_set_restitution(handle_, 0, cid(shape), restitution)); }
    }
    void setRollingResistance(ShapeId shape, float rollingResistance) {
        if (isValid(shape)) { note(tf_shape_set_rolling_resistance(handle_, 0, cid(shape), rollingResistance)); }
    }
    void setFilter(ShapeId shape, uint32_t category, uint32_t mask) {
        if (isValid(shape)) { note(tf_shape_set_filter(handle_, 0, cid(shape), category, mask)); }
    }
    void setTransform(BodyId body, const Vec3& position, const Quat& rotation) {
        if (!isValid(body)) { return; }
        float p[3], q[4];
        put3(p, position);
        put4(q, rotation);
        note(tf_body_set_transform(handle_, 0, cid(body), p, q));
    }
    void setKinematicTarget(BodyId body, const Vec3& position, const Quat& rotation, float dt) {
        if (!isValid(body)) { return; }
        float p[3], q[4];
        put3(p, position);
        put4(q, rotation);
        note(tf_body_set_kinematic_target(handle_, 0, cid(body), p, q, dt));
    }
    void setMotionType(BodyId body, MotionType type) {
        if (!isValid(body)) { return; }
        const int32_t t = type == MotionType::Static ? TF_STATIC : type == MotionType::Kinematic ? TF_KINEMATIC : TF_DYNAMIC;
        note(tf_body_set_motion_type(handle_, 0, cid(body), t));
    }
    void addForceAtPoint(BodyId body, const Vec3& force, const Vec3& point, bool wake = true) {
        if (!isValid(body)) { return; }
        float f[3], at[3];
        put3(f, force);
        put3(at, point);
        note(tf_body_add_force(handle_, 0, cid(body), f, at, wake ? 1 : 0));
    }
    void addImpulse(BodyId body, const Vec3& impulse, bool wake = true) {
        if (!isValid(body)) { return; }
        float j[3];
        put3(j, impulse);
        note(tf_body_add_impulse(handle_, 0, cid(body), j, nullptr, wake ? 1 : 0));
    }
    void addImpulseAtPoint(BodyId body, const Vec3& impulse, const Vec3& point, bool wake = true) {
        if (!isValid(body)) { return; }
        float j[3], at[3];
        put3(j, impulse);
        put3(at, point);
        note(tf_body_add_impulse(handle_, 0, cid(body), j, at, wake ? 1 : 0));
    }
    void setDamping(BodyId body, float linear, float angular) {
        if (isValid(body)) { note(tf_body_set_damping(handle_, 0, cid(body), linear, angular)); }
    }
    void setGravityScale(BodyId body, float scale) {
        if (isValid(body)) { note(tf_body_set_gravity_scale(handle_, 0, cid(body), scale)); }
    }
    void wake(BodyId body) {
        if (isValid(body)) { note(tf_body_wake(handle_, 0, cid(body))); }
    }
    void sleep(BodyId body) {
        if (isValid(body)) { note(tf_body_sleep(handle_, 0, cid(body))); }
    }
    void setCanSleep(BodyId body, bool canSleep) {
        if (isValid(body)) { note(tf_body_set_can_sleep(handle_, 0, cid(body), canSleep ? 1 : 0)); }
    }

    bool isValid(BodyId body) const { return body.index < bodies_.size() && bodies_[body.index] == body; }
    bool isValid(ShapeId shape) const { return shape.index < shapes_.size() && shapes_[shape.index] == shape; }
    std::vector<BodyId> bodies() const {
        std::vector<BodyId> out;
        for (const BodyId& b : bodies_) {
            if (b.index != UINT32_MAX) { out.push_back(b); }
        }
        return out;
    }

    Transform transform(BodyId body) const {
        Transform t;
        Vec3 v, w;
        state(body, t, v, w);
        return t;
    }
    Vec3 position(BodyId body) const { return transform(body).p; }
    Quat rotation(BodyId body) const { return transform(body).q; }
    Vec3 centerOfMass(BodyId body) const { return transform(body).apply(massProperties(body).center); }
    Vec3 linearVelocity(BodyId body) const {
        Transform t;
        Vec3 v, w;
        state(body, t, v, w);
        return v;
    }
    Vec3 angularVelocity(BodyId body) const {
        Transform t;
        Vec3 v, w;
        state(body, t, v, w);
        return w;
    }
    void setLinearVelocity(BodyId body, const Vec3& v) { setVelocities(body, &v, nullptr); }
    void setAngularVelocity(BodyId body, const Vec3& w) { setVelocities(body, nullptr, &w); }

    void addForce(BodyId body, const Vec3& force, bool wake = true) {
        if (!isValid(body)) { return; }
        float f[3];
        put3(f, force);
        note(tf_body_add_force(handle_, 0, cid(body), f, nullptr, wake ? 1 : 0));
    }
    void addTorque(BodyId body, const Vec3& torque, bool wake = true) {
        if (!isValid(body)) { return; }
        float t[3];
        put3(t, torque);
        note(tf_body_add_torque(handle_, 0, cid(body), t, wake ? 1 : 0));
    }

    MassProperties massProperties(BodyId body) const {
        MassProperties m;
        if (!isValid(body)) { return m; }
        float mass = 0, center[3] = {}, inertia[9] = {};
        if (!note(tf_body_get_mass(handle_, 0, tf_id{ body.index, body.generation }, &mass, center, inertia))) { return m; }
        m.mass = mass;
        m.center = Vec3{ center[0], center[1], center[2] };
        for (int i = 0; i < 3; ++i) { m.inertia.r[i] = Vec3{ inertia[3 * i], inertia[3 * i + 1], inertia[3 * i + 2] }; }
        return m;
    }

    bool isAwake(BodyId body) const {
        int32_t awake = 0;
        if (!isValid(body)) { return false; }
        note(tf_body_is_awake(handle_, 0, tf_id{ body.index, body.generation }, &awake));
        return awake != 0;
    }

    std::vector<ContactInfo> contacts(bool includeSpeculative = false) const {
        std::vector<ContactInfo> out;
        int32_t n = 0;
        const int mode = includeSpeculative ? 1 : 0;
        if (!note(tf_world_contacts(handle_, 0, mode, nullptr, 0, &n)) || n == 0) { return out; }
        std::vector<tf_contact> raw((size_t)n);
        if (!note(tf_world_contacts(handle_, 0, mode, raw.data(), n, &n))) { return out; }
        for (const tf_contact& c : raw) {
            ContactInfo o;
            o.bodyA = bodyAt(c.body_a);
            o.bodyB = bodyAt(c.body_b);
            o.shapeA = shapeAt(c.shape_a);
            o.shapeB = shapeAt(c.shape_b);
            o.normal = Vec3{ c.normal[0], c.normal[1], c.normal[2] };
            o.friction = c.friction;
            o.restitution = c.restitution;
            o.rollingResistance = c.rolling_resistance;
            o.rollingImpulse = Vec3{ c.rolling_impulse[0], c.rolling_impulse[1], c.rolling_impulse[2] };
            o.pointCount = c.point_count;
            for (int i = 0; i < c.point_count && i < 4; ++i) {
                o.points[i] = Vec3{ c.points[i][0], c.points[i][1], c.points[i][2] };
                o.separations[i] = c.separations[i];
                o.normalImpulses[i] = c.normal_impulses[i];
                o.tangentImpulses[i] = Vec3{ c.tangent_impulses[i][0], c.tangent_impulses[i][1], c.tangent_impulses[i][2] };
            }
            out.push_back(o);
        }
        return out;
    }

    // Joints (tf_joint_create, tf_joint_get_info, tf_world_broken_joints). createJoint returns an invalid id
    // for bad bodies, as the reference does, and for what the C ABI refuses (status() tells which).
    JointId createJoint(const JointDesc& d) {
        tf_joint_desc c{};
        c.body_a = d.bodyA.index == UINT32_MAX ? tf_id{ UINT32_MAX, 0 } : tf_id{ d.bodyA.index, d.bodyA.generation };
        c.body_b = tf_id{ d.bodyB.index, d.bodyB.generation };
        c.collide_connected = d.collideConnected ? 1 : 0;
        c.break_force = d.breakForce;
        c.break_torque = d.breakTorque;
        c.length = -1.0f;
        auto put = [](float* o, const Vec3& v) { o[0] = v.x, o[1] = v.y, o[2] = v.z; };
        if (const PointJoint* k = std::get_if<PointJoint>(&d.kind)) {
            c.type = TF_JOINT_POINT;
            put(c.anchor, k->anchor);
        } else if (const FixedJoint* k = std::get_if<FixedJoint>(&d.kind)) {
            c.type = TF_JOINT_FIXED;
            put(c.anchor, k->anchor);
        } else if (const HingeJoint* k = std::get_if<HingeJoint>(&d.kind)) {
            c.type = TF_JOINT_HINGE;
            put(c.anchor, k->anchor);
            put(c.axis, k->axis);
            c.limited = k->limited ? 1 : 0;
            c.lower = k->lowerAngle;
            c.upper = k->upperAngle;
            c.motor_speed = k->motorSpeed;
            c.max_motor = k->maxMotorTorque;
            c.friction = k->frictionTorque;
        } else if (const SliderJoint* k = std::get_if<SliderJoint>(&d.kind)) {
            c.type = TF_JOINT_SLIDER;
            put(c.anchor, k->anchor);
            put(c.axis, k->axis);
            c.limited = k->limited ? 1 : 0;
            c.lower = k->lowerTranslation;
            c.upper = k->upperTranslation;
            c.motor_speed = k->motorSpeed;
            c.max_motor = k->maxMotorForce;
            c.friction = k->frictionForce;
        } else if (const DistanceJoint* k = std::get_if<DistanceJoint>(&d.kind)) {
            c.type = TF_JOINT_DISTANCE;
            put(c.anchor, k->anchorA);
            put(c.anchor_b, k->anchorB);
            c.length = k->length;
            c.hertz = k->hertz;
            c.damping_ratio = k->dampingRatio;
            c.limited = k->limited ? 1 : 0;
            c.lower = k->minDistance;
            c.upper = k->maxDistance;
        } else if (const SwingTwistJoint* k = std::get_if<SwingTwistJoint>(&d.kind)) {
            c.type = TF_JOINT_SWING_TWIST;
            put(c.anchor, k->anchor);
            put(c.axis, k->axis);
            put(c.normal, k->normal);
            c.swing_y = k->swingY;
            c.swing_z = k->swingZ;
            c.lower = k->lowerTwist;
            c.upper = k->upperTwist;
            c.friction = k->frictionTorque;
        }
        tf_id id{};
        if (!note(tf_joint_create(handle_, 0, &c, &id))) { return {}; }
        if (joints_.size() <= id.index) { joints_.resize((size_t)id.index + 1); }
        joints_[id.index] = JointId{ id.index, id.generation };
        if (jointEnds_.size() < 2 * joints_.size()) { jointEnds_.resize(2 * joints_.size(), UINT32_MAX); }
        jointEnds_[2 * id.index] = d.bodyA.index;
        jointEnds_[2 * id.index + 1] = d.bodyB.index;
        return joints_[id.index];
    }
    bool isValid(JointId joint) const { return joint.index < joints_.size() && joints_[joint.index] == joint; }
    void destroyJoint(JointId joint) {
        if (!isValid(joint) || !note(tf_joint_destroy(handle_, 0, tf_id{ joint.index, joint.generation }))) { return; }
        joints_[joint.index] = JointId{ UINT32_MAX, joint.generation + 1 };
    }
    void setJointLimits(JointId joint, bool limited, float lower, float upper) {
        if (isValid(joint)) { note(tf_joint_set_limits(handle_, 0, tf_id{ joint.index, joint.generation }, limited, lower, upper)); }
    }
    void setJointMotor(JointId joint, float speed, float maxForce) {
        if (isValid(joint)) { note(tf_joint_set_motor(handle_, 0, tf_id{ joint.index, joint.generation }, speed, maxForce)); }
    }
    void setJointSpring(JointId joint, float hertz, float dampingRatio) {
        if (isValid(joint)) { note(tf_joint_set_spring(handle_, 0, tf_id{ joint.index, joint.generation }, hertz, dampingRatio)); }
    }
    void setJointFriction(JointId joint, float maxFriction) {
        if (isValid(joint)) { note(tf_joint_set_friction(handle_, 0, tf_id{ joint.index, joint.generation }, maxFriction)); }
    }
    void setJointSwing(JointId joint, float swingY, float swingZ) {
        if (isValid(joint)) { note(tf_joint_set_swing(handle_, 0, tf_id{ joint.index, joint.generation }, swingY, swingZ)); }
    }
    void setJointBreakLimits(JointId joint, float force, float torque) {
        if (isValid(joint)) { note(tf_joint_set_break_limits(handle_, 0, tf_id{ joint.index, joint.generation }, force, torque)); }
    }
    JointInfo jointInfo(JointId joint) const {
        JointInfo info;
        if (!isValid(joint)) { return info; }
        tf_joint_info raw{};
        if (!note(tf_joint_get_info(handle_, 0, tf_id{ joint.index, joint.generation }, &raw))) { return info; }
        info.joint = joint;
        info.type = (JointType)raw.type;
        if (raw.body_a != UINT32_MAX) { info.bodyA = bodyAt(raw.body_a); }
        info.bodyB = bodyAt(raw.body_b);
        info.anchorA = Vec3{ raw.anchor_a[0], raw.anchor_a[1], raw.anchor_a[2] };
        info.anchorB = Vec3{ raw.anchor_b[0], raw.anchor_b[1], raw.anchor_b[2] };
        info.axis = Vec3{ raw.axis[0], raw.axis[1], raw.axis[2] };
        info.value = raw.value;
        info.force = Vec3{ raw.force[0], raw.force[1], raw.force[2] };
        info.torque = Vec3{ raw.torque[0], raw.torque[1], raw.torque[2] };
        info.broken = raw.broken != 0;
        return info;
    }
    // Every live joint's info, in index order.
    std::vector<JointInfo> joints() const {
        std::vector<JointInfo> out;
        for (const JointId& id : joints_) {
            if (id.index != UINT32_MAX) { out.push_back(jointInfo(id)); }
        }
        return out;
    }
    // Joints that broke in the last step, in index order.
    std::vector<JointId> brokenJoints() const {
        std::vector<JointId> out;
        int32_t n = 0;
        if (!note(tf_world_broken_joints(handle_, 0, nullptr, 0, &n)) || n == 0) { return out; }
        std::vector<tf_id> raw((size_t)n);
        if (!note(tf_world_broken_joints(handle_, 0, raw.data(), n, &n))) { return out; }
        for (const tf_id& id : raw) { out.push_back(JointId{ id.index, id.generation }); }
        return out;
    }

    // Events of the last step, ordered by shape index (tf_world_contact_events, tf_world_hit_events).
    const std::vector<ContactEvent>& contactEvents() const {
        contactEvents_.clear();
        int32_t n = 0;
        if (!note(tf_world_contact_events(handle_, 0, nullptr, 0, &n)) || n == 0) { return contactEvents_; }
        std::vector<tf_contact_event> raw((size_t)n);
        if (!note(tf_world_contact_events(handle_, 0, raw.data(), n, &n))) { return contactEvents_; }
        for (const tf_contact_event& e : raw) {
            contactEvents_.push_back(ContactEvent{ bodyAt(e.body_a), bodyAt(e.body_b), shapeAt(e.shape_a),
                                                   shapeAt(e.shape_b), e.begin != 0 });
        }
        return contactEvents_;
    }
    const std::vector<HitEvent>& hitEvents() const {
        hitEvents_.clear();
        int32_t n = 0;
        if (!note(tf_world_hit_events(handle_, 0, nullptr, 0, &n)) || n == 0) { return hitEvents_; }
        std::vector<tf_hit_event> raw((size_t)n);
        if (!note(tf_world_hit_events(handle_, 0, raw.data(), n, &n))) { return hitEvents_; }
        for (const tf_hit_event& e : raw) {
            HitEvent h;
            h.bodyA = bodyAt(e.body_a);
            h.bodyB = bodyAt(e.body_b);
            h.shapeA = shapeAt(e.shape_a);
            h.shapeB = shapeAt(e.shape_b);
            h.point = Vec3{ e.point[0], e.point[1], e.point[2] };
            h.normal = Vec3{ e.normal[0], e.normal[1], e.normal[2] };
            h.speed = e.speed;
            hitEvents_.push_back(h);
        }
        return hitEvents_;
    }

    // The last C ABI status and its message; TF_OK after calls that succeeded.
    int status() const { return status_; }
    std::string statusMessage() const { return status_ == TF_OK ? std::string() : std::string(tf_last_error()); }
    // The C ABI handle, for calls this class does not wrap (batched stepping, launch shapes, profiling).
    void* handle() const { return handle_; }

private:
    static void put3(float* o, const Vec3& v) { o[0] = v.x, o[1] = v.y, o[2] = v.z; }
    static void put4(float* o, const Quat& q) { o[0] = q.x, o[1] = q.y, o[2] = q.z, o[3] = q.w; }

    static tf_settings toC(const WorldSettings& s) {
        tf_settings c{};
        put3(c.gravity, s.gravity);
        c.length_unit = s.lengthUnit;
        c.substeps = s.substeps;
        c.contact_hertz = s.contactHertz;
        c.contact_damping_ratio = s.contactDampingRatio;
        c.max_pushout_speed = s.maxPushoutSpeed;
        c.max_linear_speed = s.maxLinearSpeed;
        c.max_angular_speed = s.maxAngularSpeed;
        c.restitution_threshold = s.restitutionThreshold;
        c.hit_threshold = s.hitThreshold;
        c.sleep_threshold = s.sleepThreshold;
        c.time_to_sleep = s.timeToSleep;
        c.contact_reuse_distance = s.contactReuseDistance;
        c.contact_reuse_angle = s.contactReuseAngle;
        c.joint_hertz = s.jointHertz;
        c.joint_damping_ratio = s.jointDampingRatio;
        c.continuous = s.continuous ? 1 : 0;
        return c;
    }

    bool note(int rc) const {
        status_ = rc;
        return rc == TF_OK;
    }

    void state(BodyId body, Transform& t, Vec3& v, Vec3& w) const {
        if (!isValid(body)) { return; }
        float p[3] = {}, q[4] = { 0, 0, 0, 1 }, lv[3] = {}, av[3] = {};
        if (!note(tf_body_get_state(handle_, 0, tf_id{ body.index, body.generation }, p, q, lv, av))) { return; }
        t.p = Vec3{ p[0], p[1], p[2] };
        t.q = Quat{ q[0], q[1], q[2], q[3] };
        v = Vec3{ lv[0], lv[1], lv[2] };
        w = Vec3{ av[0], av[1], av[2] };
    }

    void setVelocities(BodyId body, const Vec3* v, const Vec3* w) {
        if (!isValid(body)) { return; }
        float a[3], b[3];
        if (v) { put3(a, *v); }
        if (w) { put3(b, *w); }
        note(tf_body_set_velocity(handle_, 0, cid(body), v ? a : nullptr, w ? b : nullptr));
    }

    static tf_id cid(BodyId b) { return tf_id{ b.index, b.generation }; }
    static tf_id cid(ShapeId s) { return tf_id{ s.index, s.generation }; }

    BodyId bodyAt(uint32_t i) const { return i < bodies_.size() ? bodies_[i] : BodyId{}; }
    ShapeId shapeAt(uint32_t i) const { return i < shapes_.size() ? shapes_[i] : ShapeId{}; }

    void* handle_ = nullptr;
    WorldSettings settings_;
    StepProfile profile_;
    std::vector<BodyId> bodies_;
    std::vector<ShapeId> shapes_;
    std::vector<JointId> joints_;
    std::vector<uint32_t> shapeOwner_;  // each shape slot's body
    std::vector<uint32_t> jointEnds_;   // each joint slot's bodies (UINT32_MAX for the world)
    std::map<const TriangleMesh*, int32_t> meshIds_;           // meshes this handle has built, by mesh
    std::vector<std::shared_ptr<const TriangleMesh>> meshes_;  // kept alive while their ids are in use
    mutable int status_ = TF_OK;
    mutable std::vector<ContactEvent> contactEvents_;
    mutable std::vector<HitEvent> hitEvents_;
};

}  // namespace twofold
