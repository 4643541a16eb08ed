// Test infrastructure only: the oracle side of every parity check. Only tests/, the smoke check and the
// CPU-baseline leg of bench.py load the library this file builds into.
//
// It compiles the unmodified AnvilFx/twofold sources (src/*.cpp, include/twofold/*.h) and wraps one
// reference World per handle behind the same plain-C descriptors the B200 library takes
// (include/twofold_b200.h), so both sides are built from identical inputs. src/world.cpp is compiled as
// part of this translation unit, so the harness can read World::Impl state that the public API hides:
// the sorted candidate keys (src/world.cpp:868-870) and each contact's clipped feature
// (src/internal.h:482-488).
#include <atomic>
#include <cstring>
#include <thread>
#include <vector>

// World::impl_ is private in include/twofold/world.h:507-509. The harness reads it, so the class is
// seen with public members in this translation unit only.
#define private public
#include "world.cpp"
#include "twofold/hull.h"
#undef private

#include "twofold_b200.h"

using namespace twofold;

namespace {

WorldSettings toSettings(const tf_settings* s) {
    WorldSettings w;
    if (!s) { return w; }
    w.gravity = { s->gravity[0], s->gravity[1], s->gravity[2] };
    w.lengthUnit = s->length_unit;
    w.substeps = s->substeps;
    w.contactHertz = s->contact_hertz;
    w.contactDampingRatio = s->contact_damping_ratio;
    w.maxPushoutSpeed = s->max_pushout_speed;
    w.maxLinearSpeed = s->max_linear_speed;
    w.maxAngularSpeed = s->max_angular_speed;
    w.restitutionThreshold = s->restitution_threshold;
    w.hitThreshold = s->hit_threshold;
    w.sleepThreshold = s->sleep_threshold;
    w.timeToSleep = s->time_to_sleep;
    w.contactReuseDistance = s->contact_reuse_distance;
    w.contactReuseAngle = s->contact_reuse_angle;
    w.jointHertz = s->joint_hertz;
    w.jointDampingRatio = s->joint_damping_ratio;
    w.continuous = s->continuous != 0;
    return w;
}

// TriangleMeshes made through ref_mesh_create, named by position; they live until the process ends.
std::vector<std::shared_ptr<const TriangleMesh>>& meshRegistry() {
    static std::vector<std::shared_ptr<const TriangleMesh>> r;
    return r;
}

Vec3 v3(const float* p) { return { p[0], p[1], p[2] }; }
Quat q4(const float* p) { return { p[0], p[1], p[2], p[3] }; }

BodyDesc toBody(const tf_body_desc* d) {
    BodyDesc b;
    b.type = (MotionType)d->type;
    b.position = v3(d->position);
    b.rotation = q4(d->rotation);
    b.linearVelocity = v3(d->linear_velocity);
    b.angularVelocity = v3(d->angular_velocity);
    b.linearDamping = d->linear_damping;
    b.angularDamping = d->angular_damping;
    b.gravityScale = d->gravity_scale;
    b.locks = (uint8_t)d->locks;
    b.lockFrame = q4(d->lock_frame);
    b.awake = d->awake != 0;
    b.canSleep = d->can_sleep != 0;
    return b;
}

bool toShape(const tf_shape_desc* d, ShapeDesc& s) {
    switch (d->geometry) {
    case TF_SPHERE: s.geometry = Sphere{ d->radius }; break;
    case TF_BOX: s.geometry = Box{ v3(d->half_extents) }; break;
    case TF_CYLINDER: s.geometry = Cylinder{ d->radius, d->half_height }; break;
    case TF_PRISM: {
        Prism p;
        for (int i = 0; i < d->point_count; ++i) { p.polygon.push_back({ d->points[2 * i], d->points[2 * i + 1] }); }
        p.zMin = d->z_min;
        p.zMax = d->z_max;
        s.geometry = p;
        break;
    }
    case TF_HULL: {
        Hull h;
        for (int i = 0; i < d->point_count; ++i) { h.points.push_back(v3(d->points + 3 * i)); }
        h.maxVertices = d->max_vertices;
        s.geometry = h;
        break;
    }
    case TF_HALFSPACE: s.geometry = HalfSpace{}; break;
    case TF_MESH:
        if (d->mesh < 0 || (size_t)d->mesh >= meshRegistry().size()) { return false; }
        s.geometry = Mesh{ meshRegistry()[(size_t)d->mesh] };
        break;
    default: return false;
    }
    s.position = v3(d->position);
    s.rotation = q4(d->rotation);
    s.density = d->density;
    s.friction = d->friction;
    s.restitution = d->restitution;
    s.rollingResistance = d->rolling_resistance;
    s.category = d->category;
    s.mask = d->mask;
    s.sensor = d->sensor != 0;
    return true;
}

void put3(float* o, const Vec3& v) {
    if (!o) { return; }
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
}

void put4(float* o, const Quat& q) {
    if (!o) { return; }
    o[0] = q.x;
    o[1] = q.y;
    o[2] = q.z;
    o[3] = q.w;
}

World* W(void* h) { return static_cast<World*>(h); }

}

extern "C" {

TF_API int ref_mesh_create(const float* vertices, int nv, const uint32_t* indices, int ni) {
    std::vector<Vec3> v((size_t)nv);
    for (int i = 0; i < nv; ++i) { v[(size_t)i] = { vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2] }; }
    meshRegistry().push_back(std::make_shared<const TriangleMesh>(v, std::vector<uint32_t>(indices, indices + ni)));
    return (int)meshRegistry().size() - 1;
}

// The built mesh, laid out as tf_mesh_read lays out its own.
TF_API int ref_mesh_read(int mesh, int32_t counts[3], float* vertices, uint32_t* indices, float* normals,
                         uint8_t* edges, float* node_bounds, int32_t* node_ranges) {
    if (mesh < 0 || (size_t)mesh >= meshRegistry().size()) { return -1; }
    const TriangleMesh::Data& d = meshRegistry()[(size_t)mesh]->data();
    counts[0] = (int32_t)d.vertices.size();
    counts[1] = (int32_t)d.normals.size();
    counts[2] = (int32_t)d.nodes.size();
    for (size_t i = 0; i < d.vertices.size(); ++i) { put3(vertices ? vertices + 3 * i : nullptr, d.vertices[i]); }
    if (indices) { std::memcpy(indices, d.indices.data(), d.indices.size() * sizeof(uint32_t)); }
    for (size_t t = 0; t < d.normals.size(); ++t) {
        put3(normals ? normals + 3 * t : nullptr, d.normals[t]);
        if (edges) { edges[t] = d.edges[t]; }
    }
    for (size_t n = 0; n < d.nodes.size(); ++n) {
        put3(node_bounds ? node_bounds + 6 * n : nullptr, d.nodes[n].lo);
        put3(node_bounds ? node_bounds + 6 * n + 3 : nullptr, d.nodes[n].hi);
        if (node_ranges) {
            node_ranges[2 * n] = d.nodes[n].first;
            node_ranges[2 * n + 1] = d.nodes[n].count;
        }
    }
    return 0;
}

// computeHull, laid out as tf_hull_compute lays out its own.
TF_API int ref_hull_compute(const float* points, int32_t count, int32_t max_vertices, int32_t counts[2], float* vertices,
                            int32_t vertex_capacity, int32_t* faces, int32_t face_capacity) {
    std::vector<Vec3> cloud((size_t)count);
    for (int32_t i = 0; i < count; ++i) { cloud[i] = { points[3 * i], points[3 * i + 1], points[3 * i + 2] }; }
    const HullMesh h = computeHull(cloud, max_vertices);
    int32_t words = 0;
    for (const auto& f : h.faces) { words += 1 + (int32_t)f.size(); }
    counts[0] = (int32_t)h.vertices.size();
    counts[1] = words;
    if (vertices && vertex_capacity >= counts[0]) {
        for (size_t i = 0; i < h.vertices.size(); ++i) { put3(vertices + 3 * i, h.vertices[i]); }
    }
    if (faces && face_capacity >= words) {
        int32_t at = 0;
        for (const auto& f : h.faces) {
            faces[at++] = (int32_t)f.size();
            for (int v : f) { faces[at++] = v; }
        }
    }
    return 0;
}

TF_API void* ref_world_create(const tf_settings* s) { return new World(toSettings(s)); }
TF_API void* ref_world_copy(void* h) { return new World(*W(h)); }
TF_API void ref_world_destroy(void* h) { delete W(h); }

TF_API int ref_body_create(void* h, const tf_body_desc* d, tf_id* out) {
    const BodyId id = W(h)->createBody(toBody(d));
    out->index = id.index;
    out->generation = id.generation;
    return 0;
}

TF_API int ref_shape_add(void* h, tf_id body, const tf_shape_desc* d, tf_id* out) {
    ShapeDesc s;
    if (!toShape(d, s)) { return -1; }
    const ShapeId id = W(h)->addShape({ body.index, body.generation }, s);
    out->index = id.index;
    out->generation = id.generation;
    return 0;
}

// Bulk scene build: n bodies, then shapes onto body_of[i] (an index into the bodies just made).
TF_API int ref_scene_build(void* h, int nb, const tf_body_desc* bodies, int ns, const uint32_t* body_of,
                           const tf_shape_desc* shapes) {
    std::vector<BodyId> ids((size_t)nb);
    for (int i = 0; i < nb; ++i) { ids[(size_t)i] = W(h)->createBody(toBody(&bodies[i])); }
    for (int i = 0; i < ns; ++i) {
        ShapeDesc s;
        if (!toShape(&shapes[i], s)) { return -1; }
        W(h)->addShape(ids[body_of[i]], s);
    }
    return 0;
}

TF_API int ref_world_step(void* h, float dt, int n) {
    for (int i = 0; i < n; ++i) { W(h)->step(dt); }
    return 0;
}

TF_API int ref_body_count(void* h) { return (int)W(h)->impl_->bodies.size(); }

// Every body slot in index order; dead slots read as zeros.
TF_API int ref_world_get_states(void* h, float* p, float* q, float* v, float* w, int32_t* awake) {
    const auto& bodies = W(h)->impl_->bodies;
    for (size_t i = 0; i < bodies.size(); ++i) {
        const Body& b = bodies[i];
        put3(p ? p + 3 * i : nullptr, b.xf.p);
        put4(q ? q + 4 * i : nullptr, b.xf.q);
        put3(v ? v + 3 * i : nullptr, b.v);
        put3(w ? w + 3 * i : nullptr, b.w);
        if (awake) { awake[i] = b.awake ? 1 : 0; }
    }
    return (int)bodies.size();
}

TF_API int ref_body_set_velocity(void* h, tf_id body, const float* v, const float* w) {
    W(h)->setLinearVelocity({ body.index, body.generation }, v3(v));
    W(h)->setAngularVelocity({ body.index, body.generation }, v3(w));
    return 0;
}

// The World calls between steps through the public API; `what` numbers them as twofold_b200.world.CALLS does.
TF_API int ref_world_call(void* h, int what, tf_id id, const float* v, uint32_t a, uint32_t b) {
    World& w = *W(h);
    const BodyId body{ id.index, id.generation };
    const ShapeId shape{ id.index, id.generation };
    switch (what) {
        case 0: w.destroyBody(body); break;
        case 1: w.removeShape(shape); break;
        case 2: w.setFriction(shape, v[0]); break;
        case 3: w.setRestitution(shape, v[0]); break;
        case 4: w.setRollingResistance(shape, v[0]); break;
        case 5: w.setFilter(shape, a, b); break;
        case 6: w.setTransform(body, v3(v), Quat(v[3], v[4], v[5], v[6])); break;
        case 7: w.setKinematicTarget(body, v3(v), Quat(v[3], v[4], v[5], v[6]), v[7]); break;
        case 8: w.setMotionType(body, (MotionType)a); break;
        case 9: w.addForce(body, v3(v), a != 0); break;
        case 10: w.addForceAtPoint(body, v3(v), v3(v + 3), a != 0); break;
        case 11: w.addTorque(body, v3(v), a != 0); break;
        case 12: w.addImpulse(body, v3(v), a != 0); break;
        case 13: w.addImpulseAtPoint(body, v3(v), v3(v + 3), a != 0); break;
        case 14: w.setDamping(body, v[0], v[1]); break;
        case 15: w.setGravityScale(body, v[0]); break;
        case 16: w.wake(body); break;
        case 17: w.sleep(body); break;
        case 18: w.setCanSleep(body, a != 0); break;
        case 19: w.setLinearVelocity(body, v3(v)); break;
        case 20: w.setAngularVelocity(body, v3(v)); break;
        default: return -1;
    }
    return 0;
}

TF_API int ref_body_get_mass(void* h, tf_id body, float* mass, float* center, float* inertia) {
    const MassProperties m = W(h)->massProperties({ body.index, body.generation });
    *mass = m.mass;
    put3(center, m.center);
    for (int r = 0; r < 3; ++r) { put3(inertia + 3 * r, m.inertia.r[r]); }
    return 0;
}

TF_API int ref_world_candidates(void* h, uint64_t* out, int cap, int* count) {
    const auto& c = W(h)->impl_->candidatePairs;
    *count = (int)c.size();
    for (size_t i = 0; i < c.size() && (int)i < cap; ++i) { out[i] = c[i]; }
    return 0;
}

// The internal contact list in (key, part) order. mode 0: touching only (as World::contacts()),
// 1: every contact not removed, 2: the raw list.
TF_API int ref_world_contacts(void* h, int mode, tf_contact* out, int cap, int* count) {
    const World::Impl& w = *W(h)->impl_;
    int n = 0;
    for (const Contact& c : w.contacts) {
        if (mode < 2 && (c.removed || (mode == 0 && !c.touching()))) { continue; }
        if (n < cap) {
            tf_contact& o = out[n];
            std::memset(&o, 0, sizeof(o));
            o.key = c.key;
            o.part = c.part;
            o.shape_a = c.shapeA;
            o.shape_b = c.shapeB;
            o.body_a = c.bodyA;
            o.body_b = c.bodyB;
            o.point_count = c.count;
            o.feature_kind = (int)c.feature.kind;
            o.feature_a = c.feature.a;
            o.feature_b = c.feature.b;
            put3(o.normal, c.normal);
            o.friction = c.friction;
            o.restitution = c.restitution;
            o.rolling_resistance = c.rollingResistance;
            put3(o.rolling_impulse, c.rollingImpulse);
            for (int i = 0; i < c.count; ++i) {
                put3(o.points[i], w.bodies[c.bodyA].xf.apply(c.points[i].localA));
                o.separations[i] = c.points[i].separation;
                o.normal_impulses[i] = c.points[i].normalImpulse;
                put3(o.tangent_impulses[i], c.points[i].tangentImpulse);
            }
        }
        ++n;
    }
    *count = n;
    return 0;
}

// World::createJoint from the library's joint descriptor, as the library reads it (tf_joint_desc).
TF_API int ref_joint_create(void* h, const tf_joint_desc* d, tf_id* out) {
    JointDesc jd;
    if (d->body_a.index != UINT32_MAX) { jd.bodyA = BodyId{ d->body_a.index, d->body_a.generation }; }
    jd.bodyB = BodyId{ d->body_b.index, d->body_b.generation };
    jd.collideConnected = d->collide_connected != 0;
    jd.breakForce = d->break_force;
    jd.breakTorque = d->break_torque;
    const Vec3 anchor{ d->anchor[0], d->anchor[1], d->anchor[2] };
    const Vec3 axis{ d->axis[0], d->axis[1], d->axis[2] };
    switch (d->type) {
        case TF_JOINT_POINT: jd.kind = PointJoint{ anchor }; break;
        case TF_JOINT_FIXED: jd.kind = FixedJoint{ anchor }; break;
        case TF_JOINT_HINGE: {
            HingeJoint k;
            k.anchor = anchor;
            k.axis = axis;
            k.limited = d->limited != 0;
            k.lowerAngle = d->lower;
            k.upperAngle = d->upper;
            k.motorSpeed = d->motor_speed;
            k.maxMotorTorque = d->max_motor;
            k.frictionTorque = d->friction;
            jd.kind = k;
            break;
        }
        case TF_JOINT_SLIDER: {
            SliderJoint k;
            k.anchor = anchor;
            k.axis = axis;
            k.limited = d->limited != 0;
            k.lowerTranslation = d->lower;
            k.upperTranslation = d->upper;
            k.motorSpeed = d->motor_speed;
            k.maxMotorForce = d->max_motor;
            k.frictionForce = d->friction;
            jd.kind = k;
            break;
        }
        case TF_JOINT_DISTANCE: {
            DistanceJoint k;
            k.anchorA = anchor;
            k.anchorB = Vec3{ d->anchor_b[0], d->anchor_b[1], d->anchor_b[2] };
            k.length = d->length;
            k.hertz = d->hertz;
            k.dampingRatio = d->damping_ratio;
            k.limited = d->limited != 0;
            k.minDistance = d->lower;
            k.maxDistance = d->upper;
            jd.kind = k;
            break;
        }
        default: {
            SwingTwistJoint k;
            k.anchor = anchor;
            k.axis = axis;
            k.normal = Vec3{ d->normal[0], d->normal[1], d->normal[2] };
            k.swingY = d->swing_y;
            k.swingZ = d->swing_z;
            k.lowerTwist = d->lower;
            k.upperTwist = d->upper;
            k.frictionTorque = d->friction;
            jd.kind = k;
            break;
        }
    }
    const JointId id = W(h)->createJoint(jd);
    out->index = id.index;
    out->generation = id.generation;
    return id.index == UINT32_MAX ? -1 : 0;
}

// The joint setters and destroyJoint through the public API; `what` and v as tf_joint_set_* take them.
TF_API int ref_joint_set(void* h, tf_id joint, int what, const float* v) {
    const JointId id{ joint.index, joint.generation };
    switch (what) {
        case 0: W(h)->setJointLimits(id, v[0] != 0.0f, v[1], v[2]); break;
        case 1: W(h)->setJointMotor(id, v[0], v[1]); break;
        case 2: W(h)->setJointSpring(id, v[0], v[1]); break;
        case 3: W(h)->setJointFriction(id, v[0]); break;
        case 4: W(h)->setJointSwing(id, v[0], v[1]); break;
        case 5: W(h)->setJointBreakLimits(id, v[0], v[1]); break;
        case 6: W(h)->destroyJoint(id); break;
        default: return -1;
    }
    return 0;
}

TF_API int ref_joint_info(void* h, tf_id joint, tf_joint_info* out) {
    const JointInfo info = W(h)->jointInfo(JointId{ joint.index, joint.generation });
    std::memset(out, 0, sizeof(*out));
    out->type = (int32_t)info.type;
    out->body_a = info.bodyA.index;
    out->body_b = info.bodyB.index;
    put3(out->anchor_a, info.anchorA);
    put3(out->anchor_b, info.anchorB);
    put3(out->axis, info.axis);
    out->value = info.value;
    put3(out->force, info.force);
    put3(out->torque, info.torque);
    out->broken = info.broken ? 1 : 0;
    return 0;
}

TF_API int ref_broken_joints(void* h, tf_id* out, int cap, int* count) {
    const std::vector<JointId> ids = W(h)->brokenJoints();
    *count = (int)ids.size();
    for (size_t i = 0; out && i < ids.size() && (int)i < cap; ++i) { out[i] = { ids[i].index, ids[i].generation }; }
    return 0;
}

// World::contactEvents() and World::hitEvents() of the last step, through the public API, as the library's
// tf_world_contact_events and tf_world_hit_events lay them out.
TF_API int ref_world_contact_events(void* h, tf_contact_event* out, int cap, int* count) {
    const std::vector<ContactEvent>& ev = W(h)->contactEvents();
    *count = (int)ev.size();
    for (size_t i = 0; out && i < ev.size() && (int)i < cap; ++i) {
        out[i].shape_a = ev[i].shapeA.index;
        out[i].shape_b = ev[i].shapeB.index;
        out[i].body_a = ev[i].bodyA.index;
        out[i].body_b = ev[i].bodyB.index;
        out[i].begin = ev[i].begin ? 1 : 0;
    }
    return 0;
}

TF_API int ref_world_hit_events(void* h, tf_hit_event* out, int cap, int* count) {
    const std::vector<HitEvent>& ev = W(h)->hitEvents();
    *count = (int)ev.size();
    for (size_t i = 0; out && i < ev.size() && (int)i < cap; ++i) {
        out[i].shape_a = ev[i].shapeA.index;
        out[i].shape_b = ev[i].shapeB.index;
        out[i].body_a = ev[i].bodyA.index;
        out[i].body_b = ev[i].bodyB.index;
        put3(out[i].point, ev[i].point);
        put3(out[i].normal, ev[i].normal);
        out[i].speed = ev[i].speed;
    }
    return 0;
}

TF_API int ref_world_profile(void* h, tf_profile* out) {
    const StepProfile& p = W(h)->profile();
    out->total = p.total;
    out->broadphase = p.broadphase;
    out->narrowphase = p.narrowphase;
    out->solver = p.solver;
    out->continuous = p.continuous;
    out->sleep = p.sleep;
    out->candidate_pairs = p.candidatePairs;
    out->swept_pairs = p.sweptPairs;
    out->impacts = p.impacts;
    out->manifolds = p.manifolds;
    out->touching_contacts = p.touchingContacts;
    out->awake_bodies = p.awakeBodies;
    out->awake_islands = p.awakeIslands;
    return 0;
}

TF_API int ref_awake_dynamic(void* h) {
    int n = 0;
    for (const Body& b : W(h)->impl_->bodies) { n += (b.alive && b.type == MotionType::Dynamic && b.awake) ? 1 : 0; }
    return n;
}

// Steps n independent worlds `steps` times each: every world is stepped start to finish by one thread
// taken from a pool of `threads`, worlds handed out in order as threads come free. Writes the awake
// dynamic body count summed over every step of every world to body_steps.
TF_API int ref_worlds_step_parallel(void** worlds, int n, float dt, int steps, int threads, int64_t* body_steps) {
    std::atomic<int> next{ 0 };
    std::atomic<int64_t> total{ 0 };
    auto work = [&] {
        int64_t mine = 0;
        for (int i = next++; i < n; i = next++) {
            World* w = W(worlds[i]);
            for (int s = 0; s < steps; ++s) {
                w->step(dt);
                mine += w->profile().awakeBodies;
            }
        }
        total += mine;
    };
    if (threads <= 1) {
        work();
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t) { pool.emplace_back(work); }
        for (std::thread& t : pool) { t.join(); }
    }
    if (body_steps) { *body_steps = total.load(); }
    return 0;
}

TF_API int ref_hardware_threads(void) { return (int)std::thread::hardware_concurrency(); }

}
