/*
 * twofold_b200 — C ABI of the B200 contact pipeline behind twofold::World::step.
 *
 * One tf_world holds one or more independent worlds ("a batch"). A plain world is a batch of one.
 * Every world has its own body and shape index spaces, numbered from 0 in creation order with freed
 * slots reused under a bumped generation, exactly as the reference World numbers them
 * (src/world.cpp:1751-1782 createBody, :1820-1857 addShape). Handles are {index, generation}.
 *
 * Conventions
 *   - Plain C types, host pointers, caller-owned buffers. No C++ or torch types cross this boundary.
 *   - Every entry point returns an int status: TF_OK (0) or a negative TF_E* code. tf_last_error()
 *     gives a one-line message for the calling thread's last failure.
 *   - Invalid handles follow the reference's convention (src/world.cpp:352-371): getters fill zeros,
 *     setters do nothing; they are not errors.
 *   - tf_world_step with dt <= 0 or non-finite dt does nothing (src/world.cpp:1565).
 *   - Device state lives in a library-owned arena on the device chosen at creation. State reads
 *     (tf_body_get_*) copy back on demand.
 *
 * Reference interface each group replaces (paths inside AnvilFx/twofold):
 *   tf_settings        <- WorldSettings            include/twofold/world.h:216-241
 *   tf_body_desc       <- BodyDesc                 include/twofold/world.h:108-123
 *   tf_shape_desc      <- ShapeDesc + Geometry     include/twofold/world.h:51-106
 *   tf_world_create    <- World::World             include/twofold/world.h:364
 *   tf_body_create     <- World::createBody        include/twofold/world.h:381
 *   tf_shape_add       <- World::addShape          include/twofold/world.h:386
 *   tf_world_step      <- World::step              include/twofold/world.h:378
 *   tf_body_get_state  <- World::transform/linearVelocity/angularVelocity  world.h:404-411
 *   tf_world_contacts  <- World::contacts          include/twofold/world.h:473
 *   tf_world_profile   <- World::profile           include/twofold/world.h:379
 */
#ifndef TWOFOLD_B200_H
#define TWOFOLD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define TF_API __declspec(dllexport)
#else
#define TF_API __attribute__((visibility("default")))
#endif

#define TF_ABI_VERSION 1

enum tf_status {
    TF_OK = 0,
    TF_E_INVALID = -1,   /* bad argument (null pointer, out-of-range world, bad enum) */
    TF_E_CUDA = -2,      /* a CUDA call failed; the message names it */
    TF_E_CAPACITY = -3,  /* a device buffer overflowed and could not be grown */
    TF_E_NUMERIC = -4,   /* the step produced a non-finite body state */
    TF_E_TIMEOUT = -5,   /* a bounded device wait ran out */
    TF_E_UNSUPPORTED = -6 /* the scene uses a feature this build does not run on the device */
};

/* Device-side error bits, as returned by tf_world_device_status. */
enum tf_device_flags {
    TF_DEV_PAIR_OVERFLOW = 1u << 0,
    TF_DEV_CONTACT_OVERFLOW = 1u << 1,
    TF_DEV_NONFINITE = 1u << 2,
    TF_DEV_TIMEOUT = 1u << 3,
    TF_DEV_UNSUPPORTED_PAIR = 1u << 4,
    TF_DEV_CONTINUOUS_SKIPPED = 1u << 5, /* not set: the continuous pass runs on the device */
    TF_DEV_LIST_OVERFLOW = 1u << 6
};

enum tf_motion_type { TF_STATIC = 0, TF_KINEMATIC = 1, TF_DYNAMIC = 2 };

enum tf_lock_flags {
    TF_LOCK_TRANSLATION_X = 1 << 0,
    TF_LOCK_TRANSLATION_Y = 1 << 1,
    TF_LOCK_TRANSLATION_Z = 1 << 2,
    TF_LOCK_ROTATION_X = 1 << 3,
    TF_LOCK_ROTATION_Y = 1 << 4,
    TF_LOCK_ROTATION_Z = 1 << 5,
    TF_LOCK_PLANAR = (1 << 2) | (1 << 3) | (1 << 4)
};

enum tf_geometry { TF_SPHERE = 0, TF_BOX = 1, TF_CYLINDER = 2, TF_PRISM = 3, TF_HULL = 4, TF_HALFSPACE = 5, TF_MESH = 6 };

typedef struct tf_id {
    uint32_t index;
    uint32_t generation;
} tf_id;

/* WorldSettings, field for field (include/twofold/world.h:216-241). */
typedef struct tf_settings {
    float gravity[3];
    float length_unit;
    int32_t substeps;
    float contact_hertz;
    float contact_damping_ratio;
    float max_pushout_speed;
    float max_linear_speed;
    float max_angular_speed;
    float restitution_threshold;
    float hit_threshold;
    float sleep_threshold;
    float time_to_sleep;
    float contact_reuse_distance;
    float contact_reuse_angle;
    float joint_hertz;
    float joint_damping_ratio;
    int32_t continuous;
} tf_settings;

/* BodyDesc (include/twofold/world.h:108-123). Quaternions are x, y, z, w. */
typedef struct tf_body_desc {
    int32_t type;
    float position[3];
    float rotation[4];
    float linear_velocity[3];
    float angular_velocity[3];
    float linear_damping;
    float angular_damping;
    float gravity_scale;
    uint32_t locks;
    float lock_frame[4];
    int32_t awake;
    int32_t can_sleep;
} tf_body_desc;

/* ShapeDesc plus its Geometry alternative (include/twofold/world.h:51-106).
 *   TF_SPHERE: radius.  TF_BOX: half_extents.  TF_CYLINDER: radius, half_height.
 *   TF_PRISM: points = point_count (x, y) pairs, z_min, z_max.
 *   TF_HULL: points = point_count (x, y, z) triples, max_vertices.
 *   TF_HALFSPACE: no parameters (static bodies only).
 *   TF_MESH: mesh = an id from tf_mesh_create (static and kinematic bodies only).
 * points is read during tf_shape_add only. */
typedef struct tf_shape_desc {
    int32_t geometry;
    float radius;
    float half_extents[3];
    float half_height;
    const float* points;
    int32_t point_count;
    int32_t max_vertices;
    float z_min;
    float z_max;
    float position[3];
    float rotation[4];
    float density;
    float friction;
    float restitution;
    float rolling_resistance;
    uint32_t category;
    uint32_t mask;
    int32_t sensor;
    int32_t mesh;
} tf_shape_desc;

/* StepProfile (include/twofold/world.h:346-360). Times are device milliseconds per phase. */
typedef struct tf_profile {
    float total;
    float broadphase;
    float narrowphase;
    float solver;
    float continuous;
    float sleep;
    int32_t candidate_pairs;
    int32_t swept_pairs;
    int32_t impacts;
    int32_t manifolds;
    int32_t touching_contacts;
    int32_t awake_bodies;
    int32_t awake_islands;
} tf_profile;

/* One contact of World::contacts (ContactInfo, include/twofold/world.h:252-266) plus the
 * pair key, part and clipped feature the parity tests compare. */
typedef struct tf_contact {
    uint64_t key;
    uint32_t part;
    uint32_t shape_a, shape_b;
    uint32_t body_a, body_b;
    int32_t point_count;
    int32_t feature_kind; /* 0 none, 1 face of A, 2 face of B, 3 edge pair */
    int32_t feature_a, feature_b;
    float normal[3];
    float friction, restitution, rolling_resistance;
    float rolling_impulse[3];
    float points[4][3];
    float separations[4];
    float normal_impulses[4];
    float tangent_impulses[4][3];
} tf_contact;

/* JointType (include/twofold/world.h:202). */
enum tf_joint_type {
    TF_JOINT_POINT = 0, TF_JOINT_FIXED = 1, TF_JOINT_HINGE = 2, TF_JOINT_SLIDER = 3, TF_JOINT_DISTANCE = 4,
    TF_JOINT_SWING_TWIST = 5
};

/* JointDesc plus its JointKind alternative (include/twofold/world.h:132-214), in world space at the bodies'
 * current poses. body_a with index UINT32_MAX joins body B to the world.
 *   every kind: anchor (a distance joint's anchorA), collide_connected, break_force, break_torque
 *               (infinity for none).
 *   TF_JOINT_HINGE:  axis, limited, lower/upper angle, motor_speed, max_motor (torque), friction (torque).
 *   TF_JOINT_SLIDER: axis, limited, lower/upper translation, motor_speed, max_motor (force), friction (force).
 *   TF_JOINT_DISTANCE: anchor_b, length (negative: the distance the anchors start at), hertz, damping_ratio,
 *               limited, lower/upper = minDistance/maxDistance.
 *   TF_JOINT_SWING_TWIST: axis, normal, swing_y, swing_z, lower/upper twist, friction (torque). */
typedef struct tf_joint_desc {
    int32_t type;
    tf_id body_a;
    tf_id body_b;
    float anchor[3];
    float anchor_b[3];
    float axis[3];
    float normal[3];
    int32_t limited;
    float lower;
    float upper;
    float motor_speed;
    float max_motor;
    float friction;
    float length;
    float hertz;
    float damping_ratio;
    float swing_y;
    float swing_z;
    int32_t collide_connected;
    float break_force;
    float break_torque;
} tf_joint_desc;

/* JointInfo (include/twofold/world.h:300-316) with world-local body indices (body_a UINT32_MAX: the world). */
typedef struct tf_joint_info {
    int32_t type;
    uint32_t body_a, body_b;
    float anchor_a[3];
    float anchor_b[3];
    float axis[3];
    float value;
    float force[3];
    float torque[3];
    int32_t broken;
} tf_joint_info;

/* ContactEvent (include/twofold/world.h:269-276) with world-local indices. */
typedef struct tf_contact_event {
    uint32_t shape_a, shape_b;
    uint32_t body_a, body_b;
    int32_t begin;
} tf_contact_event;

/* HitEvent (include/twofold/world.h:278-288) with world-local indices. */
typedef struct tf_hit_event {
    uint32_t shape_a, shape_b;
    uint32_t body_a, body_b;
    float point[3];
    float normal[3];
    float speed;
} tf_hit_event;

TF_API int tf_abi_version(void);
TF_API const char* tf_last_error(void);
TF_API void tf_default_settings(tf_settings* out);

/* Creates n_worlds empty worlds sharing settings on CUDA device `device`. */
TF_API int tf_world_create(const tf_settings* settings, int32_t n_worlds, int32_t device, void** out_world);
TF_API int tf_world_destroy(void* world);
TF_API int tf_world_count(void* world, int32_t* n_worlds);
TF_API int tf_world_set_settings(void* world, const tf_settings* settings);

/* TriangleMesh (include/twofold/mesh.h:13-30, src/mesh.cpp:122-245): builds a mesh that every world of the
 * handle may share; TF_MESH shapes name it by *out_mesh. vertices holds x, y, z per vertex, indices three
 * per triangle; both are read during the call only. */
TF_API int tf_mesh_create(void* world, const float* vertices, int32_t vertex_count, const uint32_t* indices,
                          int32_t index_count, int32_t* out_mesh);
/* The built mesh (TriangleMesh::vertices, indices, triangleCount and its tree): counts[0] vertices, [1]
 * triangles, [2] tree nodes. Every output may be null; the others take x, y, z per vertex, three indices,
 * x, y, z and one edge-flag byte per triangle, lo and hi (6 floats) and first, count (2 ints) per node. */
TF_API int tf_mesh_read(void* world, int32_t mesh, int32_t counts[3], float* vertices, uint32_t* indices,
                        float* normals, uint8_t* edges, float* node_bounds, int32_t* node_ranges);

/* computeHull (include/twofold/hull.h:17, src/hull.cpp:401-411): the convex hull of `count` points (x, y, z
 * each) with at most max_vertices corners (at least 4), as hull shapes build it. counts[0] receives the
 * vertex count and counts[1] the words of the face list; vertices (3 floats each) and faces (per face its
 * vertex count, then its vertex loop, counter-clockwise seen from outside) are written only when both
 * capacities hold them, so a first call with null outputs can size the buffers. Host only; allocates no
 * device memory. */
TF_API int tf_hull_compute(const float* points, int32_t count, int32_t max_vertices, int32_t counts[2], float* vertices,
                           int32_t vertex_capacity, int32_t* faces, int32_t face_capacity);
TF_API int tf_body_create(void* world, int32_t w, const tf_body_desc* desc, tf_id* out_body);
TF_API int tf_shape_add(void* world, int32_t w, tf_id body, const tf_shape_desc* desc, tf_id* out_shape);
/* Bulk forms: n bodies into worlds world_of[i]; n shapes onto body_of[i] (indices in world_of[i]). */
TF_API int tf_bodies_create(void* world, int32_t n, const int32_t* world_of, const tf_body_desc* descs,
                            tf_id* out_bodies);
TF_API int tf_shapes_add(void* world, int32_t n, const int32_t* world_of, const uint32_t* body_of,
                         const tf_shape_desc* descs, tf_id* out_shapes);

/* Steps every world of the batch n_steps times by dt. Returns TF_OK, or an error with the device
 * flags available from tf_world_device_status. */
/* World::createJoint (include/twofold/world.h:428; src/world.cpp:2221-2333) in world w. Invalid bodies give
 * TF_E_INVALID (the reference returns an invalid id). Refused with TF_E_UNSUPPORTED: joining bodies that
 * already have contacts without collide_connected (the reference drops those contacts), and a sleeping
 * dynamic end (the reference wakes it). */
TF_API int tf_joint_create(void* world, int32_t w, const tf_joint_desc* desc, tf_id* out_joint);
/* World::jointInfo (include/twofold/world.h:441): pose, value, last force and torque, broken. An invalid id
 * reads as zeros. */
TF_API int tf_joint_get_info(void* world, int32_t w, tf_id joint, tf_joint_info* out);
/* World::setJointLimits, setJointMotor, setJointSpring, setJointFriction, setJointSwing, setJointBreakLimits
 * (include/twofold/world.h:433-439; src/world.cpp:2341-2397) and World::destroyJoint (:429; src/world.cpp:399-406,
 * its slot reused by the next tf_joint_create with the generation bumped). An invalid id does nothing, as in
 * the reference. Where the reference wakes a sleeping dynamic end, these return TF_E_UNSUPPORTED and change
 * nothing. */
TF_API int tf_joint_set_limits(void* world, int32_t w, tf_id joint, int32_t limited, float lower, float upper);
TF_API int tf_joint_set_motor(void* world, int32_t w, tf_id joint, float speed, float max_force);
TF_API int tf_joint_set_spring(void* world, int32_t w, tf_id joint, float hertz, float damping_ratio);
TF_API int tf_joint_set_friction(void* world, int32_t w, tf_id joint, float max_friction);
TF_API int tf_joint_set_swing(void* world, int32_t w, tf_id joint, float swing_y, float swing_z);
TF_API int tf_joint_set_break_limits(void* world, int32_t w, tf_id joint, float force, float torque);
TF_API int tf_joint_destroy(void* world, int32_t w, tf_id joint);
/* World::brokenJoints (include/twofold/world.h:443): the joints that broke in world w's last step, in index
 * order; *count gets their number, at most capacity are written. */
TF_API int tf_world_broken_joints(void* world, int32_t w, tf_id* out, int32_t capacity, int32_t* count);

TF_API int tf_world_step(void* world, float dt, int32_t n_steps);
/* Records n_steps steps of every world into a CUDA graph on first use and replays it afterwards. */
TF_API int tf_world_step_graph(void* world, float dt, int32_t n_steps);
TF_API int tf_world_synchronize(void* world);
TF_API int tf_world_device_status(void* world, uint32_t* flags);

/* Body state of world w: position, rotation (x,y,z,w), linear and angular velocity. */
TF_API int tf_body_get_state(void* world, int32_t w, tf_id body, float position[3], float rotation[4],
                             float linear_velocity[3], float angular_velocity[3]);
/* World::setLinearVelocity, setAngularVelocity (include/twofold/world.h:412-413): either pointer may be null;
 * each given velocity is projected on the free axes and wakes the body's island. */
TF_API int tf_body_set_velocity(void* world, int32_t w, tf_id body, const float linear_velocity[3],
                                const float angular_velocity[3]);

/* ---- Calls between steps (include/twofold/world.h:375-463) ----
 *
 * Each changes world w as the reference's World call of the same name does, before the next step: contacts the
 * change removes are dropped by that step (pairs that touched and whose shapes go away end now, their contact
 * event reported first among the next step's events), and the bodies the reference wakes are woken, through
 * contacts with points and unbroken joints. An invalid id does nothing, as in the reference. */
/* World::destroyBody (world.h:382): its shapes, contacts and joints go with it; the slot is reused. */
TF_API int tf_body_destroy(void* world, int32_t w, tf_id body);
/* World::removeShape (world.h:387): the shape's contacts go, the body's mass is recomputed and it wakes. */
TF_API int tf_shape_remove(void* world, int32_t w, tf_id shape);
/* World::setFriction, setRestitution, setRollingResistance (world.h:397-399). */
TF_API int tf_shape_set_friction(void* world, int32_t w, tf_id shape, float friction);
TF_API int tf_shape_set_restitution(void* world, int32_t w, tf_id shape, float restitution);
TF_API int tf_shape_set_rolling_resistance(void* world, int32_t w, tf_id shape, float rolling_resistance);
/* World::setFilter (world.h:400): the shape's contacts are dropped (not ended) and their bodies woken. */
TF_API int tf_shape_set_filter(void* world, int32_t w, tf_id shape, uint32_t category, uint32_t mask);
/* World::setTransform (world.h:408): position and rotation (x, y, z, w); wakes what it touches. */
TF_API int tf_body_set_transform(void* world, int32_t w, tf_id body, const float position[3], const float rotation[4]);
/* World::setKinematicTarget (world.h:415): velocities that carry a kinematic body to the pose over dt. */
TF_API int tf_body_set_kinematic_target(void* world, int32_t w, tf_id body, const float position[3],
                                        const float rotation[4], float dt);
/* World::setMotionType (world.h:418): TF_STATIC, TF_KINEMATIC or TF_DYNAMIC. A body with a mesh or half-space
 * shape cannot become dynamic (TF_E_UNSUPPORTED), as those shapes belong to static and kinematic bodies. */
TF_API int tf_body_set_motion_type(void* world, int32_t w, tf_id body, int32_t type);
/* World::addForce / addForceAtPoint (world.h:421-422; point may be null), addTorque (:423), addImpulse /
 * addImpulseAtPoint (:424-425): dynamic bodies only; wake as the reference's wake argument; a sleeping body
 * takes nothing. */
TF_API int tf_body_add_force(void* world, int32_t w, tf_id body, const float force[3], const float* point, int32_t wake);
TF_API int tf_body_add_torque(void* world, int32_t w, tf_id body, const float torque[3], int32_t wake);
TF_API int tf_body_add_impulse(void* world, int32_t w, tf_id body, const float impulse[3], const float* point,
                               int32_t wake);
/* World::setDamping (world.h:455), setGravityScale (:457). */
TF_API int tf_body_set_damping(void* world, int32_t w, tf_id body, float linear, float angular);
TF_API int tf_body_set_gravity_scale(void* world, int32_t w, tf_id body, float scale);
/* World::wake, sleep (world.h:460-461), setCanSleep (:463; false wakes the body). */
TF_API int tf_body_wake(void* world, int32_t w, tf_id body);
TF_API int tf_body_sleep(void* world, int32_t w, tf_id body);
TF_API int tf_body_set_can_sleep(void* world, int32_t w, tf_id body, int32_t can_sleep);
/* World::setFrictionMix, setRestitutionMix (world.h:375-376): `which` 0 friction, 1 restitution. Mixing is done
 * on the device, where a host function cannot run: mix 0 (the reference's default, geometric mean for friction
 * and maximum for restitution) is accepted and any other mix is refused with TF_E_UNSUPPORTED. */
TF_API int tf_world_set_mix(void* world, int32_t which, int32_t mix);
/* Mass, local center and local inertia (row-major 3x3) as World::massProperties returns them. */
TF_API int tf_body_get_mass(void* world, int32_t w, tf_id body, float* mass, float center[3], float inertia[9]);
TF_API int tf_body_is_awake(void* world, int32_t w, tf_id body, int32_t* awake);

/* All body states of the batch in body order, world after world. Arrays hold total-body entries;
 * any pointer may be null. counts_out[w] gets the body count of world w when non-null. */
TF_API int tf_world_body_count(void* world, int64_t* total_bodies);
TF_API int tf_world_get_states(void* world, float* positions, float* rotations, float* linear_velocities,
                               float* angular_velocities, int32_t* awake);

/* Contacts of world w after the last step, in (key, part) order. include_speculative as in
 * World::contacts. Writes up to capacity entries and the total count. */
TF_API int tf_world_contacts(void* world, int32_t w, int32_t include_speculative, tf_contact* out,
                             int32_t capacity, int32_t* count);
/* World::contactEvents (include/twofold/world.h:477; ContactEvent :269-276): the pairs of shapes in world w
 * that began (begin = 1) or stopped touching in its last step, ordered by shape pair (world-local indices,
 * shape_a the lower). Sets *count to the number of events and writes at most capacity of them. After
 * tf_world_restore_state or tf_world_autotune there are none until the next step. */
TF_API int tf_world_contact_events(void* world, int32_t w, tf_contact_event* out, int32_t capacity, int32_t* count);
/* World::hitEvents (include/twofold/world.h:478; HitEvent :278-288): for each touching pair whose fastest
 * pushed point approached faster than hit_threshold in the last step, that point on shape A in the world,
 * the contact normal (A to B) and the speed; ordered by shape pair. */
TF_API int tf_world_hit_events(void* world, int32_t w, tf_hit_event* out, int32_t capacity, int32_t* count);
/* Sorted, unique shape-pair keys (minShape << 32 | maxShape) the last broadphase produced. */
TF_API int tf_world_candidates(void* world, int32_t w, uint64_t* out, int32_t capacity, int32_t* count);
TF_API int tf_world_profile(void* world, int32_t w, tf_profile* out);
/* Sum over worlds of awake dynamic bodies after the last step. */
TF_API int tf_world_awake_bodies(void* world, int64_t* count);

/* Number of kernel launches the library issued since creation (for launch accounting). */
TF_API int tf_world_launch_count(void* world, int64_t* launches);

/* Device time in milliseconds of the last tf_world_step / tf_world_step_graph call, measured with CUDA
 * events on the library's stream around the step launches. */
TF_API int tf_world_elapsed_ms(void* world, float* ms);

/* Awake dynamic bodies summed over every step of every world since creation, as each step's
 * StepProfile::awakeBodies counts them (src/world.cpp:1227-1235). */
TF_API int tf_world_body_steps(void* world, int64_t* body_steps);

/* Forces and torques (3 floats per body, all bodies of the batch in body order) added to every awake
 * dynamic body for the next step only, as World::addForce / addTorque with wake = false
 * (include/twofold/world.h:421-423). Either pointer may be null. */
TF_API int tf_world_add_forces(void* world, const float* forces, const float* torques);

/* Positions and rotations (x, y, z, w) of every body of the batch in body order, copied straight from the
 * device without refreshing any other host state (World::transform, include/twofold/world.h:404). */
TF_API int tf_world_read_poses(void* world, float* positions, float* rotations);
/* The same read queued without waiting, for a loop that steps while the last step's poses travel: the poses
 * are packed on the world's stream now and copied to positions and rotations on a copy stream of the library,
 * beside whatever the world's stream runs next. The buffers (pinned host memory, for the copy to be
 * asynchronous) must stay valid until tf_world_poses_wait returns, which waits for every queued read. Reads
 * alternate between two device staging buffers; a third waits on the device for the first one's copy. */
TF_API int tf_world_read_poses_async(void* world, float* positions, float* rotations);
TF_API int tf_world_poses_wait(void* world);

/* Per-kernel device timing of direct (non-graph) steps. When on, every kernel launch is bracketed by CUDA
 * events; tf_world_kernel_times returns, for each kernel in the order tf_kernel_name gives, the summed
 * milliseconds and the launch count since profiling was turned on. */
TF_API int tf_world_set_profiling(void* world, int32_t on);
TF_API int tf_world_kernel_times(void* world, float* ms, int64_t* launches, int32_t capacity, int32_t* count);
TF_API const char* tf_kernel_name(int32_t kernel);

/* Work of the last step, summed over the batch: out[0] bodies, [1] awake dynamic bodies, [2] candidate
 * pairs, [3] contacts, [4] active contacts, [5] active contact points. */
TF_API int tf_world_work_counts(void* world, int64_t out[6]);

/* Solver work of world w in the last step: out[0] active contacts, [1] colors, [2] contacts solved one at a
 * time (planar, rolling or beyond the last color), [3] impact contacts, [4] impact colors, [5] impact
 * contacts solved one at a time, [6] fast contacts, [7] fast contacts between solid bodies. */
TF_API int tf_world_solver_counts(void* world, int32_t w, int32_t out[8]);

/* ---- Differentiation (no counterpart in the reference) ----
 *
 * tf_tape_record steps the batch n_steps times by dt (as tf_world_step does) and records what each step's
 * solve saw: the contacts with their anchors, frames, adjusted separations and warm-start impulses, the
 * color lists, and the awake bodies. The recorded run is the differentiable model: the substepped soft solve
 * and integration with each step's contact set held fixed (no mid-step collision; speed limits inactive).
 *
 * tf_adjoint_forward runs the model from the recorded initial state in float (precision 32) or double (64)
 * and writes the final state: 13 doubles per body of the batch, center of mass (3), rotation (x, y, z, w),
 * linear and angular velocity. initial_state (same layout), mass (per body) and friction (per shape of the
 * batch) replace the recorded values when non-null; a body's local inverse inertia scales with 1/mass.
 * It keeps the state at every step boundary on the device.
 *
 * tf_adjoint_backward takes d loss / d final state (13 per body) and writes d loss / d initial state,
 * d loss / d mass and d loss / d friction (any output may be null). It recomputes each step from its
 * checkpoint and walks it in reverse, in the precision of the last forward run.
 *
 * tf_adjoint_elapsed_ms: device time of the last forward and backward runs, ms[0] and ms[1].
 * tf_adjoint_backward_ms: the last backward's recomputation and reverse walk, each summed over the chunks the
 * backward ran them in, ms[0] and ms[1] (the two run side by side, so together they can exceed its time).
 *
 * tf_adjoint_branches: per world, a signature of the branches the last forward run took at the model's
 * non-smooth points (effective masses, bias cases, impulse clamps, friction cones, restitution): equal
 * signatures for two runs mean that, up to a 64-bit hash collision, every row took the same branches, so the
 * model is smooth between them (a finite difference over them measures a slope, not a jump). */
TF_API int tf_tape_record(void* world, float dt, int32_t n_steps);
TF_API int tf_adjoint_forward(void* world, int32_t precision, const double* initial_state, const double* mass,
                              const double* friction, double* final_state);
TF_API int tf_adjoint_backward(void* world, const double* grad_final, double* grad_initial, double* grad_mass,
                               double* grad_friction);
TF_API int tf_adjoint_elapsed_ms(void* world, float ms[2]);
TF_API int tf_adjoint_backward_ms(void* world, float ms[2]);
TF_API int tf_adjoint_branches(void* world, uint64_t* per_world);

/* Snapshots of the dynamic device state (bodies, shape bounds, contacts with their impulses, sleep and wake
 * bookkeeping) in numbered slots, copied on the device without a host round trip. A snapshot can be put back
 * until the batch is laid out again (a body or shape added, or a device list grown), after which
 * tf_world_restore_state returns TF_E_INVALID. No counterpart in the reference, where copying a World is
 * the snapshot (include/twofold/world.h:366-369). */
TF_API int tf_world_save_state(void* world, int32_t slot);
TF_API int tf_world_restore_state(void* world, int32_t slot);

/* Times candidate launch shapes for every kernel on the batch's current state (trial_steps steps per
 * candidate, the state put back after each) and keeps the fastest; the batch ends in the state it started
 * in. out, when non-null, receives 8 x 3 words: threads, big-world threshold and shared bytes per kernel,
 * in tf_world_set_launch's kernel order (plus 7 = the pair collisions). No counterpart in the reference. */
TF_API int tf_world_autotune(void* world, float dt, int32_t trial_steps, uint32_t* out);

/* Launch shape of one kernel (0 broadphase, 1 narrowphase, 2 wake, 3 prepare, 4 refresh, 5 substep,
 * 6 finish, 7 pair collisions; -1 every kernel): threads per CTA (a multiple of 32, at most 512), the world size in bodies
 * above which a world is stepped by a whole CTA (smaller worlds take one warp each), and the shared memory
 * a CTA stages worlds in (clamped to what the device allows). For the substep, big_bodies = -1 selects the
 * flat solve instead (every world's contacts of a color at once across the device, at most 256 threads per
 * CTA, no staging). Takes effect at the next step. No counterpart in the reference, which steps each world on
 * one host thread; the autotuner uses it. */
TF_API int tf_world_set_launch(void* world, int32_t kernel, int32_t threads, int32_t big_bodies, int32_t smem_bytes);
/* The shape in use: out[0] threads, [1] big-world threshold (0xffffffff for the flat solve), [2] shared bytes,
 * [3] grid size, [4] bodies a whole-CTA world can stage, [5] bodies a warp's world can stage. */
TF_API int tf_world_get_launch(void* world, int32_t kernel, uint32_t out[6]);

/* ---- Candidate pairs without device allocation (no counterpart in the reference) ----
 *
 * The broadphase's candidate pairs for one world whose bodies have one shape each (shape index = body
 * index), from device arrays the caller owns: lo and hi (n x 3 floats, the shapes' world bounds), grow (n
 * floats, each body's growth for the step) and flags (n words of TF_PAIR_* bits). The pair rules are the
 * step's (World::Impl::updateContacts, src/world.cpp:788-842, for single-shape bodies), and the result is
 * what tf_world_candidates reports for such a world: keys min << 32 | max, sorted and unique, as long as the
 * world also has default collision filters (every category and mask bit set), no joints and no half-space
 * shapes. Three of the step's rules are not applied here: the category/mask filter (src/world.cpp:334-337),
 * the exclusion of jointed body pairs (:796, :829) and the half-space pairs (:843-866); a caller with any
 * of those filters, joints or planes drops or adds those pairs itself. Up to
 * `capacity` keys go to the device array `keys`; the device word `count` receives the number of unique
 * keys (more than capacity when they did not all fit), or -1 when the pair tests found more than
 * TF_NOALLOC_MAX_PAIRS keys before repeats were dropped (keys is then left as it was).
 *
 * It allocates nothing: its scratch is a fixed array in the library's device image. n above
 * TF_NOALLOC_MAX_BODIES is refused with TF_E_CAPACITY. The work is queued on `stream` (a cudaStream_t; NULL
 * for the default stream) on the current device and the call returns without waiting. Each call looks up the
 * scratch's address in the current context (a host-side lookup), so after cudaDeviceReset a new context
 * finds it wherever the library's device image now is. The first lookup in a context may load that image,
 * so make one call before any stream capture. Calls whose work overlaps on one device (other streams, other host threads) share the scratch and race;
 * order them on one stream. */
#define TF_NOALLOC_MAX_BODIES 4096
#define TF_NOALLOC_MAX_PAIRS 32768
enum tf_pair_flags { TF_PAIR_LIVE = 1u << 0, TF_PAIR_DYNAMIC = 1u << 1, TF_PAIR_MOVING = 1u << 2 };
TF_API int tf_candidates_noalloc(const float* lo, const float* hi, const float* grow, const uint32_t* flags, int32_t n,
                                 uint64_t* keys, int32_t capacity, int32_t* count, void* stream);

#ifdef __cplusplus
}
#endif

#endif
