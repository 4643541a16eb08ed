// Joints of every kind stepped through the public World API, printed body by body and joint by joint. The
// same source builds against the reference's include/twofold/twofold.h and against
// include/twofold_b200/world.hpp: TWOFOLD_HEADER names the header to use.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include TWOFOLD_HEADER

int main(int argc, char** argv) {
    using namespace twofold;
    const int steps = argc > 1 ? std::atoi(argv[1]) : 60;
    World world;
    BodyDesc ground;
    ground.type = MotionType::Static;
    ground.rotation = Quat{ -0.70710677f, 0.0f, 0.0f, 0.70710677f };
    ShapeDesc plane;
    plane.geometry = HalfSpace{};
    world.addShape(world.createBody(ground), plane);
    std::vector<BodyId> bodies;
    auto box = [&](const Vec3& p, const Vec3& half, const Vec3& w) {
        BodyDesc d;
        d.position = p;
        d.angularVelocity = w;
        d.canSleep = false;
        const BodyId b = world.createBody(d);
        ShapeDesc s;
        s.geometry = Box{ half };
        world.addShape(b, s);
        bodies.push_back(b);
        return b;
    };
    std::vector<JointId> joints;
    auto join = [&](BodyId a, BodyId b, const JointKind& kind, float breakForce) {
        JointDesc j;
        j.bodyA = a;
        j.bodyB = b;
        j.kind = kind;
        j.breakForce = breakForce;
        joints.push_back(world.createJoint(j));
    };
    const float inf = INFINITY;
    // A limited hinge pendulum with a motor, held from the world.
    HingeJoint hinge;
    hinge.anchor = Vec3{ 0.0f, 3.0f, 0.0f };
    hinge.limited = true;
    hinge.lowerAngle = -0.5f;
    hinge.upperAngle = 1.0f;
    hinge.motorSpeed = 1.5f;
    hinge.maxMotorTorque = 5.0f;
    join({}, box(Vec3{ 0.6f, 3.0f, 0.0f }, Vec3{ 0.5f, 0.1f, 0.1f }, Vec3{}), hinge, inf);
    // A spring from the world and a rod between two boxes.
    DistanceJoint spring;
    spring.anchorA = Vec3{ 3.0f, 4.0f, 0.0f };
    spring.anchorB = Vec3{ 3.0f, 2.7f, 0.0f };
    spring.hertz = 1.5f;
    spring.dampingRatio = 0.2f;
    join({}, box(Vec3{ 3.0f, 2.5f, 0.0f }, Vec3{ 0.2f, 0.2f, 0.2f }, Vec3{}), spring, inf);
    const BodyId r1 = box(Vec3{ 5.0f, 3.0f, 0.0f }, Vec3{ 0.2f, 0.2f, 0.2f }, Vec3{ 0.0f, 0.0f, 1.0f });
    const BodyId r2 = box(Vec3{ 5.8f, 3.0f, 0.0f }, Vec3{ 0.2f, 0.2f, 0.2f }, Vec3{});
    DistanceJoint rod;
    rod.anchorA = Vec3{ 5.0f, 3.0f, 0.0f };
    rod.anchorB = Vec3{ 5.8f, 3.0f, 0.0f };
    join(r1, r2, rod, inf);
    // A limited slider with a motor, a point joint that breaks, a fixed pair, a swing-twist pair.
    SliderJoint slider;
    slider.anchor = Vec3{ 8.0f, 2.0f, 0.0f };
    slider.limited = true;
    slider.lowerTranslation = -0.4f;
    slider.upperTranslation = 0.4f;
    slider.motorSpeed = 0.5f;
    slider.maxMotorForce = 10.0f;
    join({}, box(Vec3{ 8.0f, 2.0f, 0.0f }, Vec3{ 0.3f, 0.1f, 0.1f }, Vec3{}), slider, inf);
    PointJoint point;
    point.anchor = Vec3{ 10.0f, 3.2f, 0.0f };
    join({}, box(Vec3{ 10.0f, 3.0f, 0.0f }, Vec3{ 0.2f, 0.2f, 0.2f }, Vec3{}), point, 0.2f);
    const BodyId f1 = box(Vec3{ 12.0f, 1.0f, 0.0f }, Vec3{ 0.3f, 0.3f, 0.3f }, Vec3{});
    const BodyId f2 = box(Vec3{ 12.6f, 1.0f, 0.0f }, Vec3{ 0.3f, 0.3f, 0.3f }, Vec3{});
    FixedJoint fixed;
    fixed.anchor = Vec3{ 12.3f, 1.0f, 0.0f };
    join(f1, f2, fixed, inf);
    SwingTwistJoint swing;
    swing.anchor = Vec3{ 14.0f, 4.0f, 0.0f };
    swing.axis = Vec3{ 0.0f, -1.0f, 0.0f };
    swing.swingY = 0.4f;
    swing.swingZ = 0.6f;
    swing.lowerTwist = -0.2f;
    swing.upperTwist = 0.2f;
    join({}, box(Vec3{ 14.0f, 3.6f, 0.0f }, Vec3{ 0.1f, 0.4f, 0.1f }, Vec3{ 2.0f, 0.0f, 1.0f }), swing, inf);
    int broken = 0;
    for (int k = 0; k < steps; ++k) {
        world.step(1.0f / 60.0f);
        broken += (int)world.brokenJoints().size();
    }
    std::printf("broken %d\n", broken);
    for (const BodyId& b : bodies) {
        const Vec3 p = world.position(b);
        const Quat q = world.rotation(b);
        const Vec3 v = world.linearVelocity(b);
        const Vec3 w = world.angularVelocity(b);
        std::printf("%u %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g\n", b.index, p.x, p.y, p.z, q.x,
                    q.y, q.z, q.w, v.x, v.y, v.z, w.x, w.y, w.z);
    }
    std::printf("live %d\n", (int)world.joints().size());
    for (const JointId& j : joints) {
        const JointInfo info = world.jointInfo(j);
        std::printf("joint %u %d %.9g %.9g %.9g %.9g %d\n", j.index, (int)info.type, info.value, info.force.x,
                    info.force.y, info.force.z, info.broken ? 1 : 0);
    }
    return 0;
}
