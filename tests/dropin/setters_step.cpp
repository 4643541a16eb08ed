// The World calls made between steps, each used mid-run through the public World API, with the bodies printed
// every 20 steps. The same source builds against the reference's include/twofold/twofold.h and against
// include/twofold_b200/world.hpp: TWOFOLD_HEADER names the header to use.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include TWOFOLD_HEADER

using namespace twofold;

static void print(World& world, int step) {
    std::printf("step %d\n", step);
    for (const BodyId& b : world.bodies()) {
        const Vec3 p = world.position(b);
        const Quat q = world.rotation(b);
        const Vec3 v = world.linearVelocity(b);
        const Vec3 w = world.angularVelocity(b);
        std::printf("%u %u %d %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g\n", b.index,
                    b.generation, world.isAwake(b) ? 1 : 0, p.x, p.y, p.z, q.x, q.y, q.z, q.w, v.x, v.y, v.z, w.x,
                    w.y, w.z);
    }
}

int main(int argc, char** argv) {
    const int steps = argc > 1 ? std::atoi(argv[1]) : 160;
    World world;
    BodyDesc ground;
    ground.type = MotionType::Static;
    ground.rotation = Quat{ -0.70710677f, 0.0f, 0.0f, 0.70710677f };
    ShapeDesc plane;
    plane.geometry = HalfSpace{};
    world.addShape(world.createBody(ground), plane);

    auto body = [&](const Vec3& p, MotionType type = MotionType::Dynamic) {
        BodyDesc d;
        d.position = p;
        d.type = type;
        return world.createBody(d);
    };
    auto boxShape = [&](BodyId b, const Vec3& half, const Vec3& at = Vec3{}) {
        ShapeDesc s;
        s.geometry = Box{ half };
        s.position = at;
        return world.addShape(b, s);
    };
    auto sphereShape = [&](BodyId b, float r) {
        ShapeDesc s;
        s.geometry = Sphere{ r };
        return world.addShape(b, s);
    };

    // A stack of three boxes, a rolling sphere, a two-box body, a kinematic paddle, and a few loose boxes.
    std::vector<BodyId> stack;
    std::vector<ShapeId> stackShapes;
    for (int i = 0; i < 3; ++i) {
        stack.push_back(body(Vec3{ 0.0f, 0.5f + 1.0f * (float)i, 0.0f }));
        stackShapes.push_back(boxShape(stack.back(), Vec3{ 0.5f, 0.5f, 0.5f }));
    }
    const BodyId ball = body(Vec3{ 3.0f, 0.4f, 0.0f });
    const ShapeId ballShape = sphereShape(ball, 0.4f);
    world.setLinearVelocity(ball, Vec3{ -1.0f, 0.0f, 0.0f });
    const BodyId pair = body(Vec3{ -3.0f, 0.5f, 0.0f });
    boxShape(pair, Vec3{ 0.4f, 0.4f, 0.4f }, Vec3{ -0.4f, 0.0f, 0.0f });
    const ShapeId pairRight = boxShape(pair, Vec3{ 0.4f, 0.4f, 0.4f }, Vec3{ 0.4f, 0.0f, 0.0f });
    const BodyId paddle = body(Vec3{ 0.0f, 0.3f, 3.0f }, MotionType::Kinematic);
    boxShape(paddle, Vec3{ 1.0f, 0.2f, 0.2f });
    std::vector<BodyId> loose;
    std::vector<ShapeId> looseShapes;
    for (int i = 0; i < 4; ++i) {
        loose.push_back(body(Vec3{ 6.0f + 1.2f * (float)i, 0.5f, 2.0f }));
        looseShapes.push_back(boxShape(loose.back(), Vec3{ 0.5f, 0.5f, 0.5f }));
    }

    const float dt = 1.0f / 60.0f;
    BodyId reborn{};
    for (int k = 1; k <= steps; ++k) {
        switch (k) {
        case 10:
            world.setFriction(stackShapes[0], 0.1f);
            world.setRestitution(ballShape, 0.8f);
            world.setRollingResistance(ballShape, 0.05f);
            break;
        case 15:
            world.addForce(stack[2], Vec3{ 40.0f, 0.0f, 0.0f });
            world.addForceAtPoint(loose[0], Vec3{ 0.0f, 0.0f, 30.0f }, Vec3{ 6.4f, 0.9f, 2.0f });
            world.addTorque(loose[1], Vec3{ 0.0f, 8.0f, 0.0f });
            world.addImpulse(pair, Vec3{ 0.0f, 3.0f, 1.0f });
            world.addImpulseAtPoint(loose[2], Vec3{ 1.0f, 2.0f, 0.0f }, Vec3{ 8.4f, 0.2f, 2.3f });
            break;
        case 20:
            world.setTransform(loose[3], Vec3{ 9.6f, 2.5f, 2.0f }, Quat{ 0.0f, 0.38268343f, 0.0f, 0.92387953f });
            world.setAngularVelocity(loose[3], Vec3{ 1.0f, 0.0f, 2.0f });
            break;
        case 25:
        case 26:
        case 27:
        case 28:
            world.setKinematicTarget(paddle, Vec3{ 0.0f, 0.3f, 3.0f - 0.1f * (float)(k - 24) },
                                     Quat{ 0.0f, 0.04997917f * (float)(k - 24), 0.0f,
                                           std::sqrt(1.0f - 0.0024979174f * (float)((k - 24) * (k - 24))) },
                                     dt);
            break;
        case 30:
            world.setMotionType(loose[1], MotionType::Kinematic);
            world.setMotionType(loose[2], MotionType::Static);
            break;
        case 40:
            world.setMotionType(loose[1], MotionType::Dynamic);
            world.setMotionType(loose[2], MotionType::Dynamic);
            world.setFilter(stackShapes[1], 2u, ~2u);
            break;
        case 50:
            world.removeShape(pairRight);
            world.setDamping(ball, 0.5f, 0.8f);
            world.setGravityScale(loose[3], -0.2f);
            break;
        case 60:
            world.destroyBody(loose[0]);
            reborn = body(Vec3{ 6.0f, 3.0f, 2.0f });
            sphereShape(reborn, 0.3f);
            world.setLinearVelocity(reborn, Vec3{ 0.5f, 0.0f, 0.0f });
            std::printf("valid %d %d %d\n", world.isValid(loose[0]) ? 1 : 0, world.isValid(looseShapes[0]) ? 1 : 0,
                        world.isValid(reborn) ? 1 : 0);
            break;
        case 70:
            world.setGravityScale(loose[3], 1.0f);
            world.sleep(stack[0]);
            break;
        case 80:
            world.wake(stack[0]);
            world.setCanSleep(pair, false);
            world.addForce(stack[1], Vec3{ 0.0f, 50.0f, 0.0f }, false);
            break;
        case 100:
            world.setCanSleep(pair, true);
            world.setLinearVelocity(paddle, Vec3{});
            world.setAngularVelocity(paddle, Vec3{});
            break;
        default:
            break;
        }
        world.step(dt);
        if (k % 20 == 0) { print(world, k); }
    }
    return 0;
}
