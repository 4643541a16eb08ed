// A box pyramid on a half-space, stepped through the public World API and printed body by body.
// The same source builds against the reference's include/twofold/twofold.h and against
// include/twofold_b200/world.hpp: TWOFOLD_HEADER names the header to use.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include TWOFOLD_HEADER

int main(int argc, char** argv) {
    using namespace twofold;
    const int rows = argc > 1 ? std::atoi(argv[1]) : 6;
    const int steps = argc > 2 ? std::atoi(argv[2]) : 60;
    World world;
    BodyDesc ground;
    ground.type = MotionType::Static;
    // Turns the half-space's +z normal onto +y: a quarter turn about -x.
    ground.rotation = Quat{ -0.70710677f, 0.0f, 0.0f, 0.70710677f };
    const BodyId g = world.createBody(ground);
    ShapeDesc plane;
    plane.geometry = HalfSpace{};
    plane.friction = 0.6f;
    world.addShape(g, plane);
    std::vector<BodyId> boxes;
    for (int r = 0; r < rows; ++r) {
        for (int i = 0; i < rows - r; ++i) {
            BodyDesc d;
            d.position = Vec3{ (float)i - 0.5f * (float)(rows - 1 - r), 0.5f + (float)r, 0.0f };
            d.canSleep = false;
            const BodyId b = world.createBody(d);
            ShapeDesc s;
            s.geometry = Box{ Vec3{ 0.5f, 0.5f, 0.5f } };
            s.friction = 0.6f;
            world.addShape(b, s);
            boxes.push_back(b);
        }
    }
    // A sphere thrown at the pyramid, so that the solve has work beyond resting contact.
    BodyDesc ball;
    ball.position = Vec3{ -6.0f, 1.0f, 0.2f };
    ball.linearVelocity = Vec3{ 8.0f, 1.0f, 0.0f };
    ball.canSleep = false;
    const BodyId s = world.createBody(ball);
    ShapeDesc sd;
    sd.geometry = Sphere{ 0.4f };
    sd.density = 3.0f;
    sd.friction = 0.4f;
    world.addShape(s, sd);
    boxes.push_back(s);
    // Events summed over the run: pairs that began and stopped touching, hits and their speeds.
    int began = 0, ended = 0, hits = 0;
    double hitSpeed = 0.0;
    for (int k = 0; k < steps; ++k) {
        world.step(1.0f / 60.0f);
        for (const ContactEvent& e : world.contactEvents()) { (e.begin ? began : ended) += 1; }
        for (const HitEvent& h : world.hitEvents()) {
            ++hits;
            hitSpeed += h.speed;
        }
    }
    std::printf("manifolds %d\n", world.profile().manifolds);
    std::printf("events %d %d %d %.6g %d\n", began, ended, hits, hitSpeed, world.profile().touchingContacts);
    for (const BodyId& b : boxes) {
        const Vec3 p = world.position(b);
        const Quat q = world.rotation(b);
        const Vec3 v = world.linearVelocity(b);
        const Vec3 w = world.angularVelocity(b);
        std::printf("%u %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g\n", b.index, p.x, p.y, p.z, q.x,
                    q.y, q.z, q.w, v.x, v.y, v.z, w.x, w.y, w.z);
    }
    return 0;
}
