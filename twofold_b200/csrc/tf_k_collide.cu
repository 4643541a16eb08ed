// The pair collisions, one kernel per pair class and one over every class (tf_kernels.cuh), compiled on their own.
#include "tf_kernels.cuh"
#include "tf_launch.h"

namespace tfb {

const void* collideKernels(int id) {
    switch (id) {
        case kKCollideAll: return (const void*)k_collide_all<0>;
        case kKCollide + kClassSpheres: return (const void*)k_collide<kClassSpheres>;
        case kKCollide + kClassSpherePoly: return (const void*)k_collide<kClassSpherePoly>;
        case kKCollide + kClassPlane: return (const void*)k_collide<kClassPlane>;
        case kKCollide + kClassConvex: return (const void*)k_collide<kClassConvex>;
        case kKCollide + kClassPlanar: return (const void*)k_collide<kClassPlanar>;
        case kKCollide + kClassMesh: return (const void*)k_collide<kClassMesh>;
        default: return nullptr;
    }
}

}  // namespace tfb
