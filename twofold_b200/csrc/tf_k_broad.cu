// Broadphase, the big worlds' pair sweep, narrowphase merge and wake (tf_kernels.cuh), compiled on their own.
#include "tf_kernels.cuh"
#include "tf_launch.h"

namespace tfb {

const void* broadKernels(int id) {
    switch (id) {
        case kKBroadphase: return (const void*)k_broadphase<0>;
        case kKBroadPairs: return (const void*)k_broad_pairs<0>;
        case kKBroadFinish: return (const void*)k_broad_finish<0>;
        case kKNarrowphase: return (const void*)k_narrowphase<0>;
        case kKWake: return (const void*)k_wake<0>;
        default: return nullptr;
    }
}

}  // namespace tfb
