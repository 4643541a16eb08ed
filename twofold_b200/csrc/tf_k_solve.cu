// Step preparation and the substep (tf_kernels.cuh), compiled on their own.
#include "tf_kernels.cuh"
#include "tf_launch.h"

namespace tfb {

const void* solveKernels(int id) {
    switch (id) {
        case kKPrepare: return (const void*)k_prepare<0>;
        case kKSubstep: return (const void*)k_substep<false>;
        case kKSubstepJoints: return (const void*)k_substep<true>;
        default: return nullptr;
    }
}

}  // namespace tfb
