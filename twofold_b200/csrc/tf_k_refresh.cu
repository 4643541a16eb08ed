// The mid-step refreshes, one kernel per list and one over every list (tf_kernels.cuh), compiled on their own.
#include "tf_kernels.cuh"
#include "tf_launch.h"

namespace tfb {

const void* refreshKernels(int id) {
    switch (id) {
        case kKRefreshAll: return (const void*)k_refresh_all<0>;
        case kKRefresh + kClassSpheres: return (const void*)k_refresh<kClassSpheres>;
        case kKRefresh + kClassSpherePoly: return (const void*)k_refresh<kClassSpherePoly>;
        case kKRefresh + kClassPlane: return (const void*)k_refresh<kClassPlane>;
        case kKRefresh + kClassConvex: return (const void*)k_refresh<kClassConvex>;
        case kKRefresh + kClassPlanar: return (const void*)k_refresh<kClassPlanar>;
        case kKRefresh + kClassMesh: return (const void*)k_refresh<kClassMesh>;
        case kKRefresh + kPairClasses: return (const void*)k_refresh<kClassAny>;
        default: return nullptr;
    }
}

}  // namespace tfb
