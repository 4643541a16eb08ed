// The flat solve (k_substep_flat, tf_kernels.cuh), compiled on its own with global loads cached in L2 only
// (-Xptxas -dlcm=cg): its CTAs read what other CTAs wrote before the last grid barrier, which an SM's L1 would
// not see.
#include "tf_kernels.cuh"
#include "tf_launch.h"

namespace tfb {

const void* flatKernels(int id) {
    switch (id) {
        case kKSubstepFlat: return (const void*)k_substep_flat<false>;
        case kKSubstepFlatJoints: return (const void*)k_substep_flat<true>;
        default: return nullptr;
    }
}

}  // namespace tfb
