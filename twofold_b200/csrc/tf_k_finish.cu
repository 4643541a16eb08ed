// The end of the step, the tape recorder and the host-buffer helpers (tf_kernels.cuh), compiled on their own.
#include "tf_kernels.cuh"
#include "tf_launch.h"

namespace tfb {

const void* finishKernels(int id) {
    switch (id) {
        case kKFinish: return (const void*)k_finish<false>;
        case kKFinishJoints: return (const void*)k_finish<true>;
        case kKTapeRecord: return (const void*)k_tape_record<0>;
        case kKAddForces: return (const void*)k_add_forces<0>;
        case kKPackPoses: return (const void*)k_pack_poses<0>;
        case kKStepSummary: return (const void*)k_step_summary<0>;
        default: return nullptr;
    }
}

}  // namespace tfb
