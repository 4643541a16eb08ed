// The kernels of a step, by name, for the engine's launches.
//
// The kernels are templates (tf_kernels.cuh), so a translation unit compiles only the ones it takes the address
// of. Each tf_k_*.cu file instantiates one group of them and hands out their entry addresses; the engine launches
// them with cudaLaunchKernel and never instantiates a kernel itself. The groups compile in parallel.
#pragma once

#include <cuda_runtime.h>

namespace tfb {

enum KernelId : int {
    kKBroadphase = 0,
    kKBroadPairs,
    kKBroadFinish,
    kKNarrowphase,
    kKWake,
    kKCollideAll,
    kKCollide,  // + pair class (kClassSpheres .. kClassMesh)
    kKRefreshAll = kKCollide + 6,
    kKRefresh,  // + pair class, kClassAny (the other active contacts) last
    kKPrepare = kKRefresh + 7,
    kKSubstep,
    kKSubstepJoints,
    kKFinish,
    kKFinishJoints,
    kKTapeRecord,
    kKAddForces,
    kKPackPoses,
    kKStepSummary,
    kKSubstepFlat,
    kKSubstepFlatJoints,
    kKernelIds
};

// Entry addresses, each defined in the translation unit that compiles the group (nullptr for other ids).
const void* broadKernels(int id);    // tf_k_broad.cu: broadphase, pair sweep, narrowphase, wake
const void* collideKernels(int id);  // tf_k_collide.cu: pair collisions
const void* refreshKernels(int id);  // tf_k_refresh.cu: mid-step refreshes
const void* solveKernels(int id);    // tf_k_solve.cu: preparation and substeps
const void* finishKernels(int id);   // tf_k_finish.cu: end of step, tape, host-buffer helpers
const void* flatKernels(int id);     // tf_k_flat.cu: the flat solve (its global loads bypass L1)

inline const void* kernelEntry(int id) {
    if (id < kKCollideAll) { return broadKernels(id); }
    if (id < kKRefreshAll) { return collideKernels(id); }
    if (id < kKPrepare) { return refreshKernels(id); }
    if (id < kKFinish) { return solveKernels(id); }
    if (id < kKSubstepFlat) { return finishKernels(id); }
    return flatKernels(id);
}

}  // namespace tfb
