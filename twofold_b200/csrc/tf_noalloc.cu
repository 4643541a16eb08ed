// tf_candidates_noalloc: the broadphase's candidate pairs for one world of single-shape bodies, computed
// with scratch memory that is part of the library image instead of memory allocated on the device.
//
// The pair rules are the step's (src/world.cpp:788-842 in the reference, k_broadphase here) specialised to
// one shape per body, with shape index = body index: both bodies live, one of them dynamic, one of them
// moving; their bounds overlap after growing one by the sum of both growths; each shape's bounds overlap
// the other body's bounds grown by that sum; and the shapes' bounds, each grown by its own body's growth,
// overlap. The keys (min << 32 | max) come out sorted and unique, as World::Impl::updateContacts leaves them
// (src/world.cpp:868-869). The step's other rules (category/mask filters, jointed pairs, half-space pairs)
// are not applied: the inputs carry no filters, joints or planes.
//
// Scratch: g_pairScratch below, a fixed-size array in the library's device image. Its address on a device is
// looked up once, with that device current, on the first call made there; later calls on that device reuse
// it, so the library must not be called on a device again after a cudaDeviceReset there. Nothing here
// allocates device or host memory through CUDA or any other library. Because the scratch is one per device,
// calls whose work overlaps on the device (different streams, or different host threads) race on it and give
// wrong results; issue them on one stream or serialise them.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/twofold_b200.h"
#include "tf_body.cuh"

namespace tfb {

int noteError(int code, const std::string& msg);

namespace {

constexpr int32_t kMaxBodies = TF_NOALLOC_MAX_BODIES;
constexpr int32_t kMaxPairs = TF_NOALLOC_MAX_PAIRS;
constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;

struct PairScratch {
    uint64_t emitted[kMaxPairs];  // keys in the order the pair tests found them
    uint64_t sorted[kMaxPairs];   // the same keys, sorted
    uint32_t row[kMaxBodies];     // keys per first shape, then their running offsets
    uint32_t total;               // keys found
};

}  // namespace

// 256-byte aligned so that every field above starts on a 16-byte boundary.
static __device__ __align__(256) unsigned char g_pairScratch[sizeof(PairScratch)];

namespace {

// Exclusive prefix sum over the CTA; every thread calls it.
__device__ uint32_t ctaScan(uint32_t v, uint32_t& total) {
    __shared__ uint32_t sums[kWarps];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if ((int)lane >= o) { x += y; }
    }
    if (lane == 31) { sums[warp] = x; }
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < kWarps ? sums[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if ((int)lane >= o) { s += y; }
        }
        if (lane < kWarps) { sums[lane] = s; }
    }
    __syncthreads();
    const uint32_t prefix = (warp > 0 ? sums[warp - 1] : 0u) + x - v;
    total = sums[kWarps - 1];
    __syncthreads();
    return prefix;
}

__device__ __forceinline__ Vec3 at(const float* p, uint32_t i) { return Vec3{ p[3 * i], p[3 * i + 1], p[3 * i + 2] }; }

// One CTA does everything: clear, pair tests (a warp per first body, lanes over the bodies after it),
// a counting sort by first shape, each row sorted on its own, repeats dropped.
__global__ void __launch_bounds__(kThreads) k_candidates_noalloc(const float* lo, const float* hi, const float* grow,
                                                                 const uint32_t* flags, uint32_t n, uint64_t* keys,
                                                                 uint32_t capacity, int32_t* count, PairScratch* S) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t r = tid; r < n; r += kThreads) { S->row[r] = 0; }
    if (tid == 0) { S->total = 0; }
    __syncthreads();
    for (uint32_t a = warp; a + 1 < n; a += kWarps) {
        const uint32_t fa = flags[a];
        if (!(fa & TF_PAIR_LIVE)) { continue; }
        const Vec3 loA = at(lo, a), hiA = at(hi, a);
        const float gA = grow[a];
        for (uint32_t b = a + 1 + lane; b < n; b += 32) {
            const uint32_t fb = flags[b];
            if (!(fb & TF_PAIR_LIVE) || !((fa | fb) & TF_PAIR_DYNAMIC) || !((fa | fb) & TF_PAIR_MOVING)) { continue; }
            const Vec3 loB = at(lo, b), hiB = at(hi, b);
            const float gB = grow[b];
            const float gg = gA + gB;
            const Vec3 reach{ gg, gg, gg };
            if (!boxesOverlap(loA - reach, hiA + reach, loB, hiB)) { continue; }
            if (!boxesOverlap(loA, hiA, loB - reach, hiB + reach)) { continue; }
            if (!boxesOverlap(loB, hiB, loA - reach, hiA + reach)) { continue; }
            const Vec3 g3a{ gA, gA, gA }, g3b{ gB, gB, gB };
            if (!boxesOverlap(loA - g3a, hiA + g3a, loB - g3b, hiB + g3b)) { continue; }
            const uint32_t pos = atomicAdd(&S->total, 1u);
            if (pos < (uint32_t)kMaxPairs) { S->emitted[pos] = ((uint64_t)a << 32) | (uint64_t)b; }
        }
    }
    __syncthreads();
    const uint32_t total = S->total;
    if (total > (uint32_t)kMaxPairs) {
        if (tid == 0) { *count = -1; }
        return;
    }
    for (uint32_t i = tid; i < total; i += kThreads) { atomicAdd(&S->row[(uint32_t)(S->emitted[i] >> 32)], 1u); }
    __syncthreads();
    uint32_t base = 0;
    for (uint32_t start = 0; start < n; start += kThreads) {
        const uint32_t r = start + tid;
        const uint32_t v = r < n ? S->row[r] : 0u;
        uint32_t tot;
        const uint32_t pre = ctaScan(v, tot);
        if (r < n) { S->row[r] = base + pre; }
        base += tot;
    }
    __syncthreads();
    // Scattering advances each row's start to its end.
    for (uint32_t i = tid; i < total; i += kThreads) {
        const uint64_t k = S->emitted[i];
        S->sorted[atomicAdd(&S->row[(uint32_t)(k >> 32)], 1u)] = k;
    }
    __syncthreads();
    for (uint32_t r = tid; r < n; r += kThreads) {
        const uint32_t s = r > 0 ? S->row[r - 1] : 0u, e = S->row[r];
        for (uint32_t i = s + 1; i < e; ++i) {
            const uint64_t k = S->sorted[i];
            uint32_t j = i;
            while (j > s && S->sorted[j - 1] > k) {
                S->sorted[j] = S->sorted[j - 1];
                --j;
            }
            S->sorted[j] = k;
        }
    }
    __syncthreads();
    uint32_t unique = 0;
    for (uint32_t start = 0; start < total; start += kThreads) {
        const uint32_t i = start + tid;
        const bool first = i < total && (i == 0 || S->sorted[i] != S->sorted[i - 1]);
        uint32_t tot;
        const uint32_t pos = unique + ctaScan(first ? 1u : 0u, tot);
        if (first && pos < capacity) { keys[pos] = S->sorted[i]; }
        unique += tot;
    }
    if (tid == 0) { *count = (int32_t)unique; }
}

// The scratch's device address in the current context, looked up on every call (a host-side table lookup of the
// loaded module, cheap): a context made after a device reset may place the module elsewhere.
int scratchAddress(PairScratch** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_pairScratch);
    if (e != cudaSuccess) {
        return noteError(TF_E_CUDA, std::string("tf_candidates_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    }
    *out = static_cast<PairScratch*>(p);
    return TF_OK;
}

}  // namespace
}  // namespace tfb

extern "C" {

TF_API int tf_candidates_noalloc(const float* lo, const float* hi, const float* grow, const uint32_t* flags, int32_t n,
                                 uint64_t* keys, int32_t capacity, int32_t* count, void* stream) {
    using namespace tfb;
    if (n < 0 || capacity < 0) { return noteError(TF_E_INVALID, "tf_candidates_noalloc: negative size"); }
    if (n > kMaxBodies) {
        return noteError(TF_E_CAPACITY, "tf_candidates_noalloc: " + std::to_string(n) + " bodies; at most " +
                                            std::to_string(kMaxBodies) + " fit its fixed scratch");
    }
    if (!count || (n > 0 && (!lo || !hi || !grow || !flags)) || (capacity > 0 && !keys)) {
        return noteError(TF_E_INVALID, "tf_candidates_noalloc: null pointer");
    }
    PairScratch* S = nullptr;
    const int rc = scratchAddress(&S);
    if (rc != TF_OK) { return rc; }
    k_candidates_noalloc<<<1, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(lo, hi, grow, flags, (uint32_t)n, keys,
                                                                                (uint32_t)capacity, count, S);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { return noteError(TF_E_CUDA, std::string("tf_candidates_noalloc: launch: ") + cudaGetErrorString(e)); }
    return TF_OK;
}

}  // extern "C"
