// Shared kernel prologue: make the scene program visible to the CTA, and the
// persistent ray-queue machinery the tracing kernels share.
#pragma once

#include "device.cuh"
#include "kernels.h"

namespace ifx {

static constexpr int kWarp = 32;
static constexpr unsigned kFull = 0xffffffffu;

// Dynamic shared memory of a tracing CTA: the staged blob (when it fits)
// followed by the threads' BVH stacks.
static inline size_t blob_smem(const BlobRef& b, int block) {
    size_t s = b.staged ? (size_t)align16(b.stage_bytes) : 0;
    return s + (size_t)b.stack_depth * (size_t)block * 8u;  // node index + box distance
}

// Stages the blob's geometry prefix into dynamic shared memory (one bulk
// copy) or, for large scenes, reads it in place, and points the view at this
// thread's stack. All threads of the CTA must call this before any of them
// exits. Returns false if staging timed out.
__device__ __forceinline__ bool scene_prologue(const BlobRef& blob, uint8_t* dsmem, uint64_t* mbar,
                                               uint32_t* status, SceneView& sv) {
    sv = make_view(blob.ptr);
    sv.status = status;
    sv.lg = blob.lg;
    uint32_t used = 0;
    if (blob.staged) {
        if (!stage_scene(blob.ptr, blob.stage_bytes, dsmem, mbar, status, blob.wait_polls)) return false;
        const SceneView s = make_view(dsmem);
        sv.objs = s.objs;
        sv.prims = s.prims;
        sv.nodes = s.nodes;
        used = align16(blob.stage_bytes);
    }
    uint32_t* stk = reinterpret_cast<uint32_t*>(dsmem + used);
    sv.stk = stk + threadIdx.x;
    sv.stkd = reinterpret_cast<float*>(stk + (size_t)blob.stack_depth * blockDim.x) + threadIdx.x;
    sv.stk_stride = (int)blockDim.x;
    sv.stk_depth = blob.stack_depth;
    return true;
}

#define IFX_SCENE_PROLOGUE(blob, status, sv)                                  \
    extern __shared__ __align__(128) uint8_t ifx_dsmem[];                     \
    __shared__ __align__(8) uint64_t ifx_mbar;                                \
    SceneView sv;                                                             \
    if (!scene_prologue(blob, ifx_dsmem, &ifx_mbar, status, sv)) return;

// Bounded grid barrier over the CTAs of one cooperative launch (every CTA is
// resident, so all of them arrive unless one has left after an error).
// Returns false, with kStatusBarrier set in *status, when the other CTAs did
// not arrive within `polls` polls; the caller then leaves the kernel. The
// barrier's count must be zero at launch.
static constexpr uint32_t kStatusBarrier = 1u << 4;
__device__ __forceinline__ bool grid_barrier(MsBarrier* b, uint32_t* status, uint32_t polls) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile uint32_t* vgen = &b->gen;
        const uint32_t g = *vgen;
        __threadfence();
        if (atomicAdd(&b->count, 1u) == gridDim.x - 1) {
            atomicExch(&b->count, 0u);
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            uint32_t n = 0;
            while (*vgen == g) {
                if (++n > polls) {
                    atomicOr(status, kStatusBarrier);
                    ok = 0;
                    break;
                }
                __nanosleep(128);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// Number of CTAs for a grid-stride kernel: enough to fill every SM several
// times over, never more than the work needs.
static inline int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cached[dev]) {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = sms;
    }
    return cached[dev];
}

static inline unsigned grid_for(unsigned long long items, int block, int per_sm_ctas = 8) {
    unsigned long long need = (items + (unsigned long long)block - 1) / (unsigned long long)block;
    unsigned long long cap = (unsigned long long)sm_count() * (unsigned long long)per_sm_ctas;
    if (need < 1) need = 1;
    return (unsigned)(need < cap ? need : cap);
}

// Persistent kernels: one wave of CTAs, as many as are co-resident.
template <class K>
static inline unsigned persistent_grid(K kernel, int block, size_t smem, unsigned long long items) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem);
    if (per_sm < 1) per_sm = 1;
    unsigned long long cap = (unsigned long long)sm_count() * (unsigned long long)per_sm;
    unsigned long long need = (items + (unsigned long long)block - 1) / (unsigned long long)block;
    if (need < 1) need = 1;
    return (unsigned)(need < cap ? need : cap);
}

// Warp-level work distribution for persistent ray kernels. Every lane holds
// at most one item (a ray); lanes whose ray finished are refilled from the
// warp's private range of item indices, which is replenished in chunks of
// kChunk indices from a global cursor with one atomic per chunk. Which lane
// or warp traces an item never affects its result: each item's output is
// written to a slot fixed by its index.
struct WarpQueue {
    uint32_t cur, end;  // warp-uniform private range [cur, end)
    uint32_t kChunk;    // items taken per atomic: about 1/8 of a fair share per warp, 32..256
    bool drained;

    __device__ __forceinline__ WarpQueue() : cur(0), end(0), kChunk(32), drained(false) {}
    __device__ __forceinline__ explicit WarpQueue(unsigned long long total) : cur(0), end(0), drained(false) {
        const unsigned long long warps = (unsigned long long)gridDim.x * blockDim.x / 32u;
        unsigned long long c = total / (warps * 8ull + 1ull);
        c = c < 32ull ? 32ull : (c > 256ull ? 256ull : c);
        kChunk = (uint32_t)(c & ~31ull);
    }

    // Returns the item for this lane (or ~0u) when it is idle; `idle` says
    // whether this lane needs an item. Must be called by all 32 lanes.
    __device__ __forceinline__ uint32_t refill(bool idle, unsigned long long total, unsigned long long* cursor) {
        const int lane = threadIdx.x & 31;
        unsigned need = __ballot_sync(kFull, idle);
        uint32_t item = ~0u;
        if (!need) return item;
        if (cur >= end && !drained) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(cursor, (unsigned long long)kChunk);
            base = __shfl_sync(kFull, base, 0);
            if (base >= total) {
                drained = true;
            } else {
                cur = (uint32_t)base;
                end = (uint32_t)(base + kChunk < total ? base + kChunk : total);
            }
        }
        if (cur < end) {
            uint32_t avail = end - cur;
            uint32_t rank = __popc(need & ((1u << lane) - 1u));
            if (idle && rank < avail) item = cur + rank;
            uint32_t k = __popc(need);
            cur += k < avail ? k : avail;
        }
        return item;
    }
    __device__ __forceinline__ bool empty() const { return drained && cur >= end; }
};

}  // namespace ifx
