// Shared kernel prologue: make the scene program visible to the CTA.
#pragma once

#include "device.cuh"
#include "kernels.h"

namespace ifx {

// Stages the blob into dynamic shared memory (one bulk copy) or, for large
// scenes, reads it in place. All threads of the CTA must call this before
// any of them exits. Returns false if staging timed out.
__device__ __forceinline__ bool scene_prologue(const BlobRef& blob, uint8_t* dsmem, uint64_t* mbar,
                                               uint32_t* status, SceneView& sv) {
    const uint8_t* base = blob.ptr;
    if (blob.staged) {
        if (!stage_scene(blob.ptr, blob.bytes, dsmem, mbar, status)) return false;
        base = dsmem;
    }
    sv = make_view(base);
    return true;
}

#define IFX_SCENE_PROLOGUE(blob, status, sv)                                  \
    extern __shared__ __align__(128) uint8_t ifx_dsmem[];                     \
    __shared__ __align__(8) uint64_t ifx_mbar;                                \
    SceneView sv;                                                             \
    if (!scene_prologue(blob, ifx_dsmem, &ifx_mbar, status, sv)) return;

static inline size_t blob_smem(const BlobRef& b) { return b.staged ? b.bytes : 0; }

static constexpr int kWarp = 32;
static constexpr unsigned kFull = 0xffffffffu;

// Number of CTAs for a grid-stride kernel: enough to fill every SM several
// times over, never more than the work needs.
static inline unsigned grid_for(unsigned long long items, int block, int per_sm_ctas = 8) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    unsigned long long need = (items + (unsigned long long)block - 1) / (unsigned long long)block;
    unsigned long long cap = (unsigned long long)sms * (unsigned long long)per_sm_ctas;
    if (need < 1) need = 1;
    return (unsigned)(need < cap ? need : cap);
}

}  // namespace ifx
