// The Jacobi solve for callers that cannot allocate GPU memory.
//
// ifx_solve (capi.cu) keeps its scratch (the per-cluster radiosity vector
// and the convergence control block) in buffers its context allocates. Some
// host programs cannot let a library call cudaMalloc: an engine that
// reserves the whole device up front and hands out memory only from its own
// arena, a frame loop that must not stall on cudaMalloc's implicit device
// synchronisation, or a binding whose allocations are owned by another
// runtime. ifx_solve_noalloc serves them: it runs the same bounce kernels on
// device buffers the caller owns, and takes its scratch from one
// statically sized array compiled into this library.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/interflect.h"
#include "kernels.h"

namespace {

// Scratch: cluster radiosity (one float4 per cluster) followed by the
// control block. Every GPU that loads the library holds these bytes
// (IFX_NOALLOC_MAX_CLUSTERS * 16 + 256) until the process exits.
constexpr size_t kScratchBytes = (size_t)IFX_NOALLOC_MAX_CLUSTERS * 16u + 256u;
static __device__ __align__(256) unsigned char g_solve_scratch[kScratchBytes];

// The array's device address, looked up once per device. In host code the
// symbol g_solve_scratch is a host-side stand-in, never a device address.
std::mutex g_mu;
void* g_addr[64] = {nullptr};

int scratch_for(int device, void** out, char* err, size_t errlen) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (device < 0 || device >= 64) return IFX_ERR_INVALID;
    if (!g_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_solve_scratch);
        if (e != cudaSuccess || !p) {
            if (err && errlen) snprintf(err, errlen, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            cudaGetLastError();
            return IFX_ERR_CUDA;
        }
        g_addr[device] = p;
    }
    *out = g_addr[device];
    return IFX_OK;
}

void put_err(char* err, size_t errlen, const char* msg) {
    if (err && errlen) snprintf(err, errlen, "%s", msg);
}

bool aligned(const void* p, uintptr_t a) { return ((uintptr_t)p & (a - 1)) == 0; }

// Puts the caller's current device back when the call returns, whichever
// way it returns: the entry point selects `device` only for its own work.
struct DeviceRestore {
    int prev = -1;
    ~DeviceRestore() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" int ifx_solve_noalloc(int device, void* stream, uint32_t n, uint32_t nc, const float* p_area4,
                                 const float* direct4, const float* albedo4, float* irr4, float* rad4,
                                 const float* cluster_p_area4, const uint32_t* cluster_ranges,
                                 const uint32_t* members, const uint32_t* starts, const uint32_t* idx,
                                 const float* w, uint32_t max_bounces, ifx_solve_stats* out, char* err,
                                 size_t errlen) {
    if (!out) {
        put_err(err, errlen, "null stats pointer");
        return IFX_ERR_INVALID;
    }
    out->iterations = 0;
    out->residual = 0.0f;
    if (nc > IFX_NOALLOC_MAX_CLUSTERS) {
        char m[160];
        snprintf(m, sizeof m, "%u clusters exceed the %u this entry point's static scratch holds", nc,
                 (unsigned)IFX_NOALLOC_MAX_CLUSTERS);
        put_err(err, errlen, m);
        return IFX_ERR_LIMIT;
    }
    if (nc == 0) return IFX_OK;  // solve.rs:49-55
    if (!p_area4 || !direct4 || !albedo4 || !irr4 || !rad4 || !cluster_p_area4 || !cluster_ranges || !members ||
        !starts || (!idx && n) || (!w && n)) {
        put_err(err, errlen, "null device pointer");
        return IFX_ERR_INVALID;
    }
    // The kernels read the float4 arrays with 16-byte loads and the cluster
    // ranges with 8-byte loads; a misaligned pointer (an arena offset aligned
    // to less) would fault inside a kernel and poison the caller's context,
    // so it is refused here, before anything is launched.
    if (!aligned(p_area4, 16) || !aligned(direct4, 16) || !aligned(albedo4, 16) || !aligned(irr4, 16) ||
        !aligned(rad4, 16) || !aligned(cluster_p_area4, 16) || !aligned(cluster_ranges, 8) ||
        !aligned(members, 4) || !aligned(starts, 4) || !aligned(idx, 4) || !aligned(w, 4)) {
        put_err(err, errlen,
                "misaligned device pointer: float4 arrays need 16-byte, cluster_ranges 8-byte and the index and "
                "weight arrays 4-byte alignment");
        return IFX_ERR_INVALID;
    }
    DeviceRestore restore;
    cudaError_t e = cudaGetDevice(&restore.prev);
    if (e == cudaSuccess) e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        put_err(err, errlen, cudaGetErrorString(e));
        return IFX_ERR_CUDA;
    }
    void* base = nullptr;
    int r = scratch_for(device, &base, err, errlen);
    if (r != IFX_OK) return r;
    cudaStream_t st = (cudaStream_t)stream;
    float4* cluster_rad = (float4*)base;
    ifx::SolveCtl* ctl = (ifx::SolveCtl*)((unsigned char*)base + (size_t)IFX_NOALLOC_MAX_CLUSTERS * 16u);
    // The control block must start at zero; the radiosity vector is fully
    // rewritten by every bounce before it is read.
    e = cudaMemsetAsync(ctl, 0, sizeof(ifx::SolveCtl), st);
    if (e != cudaSuccess) {
        put_err(err, errlen, cudaGetErrorString(e));
        return IFX_ERR_CUDA;
    }
    ifx::SurfelArrays s{(float4*)p_area4, nullptr, (float4*)albedo4, (float4*)direct4, (float4*)irr4,
                        (float4*)rad4};
    ifx::SolveCtl h{};
    const uint32_t kBatch = 16;
    for (uint32_t it = 0; it < max_bounces;) {
        uint32_t end = it + kBatch < max_bounces ? it + kBatch : max_bounces;
        for (; it < end; ++it) {
            int l = 0;
            ifx::launch_solve_bounce(st, s, n, (const float4*)cluster_p_area4, (const uint2*)cluster_ranges, members,
                                     nc, starts, idx, w, cluster_rad, ctl, it, &l);
        }
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h, ctl, sizeof h, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            put_err(err, errlen, cudaGetErrorString(e));
            return IFX_ERR_CUDA;
        }
        if (h.done) break;
    }
    out->iterations = h.iterations;
    memcpy(&out->residual, &h.last_residual, 4);
    return IFX_OK;
}
