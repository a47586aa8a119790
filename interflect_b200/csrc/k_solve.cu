// Direct light on surfels (solve.rs:27-39; for many (surfel, light) slots
// the light stage uses launch_light_slots in k_shade.cu instead) and the
// Jacobi bounce solve (solve.rs:47-108). The bounce loop runs without host round trips: every
// bounce kernel first reads a device-side `done` flag, so the host enqueues
// max_bounces bounces at once and the ones after convergence return
// immediately.
#include "kcommon.cuh"

namespace ifx {

// Programmatic dependent launch between the bounce kernels: a kernel starts
// by waiting until the previous kernel in its stream has completed and its
// writes are visible (pdl_wait), and once its main loop is done it lets the
// next kernel be scheduled (pdl_trigger), whose CTAs then wait in their own
// pdl_wait. Both are no-ops in a launch without the programmatic attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ void block_add_u64(unsigned long long v, unsigned long long* out) {
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(out, v);
}

// solve.rs:27-39
template <class C>
__global__ void __launch_bounds__(128) k_light_surfels(BlobRef blob, SurfelArrays s, uint32_t n,
                                                        unsigned long long* evals, uint32_t* status,
                                                        unsigned long long* counts, float* terms) {
    IFX_SCENE_PROLOGUE(blob, status, sv);
    C cnt;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t limit = (n + stride - 1) / stride * stride;  // keep whole warps for the reduction
    const int nl = sv.n_lights + sv.n_slights;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < limit; i += stride) {
        unsigned long long e = 0;
        if (i < n) {
            uint32_t steps = 0;
            V c = direct_diffuse(sv, mk4(s.p[i]), mk4(s.n[i]), mk4(s.albedo[i]), steps, cnt,
                                 terms ? terms + (size_t)i * nl : nullptr);
            s.direct[i] = f4(c, 0.0f);
            s.rad[i] = f4(c, 0.0f);
            s.irr[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            e = steps;
        }
        block_add_u64(e, evals);
    }
    if constexpr (sizeof(C) > 1) cnt.flush(counts);
}

// solve.rs:61-73: cluster radiosity as the area-weighted mean of its
// members' radiosity, summed sequentially in member order, by one CTA: the
// threads gather members' rad * area (each product exact per element) into
// shared memory chunk by chunk, double-buffered, and thread 0 adds them in
// member order.
template <int kBlock>
__device__ __forceinline__ void cluster_mean(const float4* rad, const float4* sp, const float4* cp,
                                             const uint2* crange, const uint32_t* members, uint32_t c,
                                             float4* cluster_rad, float4 (*buf)[kBlock]) {
    const uint2 r = crange[c];
    const uint32_t len = r.y - r.x;
    const uint32_t chunks = (len + kBlock - 1) / kBlock;
    auto load = [&](uint32_t ch, int b) {
        uint32_t k = r.x + ch * kBlock + threadIdx.x;
        if (k < r.y) {
            uint32_t m = __ldg(&members[k]);
            float4 v = __ldg(&rad[m]);
            float a = __ldg(&sp[m].w);
            buf[b][threadIdx.x] = make_float4(v.x * a, v.y * a, v.z * a, 0.0f);
        }
    };
    if (chunks) load(0, 0);
    __syncthreads();
    V acc{0.0f, 0.0f, 0.0f};
    for (uint32_t ch = 0; ch < chunks; ++ch) {
        const int b = ch & 1;
        if (threadIdx.x == 0) {
            const uint32_t cnt = min((uint32_t)kBlock, len - ch * kBlock);
            // Unrolled so that the shared-memory loads run ahead of the
            // chain of additions (which stays in member order).
            uint32_t k = 0;
            for (; k + 8 <= cnt; k += 8) {
                float4 v[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) v[j] = buf[b][k + j];
#pragma unroll
                for (int j = 0; j < 8; ++j) acc = acc + V{v[j].x, v[j].y, v[j].z};
            }
            for (; k < cnt; ++k) {
                float4 v = buf[b][k];
                acc = acc + V{v.x, v.y, v.z};
            }
            if (ch + 1 < chunks) load(ch + 1, b ^ 1);
        } else if (ch + 1 < chunks) {
            load(ch + 1, b ^ 1);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) cluster_rad[c] = f4(acc / fmaxf(__ldg(&cp[c].w), 1e-12f), 0.0f);
    __syncthreads();
}

static constexpr int kAggBlock = 128;
__global__ void __launch_bounds__(kAggBlock) k_cluster_agg(const float4* rad, const float4* sp, const float4* cp,
                                                            const uint2* crange, const uint32_t* members,
                                                            uint32_t nc, float4* cluster_rad, const SolveCtl* ctl) {
    pdl_wait();
    if (ctl->done) return;
    __shared__ float4 buf[2][kAggBlock];
    for (uint32_t c = blockIdx.x; c < nc; c += gridDim.x)
        cluster_mean<kAggBlock>(rad, sp, cp, crange, members, c, cluster_rad, buf);
    pdl_trigger();
}

// solve.rs:76-102: one Jacobi row per thread, its links added in CSR order
// (the reference's sum). Each iteration of the row loop issues the index and
// weight loads of 8 links as two 128-bit loads each, then the 8 cluster
// gathers, before the first add, so a thread keeps 12 loads in flight; the
// products crad[idx] * w and their left-to-right sum round exactly as the
// scalar loop does. `vec` is 0 when idx or w is not 16-byte aligned (caller-
// provided arrays), which keeps every load scalar. The bounce residual is the
// maximum change over rows, an order-free reduction kept as the bits of a
// non-negative f32 (NaN ignored, as the reference's f32::max fold does).
static constexpr int kJacBlock = 256;
__device__ __forceinline__ V jacobi_row(const float4* crad, const uint32_t* __restrict__ idx,
                                        const float* __restrict__ w, uint32_t k, uint32_t e, int vec) {
    V irr{0.0f, 0.0f, 0.0f};
    if (vec) {
        for (; k < e && (k & 3u); ++k) irr = irr + mk4(__ldg(&crad[__ldg(&idx[k])])) * __ldg(&w[k]);
        for (; k + 8 <= e; k += 8) {
            const uint4 i0 = __ldg(reinterpret_cast<const uint4*>(idx + k));
            const uint4 i1 = __ldg(reinterpret_cast<const uint4*>(idx + k + 4));
            const float4 w0 = __ldg(reinterpret_cast<const float4*>(w + k));
            const float4 w1 = __ldg(reinterpret_cast<const float4*>(w + k + 4));
            const float4 c0 = __ldg(&crad[i0.x]), c1 = __ldg(&crad[i0.y]),
                         c2 = __ldg(&crad[i0.z]), c3 = __ldg(&crad[i0.w]),
                         c4 = __ldg(&crad[i1.x]), c5 = __ldg(&crad[i1.y]),
                         c6 = __ldg(&crad[i1.z]), c7 = __ldg(&crad[i1.w]);
            irr = irr + mk4(c0) * w0.x;
            irr = irr + mk4(c1) * w0.y;
            irr = irr + mk4(c2) * w0.z;
            irr = irr + mk4(c3) * w0.w;
            irr = irr + mk4(c4) * w1.x;
            irr = irr + mk4(c5) * w1.y;
            irr = irr + mk4(c6) * w1.z;
            irr = irr + mk4(c7) * w1.w;
        }
    }
    for (; k < e; ++k) irr = irr + mk4(__ldg(&crad[__ldg(&idx[k])])) * __ldg(&w[k]);
    return irr;
}

// The CSR row i of one bounce: irradiance, new radiosity, |change|.
__device__ __forceinline__ float csr_row_update(float4* direct, float4* albedo, float4* irr_out, float4* rad,
                                                const uint32_t* starts, const uint32_t* idx, const float* w,
                                                const float4* cluster_rad, int vec, uint32_t i) {
    const V irr = jacobi_row(cluster_rad, idx, w, starts[i], starts[i + 1], vec);
    V nr = mk4(__ldg(&direct[i])) + mk4(__ldg(&albedo[i])) * irr;
    V diff = vabs(nr - mk4(rad[i]));
    irr_out[i] = f4(irr, 0.0f);
    rad[i] = f4(nr, 0.0f);
    return fmaxf(diff.x, fmaxf(diff.y, diff.z));
}

__global__ void __launch_bounds__(kJacBlock) k_jacobi(float4* direct, float4* albedo, float4* irr_out, float4* rad,
                                                       uint32_t n, const uint32_t* starts, const uint32_t* idx,
                                                       const float* w, const float4* cluster_rad, SolveCtl* ctl,
                                                       int vec) {
    pdl_wait();
    if (ctl->done) return;
    float dmax = 0.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float d = csr_row_update(direct, albedo, irr_out, rad, starts, idx, w, cluster_rad, vec, i);
        if (!isnan(d)) dmax = fmaxf(dmax, d);
    }
    pdl_trigger();
    for (int o = 16; o >= 1; o >>= 1) dmax = fmaxf(dmax, __shfl_xor_sync(kFull, dmax, o));
    if ((threadIdx.x & 31) == 0 && dmax > 0.0f) atomicMax(&ctl->residual_bits, __float_as_uint(dmax));
}

// solve.rs:454-462; no_exit keeps every bounce running (fixed bounce count).
__global__ void k_bounce_end(SolveCtl* ctl, uint32_t it, int no_exit) {
    pdl_wait();
    pdl_trigger();
    if (ctl->done) return;
    float res = __uint_as_float(ctl->residual_bits);
    ctl->iterations = it + 1;
    ctl->last_residual = ctl->residual_bits;
    ctl->residual_bits = 0;
    if (res < 1e-4f && !no_exit) ctl->done = 1;
}

void launch_light_surfels(cudaStream_t st, BlobRef blob, SurfelArrays s, uint32_t n, unsigned long long* evals,
                          uint32_t* status, unsigned long long* counts, float* terms) {
    const unsigned g = grid_for(n, 128, 16);
    if (counts)
        k_light_surfels<Counts><<<g, 128, blob_smem(blob, 128), st>>>(blob, s, n, evals, status, counts, terms);
    else if (blob.tree3)
        k_light_surfels<NoCount3><<<g, 128, blob_smem(blob, 128), st>>>(blob, s, n, evals, status, nullptr, terms);
    else
        k_light_surfels<NoCount><<<g, 128, blob_smem(blob, 128), st>>>(blob, s, n, evals, status, nullptr, terms);
}

// solve.rs:76-102 over the sliced-ELL copy: one thread per sorted position
// (its warp is its slice), the row's links read 4 at a time as 128-bit loads
// from the interleaved layout (a warp's loads are one contiguous 512-byte
// block) and added in CSR order, exactly as k_jacobi; a lane stops at its own
// row's length, so padding is never read. Outputs go to the original row.
__device__ __forceinline__ float sell_row_update(float4* direct, float4* albedo, float4* irr_out, float4* rad,
                                                 const SellMatrix& m, const float4* crad, uint32_t sp) {
    const uint32_t row = m.perm[sp], len = m.len[sp];
    const uint32_t* ip = m.idx + m.slice_off[sp >> 5] + (sp & 31u) * 4u;
    const float* wp = m.w + m.slice_off[sp >> 5] + (sp & 31u) * 4u;
    V irr{0.0f, 0.0f, 0.0f};
    uint32_t j = 0;
    for (; j + 8 <= len; j += 8, ip += 256, wp += 256) {
        const uint4 i0 = __ldg(reinterpret_cast<const uint4*>(ip));
        const uint4 i1 = __ldg(reinterpret_cast<const uint4*>(ip + 128));
        const float4 w0 = __ldg(reinterpret_cast<const float4*>(wp));
        const float4 w1 = __ldg(reinterpret_cast<const float4*>(wp + 128));
        const float4 c0 = __ldg(&crad[i0.x]), c1 = __ldg(&crad[i0.y]),
                     c2 = __ldg(&crad[i0.z]), c3 = __ldg(&crad[i0.w]),
                     c4 = __ldg(&crad[i1.x]), c5 = __ldg(&crad[i1.y]),
                     c6 = __ldg(&crad[i1.z]), c7 = __ldg(&crad[i1.w]);
        irr = irr + mk4(c0) * w0.x;
        irr = irr + mk4(c1) * w0.y;
        irr = irr + mk4(c2) * w0.z;
        irr = irr + mk4(c3) * w0.w;
        irr = irr + mk4(c4) * w1.x;
        irr = irr + mk4(c5) * w1.y;
        irr = irr + mk4(c6) * w1.z;
        irr = irr + mk4(c7) * w1.w;
    }
    if (j < len) {
        const uint4 i0 = __ldg(reinterpret_cast<const uint4*>(ip));
        const float4 w0 = __ldg(reinterpret_cast<const float4*>(wp));
        const uint32_t ia[4] = {i0.x, i0.y, i0.z, i0.w};
        const float wa[4] = {w0.x, w0.y, w0.z, w0.w};
        const uint32_t r4 = len - j < 4u ? len - j : 4u;
        for (uint32_t t = 0; t < r4; ++t) irr = irr + mk4(__ldg(&crad[ia[t]])) * wa[t];
        j += r4;
        if (j < len) {
            ip += 128;
            wp += 128;
            const uint4 i1 = __ldg(reinterpret_cast<const uint4*>(ip));
            const float4 w1 = __ldg(reinterpret_cast<const float4*>(wp));
            const uint32_t ib[4] = {i1.x, i1.y, i1.z, i1.w};
            const float wb[4] = {w1.x, w1.y, w1.z, w1.w};
            for (uint32_t t = 0; t < len - j; ++t) irr = irr + mk4(__ldg(&crad[ib[t]])) * wb[t];
        }
    }
    V nr = mk4(__ldg(&direct[row])) + mk4(__ldg(&albedo[row])) * irr;
    V diff = vabs(nr - mk4(rad[row]));
    irr_out[row] = f4(irr, 0.0f);
    rad[row] = f4(nr, 0.0f);
    return fmaxf(diff.x, fmaxf(diff.y, diff.z));
}

__global__ void __launch_bounds__(kJacBlock) k_jacobi_sell(float4* direct, float4* albedo, float4* irr_out,
                                                            float4* rad, uint32_t n, SellMatrix m,
                                                            const float4* __restrict__ crad, SolveCtl* ctl) {
    pdl_wait();
    if (ctl->done) return;
    float dmax = 0.0f;
    for (uint32_t sp = blockIdx.x * blockDim.x + threadIdx.x; sp < n; sp += gridDim.x * blockDim.x) {
        const float d = sell_row_update(direct, albedo, irr_out, rad, m, crad, sp);
        if (!isnan(d)) dmax = fmaxf(dmax, d);
    }
    pdl_trigger();
    for (int o = 16; o >= 1; o >>= 1) dmax = fmaxf(dmax, __shfl_xor_sync(kFull, dmax, o));
    if ((threadIdx.x & 31) == 0 && dmax > 0.0f) atomicMax(&ctl->residual_bits, __float_as_uint(dmax));
}

// A bounce kernel launched with the programmatic-serialization attribute:
// the stream (or the captured graph's edge) lets it start once the previous
// kernel has triggered, and pdl_wait orders its work after that kernel.
template <typename... K, typename... A>
static void launch_pdl(void (*kernel)(K...), unsigned grid, unsigned block, cudaStream_t st, A... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

void launch_solve_bounce(cudaStream_t st, SurfelArrays s, uint32_t n, const float4* cp, const uint2* crange,
                         const uint32_t* members, uint32_t nc, const uint32_t* starts, const uint32_t* idx,
                         const float* w, float4* cluster_rad, SolveCtl* ctl, uint32_t it, int* launches,
                         int no_exit, const SellMatrix* sell) {
    launch_pdl(k_cluster_agg, nc < 4096u ? nc : 4096u, kAggBlock, st, (const float4*)s.rad, (const float4*)s.p, cp,
               crange, members, nc, cluster_rad, (const SolveCtl*)ctl);
    if (sell && sell->perm) {
        launch_pdl(k_jacobi_sell, grid_for(n, kJacBlock), kJacBlock, st, s.direct, s.albedo, s.irr, s.rad, n, *sell,
                   (const float4*)cluster_rad, ctl);
    } else {
        const int vec = (((uintptr_t)idx | (uintptr_t)w) & 15u) == 0 ? 1 : 0;
        launch_pdl(k_jacobi, grid_for(n, kJacBlock), kJacBlock, st, s.direct, s.albedo, s.irr, s.rad, n, starts, idx,
                   w, (const float4*)cluster_rad, ctl, vec);
    }
    launch_pdl(k_bounce_end, 1u, 1u, st, ctl, it, no_exit);
    *launches += 3;
}

// ------------------------------------------------- sliced-ELL assembly ---
__global__ void k_sell_lens(const uint32_t* starts, uint32_t n, uint32_t* lens, uint32_t* rows) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        lens[i] = starts[i + 1] - starts[i];
        rows[i] = i;
    }
}

// Entries of slice k: 32 lanes x its longest row rounded up to 4 (rows are
// sorted by length, so that is the slice's first row).
__global__ void k_sell_sizes(const uint32_t* sorted_len, uint32_t n, uint32_t* sizes) {
    const uint32_t ns = (n + 31) / 32;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= ns; k += gridDim.x * blockDim.x)
        sizes[k] = k < ns ? 32u * ((sorted_len[32 * k] + 3u) & ~3u) : 0u;
}

__global__ void k_sell_fill(const uint32_t* starts, const uint32_t* idx, const float* w, uint32_t n,
                            const uint32_t* perm, const uint32_t* sorted_len, const uint32_t* slice_off,
                            uint32_t* sidx, float* sw) {
    for (uint32_t sp = blockIdx.x * blockDim.x + threadIdx.x; sp < n; sp += gridDim.x * blockDim.x) {
        const uint32_t s0 = starts[perm[sp]], len = sorted_len[sp];
        const uint32_t base = slice_off[sp >> 5] + (sp & 31u) * 4u;
        for (uint32_t j = 0; j < len; ++j) {
            const uint32_t q = base + (j >> 2) * 128u + (j & 3u);
            sidx[q] = idx[s0 + j];
            sw[q] = w[s0 + j];
        }
    }
}

int launch_sell_lens(cudaStream_t st, const uint32_t* starts, uint32_t n, uint32_t* lens, uint32_t* rows) {
    k_sell_lens<<<grid_for(n, 256), 256, 0, st>>>(starts, n, lens, rows);
    return 1;
}
int launch_sell_sizes(cudaStream_t st, const uint32_t* sorted_len, uint32_t n, uint32_t* sizes) {
    k_sell_sizes<<<grid_for((unsigned long long)(n + 31) / 32 + 1, 256), 256, 0, st>>>(sorted_len, n, sizes);
    return 1;
}
int launch_sell_fill(cudaStream_t st, const uint32_t* starts, const uint32_t* idx, const float* w, uint32_t n,
                     const uint32_t* perm, const uint32_t* sorted_len, const uint32_t* slice_off, uint32_t* sidx,
                     float* sw) {
    k_sell_fill<<<grid_for(n, 256), 256, 0, st>>>(starts, idx, w, n, perm, sorted_len, slice_off, sidx, sw);
    return 1;
}

void configure_solve_kernels(int max_dyn_smem) {
    cudaFuncSetAttribute(k_light_surfels<NoCount>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_light_surfels<NoCount3>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_light_surfels<Counts>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
}

}  // namespace ifx
