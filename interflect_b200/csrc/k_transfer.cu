// Transfer build (formfactor.rs:153-277) as a deterministic pipeline:
//   pair count -> scan -> pair fill      candidate (row, cluster) pairs in
//                                        cluster order within each row
//   visibility                           one cone-traced soft shadow per pair
//   closure                              16 hemisphere rays per row
//   row finalize -> scan -> row fill     link test, ordered row sum,
//                                        calibration, CSR in row order
// Nothing depends on scheduling: every value lands at an index fixed by the
// scans, and the only float reductions (row sums) run sequentially in the
// reference's order.
#include "kcommon.cuh"

namespace ifx {

// formfactor.rs:169-192: facing test and Nusselt disc form factor with the
// 2e-5 cull. Returns ff, or -1 when the pair is culled.
__device__ __forceinline__ float pair_ff(V sp, V sn, float4 cp, float4 cn) {
    V d = mk4(cp) - sp;
    float r2 = dot(d, d);
    if (r2 < 1e-9f) return -1.0f;
    float r = sqrtf(r2);
    V dir = d / r;
    float cos_i = dot(sn, dir);
    float cos_c = dot(mk4(cn), -dir);
    if (cos_i <= 1e-3f || cos_c <= 1e-3f) return -1.0f;
    float ff = cos_i * cos_c * cp.w / (kPiF * r2 + cp.w);
    if (ff < 2e-5f) return -1.0f;
    return ff;
}

// One warp per surfel row; lanes stride over clusters.
__global__ void __launch_bounds__(256) k_pair_count(const float4* sp, const float4* sn, uint32_t n,
                                                     const float4* cp, const float4* cn, uint32_t nc,
                                                     unsigned long long* cand_count) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += warps) {
        V p = mk4(sp[row]), nn = mk4(sn[row]);
        uint32_t cnt = 0;
        for (uint32_t c0 = 0; c0 < nc; c0 += 32) {
            uint32_t c = c0 + lane;
            bool pass = c < nc && pair_ff(p, nn, __ldg(&cp[c]), __ldg(&cn[c])) >= 0.0f;
            cnt += __popc(__ballot_sync(kFull, pass));
        }
        if (lane == 0) cand_count[row] = cnt;
    }
}

__global__ void __launch_bounds__(256) k_pair_fill(const float4* sp, const float4* sn, uint32_t n,
                                                    const float4* cp, const float4* cn, uint32_t nc,
                                                    const unsigned long long* cand_off, uint32_t* cand_c,
                                                    float* cand_ff, uint32_t* cand_row) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += warps) {
        V p = mk4(sp[row]), nn = mk4(sn[row]);
        unsigned long long at = cand_off[row];
        for (uint32_t c0 = 0; c0 < nc; c0 += 32) {
            uint32_t c = c0 + lane;
            float ff = c < nc ? pair_ff(p, nn, __ldg(&cp[c]), __ldg(&cn[c])) : -1.0f;
            unsigned mask = __ballot_sync(kFull, ff >= 0.0f);
            if (ff >= 0.0f) {
                unsigned long long j = at + __popc(mask & ((1u << lane) - 1u));
                cand_c[j] = c;
                cand_ff[j] = ff;
                cand_row[j] = row;
            }
            at += __popc(mask);
        }
    }
}

// formfactor.rs:194-205: the visibility cone of one candidate pair.
// Persistent: each lane marches one candidate's cone one SDF query per
// iteration and takes a new candidate from its warp's queue when the cone
// ends, so a warp stays full however uneven the cones' lengths are. The
// queue walks `order` (nullable: candidate order), a permutation grouping
// candidates by target cluster and then by the source surfel's cluster, so
// that a warp marches nearly parallel cones from neighbouring surfels; every
// result is written to its candidate's own slot.
template <class C>
__global__ void __launch_bounds__(128) k_visibility(BlobRef blob, SceneConsts sc, const float4* sp,
                                                     const float4* sn, const float4* cp, const float4* cn,
                                                     const uint32_t* cand_c, const uint32_t* cand_row,
                                                     const uint32_t* order, unsigned long long ncand,
                                                     float* cand_vis, uint8_t* cand_steps, uint32_t* status,
                                                     unsigned long long* counts, unsigned long long* cursor) {
    IFX_SCENE_PROLOGUE(blob, status, sv);
    C cnt;
    WarpQueue q(ncand);
    const float off = sc.diag * 5e-4f, tmin = sc.diag * 1e-3f;
    uint32_t item = ~0u;
    ShadowRay ray{};
    while (true) {
        uint32_t got = q.refill(item == ~0u, ncand, cursor);
        if (got != ~0u) {
            if (order) got = order[got];
            const uint32_t row = cand_row[got], c = cand_c[got];
            const V p = mk4(__ldg(&sp[row])), nn = mk4(__ldg(&sn[row]));
            const float4 cpc = __ldg(&cp[c]), cnc = __ldg(&cn[c]);
            V d = mk4(cpc) - p;
            float r = sqrtf(dot(d, d));
            V dir = d / r;
            float k = clampr(r / fmaxf(cnc.w, 1e-4f), 1.5f, 32.0f);
            ray = shadow_begin(p + nn * off, dir, tmin, r - cnc.w * 0.75f, k);
            if (shadow_done_before_start(ray)) {
                cand_vis[got] = clampr(ray.res, 0.0f, 1.0f);
                cand_steps[got] = 0;
            } else {
                item = got;
            }
        }
        if (!__any_sync(kFull, item != ~0u)) {
            if (q.empty()) break;
            continue;
        }
        const bool active = item != ~0u;
        float vis;
        if (shadow_step_w(sv, ray, active, vis, cnt) && active) {
            cand_vis[item] = vis;
            cand_steps[item] = (uint8_t)ray.steps;
            item = ~0u;
        }
    }
    if constexpr (sizeof(C) > 1) cnt.flush(counts);
}

// trace.rs:165-186: one persistent lane per hemisphere ray (16 per row);
// each ray's result is written to its own slot as (open << 8) | steps and
// k_row_finalize reduces the row's 16 slots. The queue walks `order`
// (nullable: item order), which groups rays by the row's cluster and then
// by direction, so a warp marches nearly parallel rays from neighbouring
// surfels. A hit's normal is never used
// here, so it is not computed, but its four taps are still counted
// (trace.rs:48).
template <class C>
__global__ void __launch_bounds__(128) k_closure(BlobRef blob, SceneConsts sc, const float4* sp,
                                                  const float4* sn, uint32_t n, const uint32_t* order, uint16_t* clo,
                                                  uint32_t* status, unsigned long long* counts,
                                                  unsigned long long* cursor) {
    IFX_SCENE_PROLOGUE(blob, status, sv);
    C cnt;
    const unsigned long long total = (unsigned long long)n * 16ull;
    WarpQueue q(total);
    const float tmax = sc.diag * 2.0f;
    uint32_t item = ~0u;
    TraceRay ray{};
    while (true) {
        uint32_t got = q.refill(item == ~0u, total, cursor);
        if (got != ~0u) {
            if (order) got = order[got];
            const uint32_t row = got >> 4, k = got & 15u;
            const V p = mk4(__ldg(&sp[row])), nn = mk4(__ldg(&sn[row]));
            V t, b;
            frame(nn, t, b);
            V d = t * sc.closure[k][0] + b * sc.closure[k][1] + nn * sc.closure[k][2];
            ray = TraceRay{p + nn * 1e-3f, nrm(d), 1e-3f, tmax, 0u};
            item = got;
        }
        if (!__any_sync(kFull, item != ~0u)) {
            if (q.empty()) break;
            continue;
        }
        const bool active = item != ~0u;
        const int st = trace_step_dist_w(sv, ray, active, cnt);
        if (active && st != kMarching) {
            clo[item] = (uint16_t)(((st == kMiss) ? 0x100u : 0u) | ray.steps);
            item = ~0u;
        }
    }
    if constexpr (sizeof(C) > 1) cnt.flush(counts);
}

// formfactor.rs:206-238: links are pairs with vis > 1e-3, weighted ff*vis,
// summed in cluster order; the row is rescaled to 1 - sky (capped at 8x)
// when its sum exceeds 1e-5. One warp per row; the ordered sum is carried
// lane-uniformly through the set bits of each 32-candidate chunk.
__global__ void __launch_bounds__(256) k_row_finalize(uint32_t n, const unsigned long long* cand_off,
                                                       const float* cand_ff, const float* cand_vis,
                                                       const uint8_t* cand_steps, const uint16_t* clo,
                                                       uint32_t* row_links, float* row_scale, float* row_sum,
                                                       float* row_sky, unsigned long long* row_evals) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += warps) {
        const unsigned long long b = cand_off[row], e = cand_off[row + 1];
        float sum = 0.0f;
        uint32_t links = 0, steps = 0;
        // The row's 16 closure rays: lanes 0..15 hold one each.
        const uint32_t cl = lane < 16 ? clo[(size_t)row * 16 + lane] : 0u;
        const uint32_t open = __popc(__ballot_sync(kFull, (cl & 0x100u) != 0));
        steps = cl & 0xffu;
        for (unsigned long long base = b; base < e; base += 32) {
            unsigned long long j = base + lane;
            bool valid = j < e;
            float vis = valid ? cand_vis[j] : 0.0f;
            float v = valid ? cand_ff[j] * vis : 0.0f;
            steps += valid ? cand_steps[j] : 0u;
            unsigned mask = __ballot_sync(kFull, valid && vis > 1e-3f);
            links += __popc(mask);
            while (mask) {
                int k = __ffs(mask) - 1;
                sum += __shfl_sync(kFull, v, k);
                mask &= mask - 1;
            }
        }
        for (int o = 16; o >= 1; o >>= 1) steps += __shfl_xor_sync(kFull, steps, o);
        if (lane == 0) {
            float sky = (float)open / 16.0f;
            float target = clampr(1.0f - sky, 0.0f, 1.0f);
            float scale = 1.0f;
            if (sum > 1e-5f) {
                scale = fminf(target / sum, 8.0f);
                sum *= scale;
            }
            row_links[row] = links;
            row_scale[row] = scale;
            row_sum[row] = fminf(sum, 1.0f);
            row_sky[row] = sky;
            row_evals[row] = (unsigned long long)steps;
        }
    }
}

__global__ void __launch_bounds__(256) k_row_fill(uint32_t n, const unsigned long long* cand_off,
                                                   const uint32_t* cand_c, const float* cand_ff,
                                                   const float* cand_vis, const float* row_scale,
                                                   const uint32_t* starts, uint32_t* idx, float* w) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += warps) {
        const unsigned long long b = cand_off[row], e = cand_off[row + 1];
        const float scale = row_scale[row];
        uint32_t at = starts[row];
        for (unsigned long long base = b; base < e; base += 32) {
            unsigned long long j = base + lane;
            bool valid = j < e;
            float vis = valid ? cand_vis[j] : 0.0f;
            bool link = valid && vis > 1e-3f;
            unsigned mask = __ballot_sync(kFull, link);
            if (link) {
                uint32_t o = at + __popc(mask & ((1u << lane) - 1u));
                idx[o] = cand_c[j];
                w[o] = (cand_ff[j] * vis) * scale;
            }
            at += __popc(mask);
        }
    }
}

// formfactor.rs:242-253: sequential f32 sum of the interior rows' sums in
// row order (the reference's iterator sum starts from -0.0). One CTA: all
// threads stream chunks of rows into shared memory (rows without links
// contribute an exact -0.0, the additive identity), thread 0 performs the
// ordered additions, four values per 16-byte shared-memory load; chunks are
// double-buffered so loads overlap the adds. The sum is one dependent chain
// of additions by nature (f32 addition does not associate), so it runs on
// its own stream beside the stages that follow it.
static constexpr int kMeanBlock = 1024;
__global__ void __launch_bounds__(kMeanBlock) k_mean_row_sum(uint32_t n, const uint32_t* starts,
                                                               const float* row_sum, float* out_mean,
                                                               unsigned long long* out_interior) {
    __shared__ __align__(16) float buf[2][kMeanBlock];
    __shared__ unsigned long long cnt;
    if (threadIdx.x == 0) cnt = 0;
    float acc = -0.0f;
    const uint32_t chunks = (n + kMeanBlock - 1) / kMeanBlock;
    unsigned long long mine = 0;
    auto load = [&](uint32_t c, int b) {
        uint32_t i = c * kMeanBlock + threadIdx.x;
        float v = -0.0f;
        if (i < n && starts[i + 1] > starts[i]) {
            v = row_sum[i];
            ++mine;
        }
        buf[b][threadIdx.x] = v;
    };
    if (chunks) load(0, 0);
    __syncthreads();
    for (uint32_t c = 0; c < chunks; ++c) {
        const int b = c & 1;
        if (threadIdx.x == 0) {
            const float4* b4 = reinterpret_cast<const float4*>(buf[b]);
#pragma unroll 8
            for (int k = 0; k < kMeanBlock / 4; ++k) {
                const float4 v = b4[k];
                acc += v.x;
                acc += v.y;
                acc += v.z;
                acc += v.w;
            }
        } else if (c + 1 < chunks) {
            load(c + 1, b ^ 1);
        }
        if (threadIdx.x == 0 && c + 1 < chunks) load(c + 1, b ^ 1);
        __syncthreads();
    }
    for (int o = 16; o >= 1; o >>= 1) mine += __shfl_xor_sync(kFull, mine, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&cnt, mine);
    __syncthreads();
    if (threadIdx.x == 0) {
        *out_mean = cnt ? acc / (float)cnt : 0.0f;
        *out_interior = cnt;
    }
}

__global__ void k_sum_u64(const unsigned long long* v, uint32_t n, unsigned long long* out) {
    unsigned long long s = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += v[i];
    for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

void launch_pair_count(cudaStream_t st, const float4* sp, const float4* sn, uint32_t n, const float4* cp,
                       const float4* cn, uint32_t nc, unsigned long long* cand_count) {
    k_pair_count<<<grid_for((unsigned long long)n * 32ull, 256), 256, 0, st>>>(sp, sn, n, cp, cn, nc, cand_count);
}
void launch_pair_fill(cudaStream_t st, const float4* sp, const float4* sn, uint32_t n, const float4* cp,
                      const float4* cn, uint32_t nc, const unsigned long long* cand_off, uint32_t* cand_c,
                      float* cand_ff, uint32_t* cand_row) {
    k_pair_fill<<<grid_for((unsigned long long)n * 32ull, 256), 256, 0, st>>>(sp, sn, n, cp, cn, nc, cand_off,
                                                                             cand_c, cand_ff, cand_row);
}
void launch_visibility(cudaStream_t st, BlobRef blob, SceneConsts sc, const float4* sp, const float4* sn,
                       const float4* cp, const float4* cn, const uint32_t* cand_c, const uint32_t* cand_row,
                       const uint32_t* order, unsigned long long ncand, float* cand_vis, uint8_t* cand_steps,
                       uint32_t* status, unsigned long long* counts, unsigned long long* cursor) {
    if (ncand == 0) return;
    const size_t sm = blob_smem(blob, 128);
    if (counts)
        k_visibility<Counts><<<persistent_grid(k_visibility<Counts>, 128, sm, ncand), 128, sm, st>>>(
            blob, sc, sp, sn, cp, cn, cand_c, cand_row, order, ncand, cand_vis, cand_steps, status, counts, cursor);
    else if (blob.tree3)
        k_visibility<NoCount3><<<persistent_grid(k_visibility<NoCount3>, 128, sm, ncand), 128, sm, st>>>(
            blob, sc, sp, sn, cp, cn, cand_c, cand_row, order, ncand, cand_vis, cand_steps, status, nullptr,
            cursor);
    else
        k_visibility<NoCount><<<persistent_grid(k_visibility<NoCount>, 128, sm, ncand), 128, sm, st>>>(
            blob, sc, sp, sn, cp, cn, cand_c, cand_row, order, ncand, cand_vis, cand_steps, status, nullptr,
            cursor);
}

// Sort keys of the visibility order: target cluster, then the source
// surfel's cluster (nc when it has none); values: candidate indices.
__global__ void k_vis_keys(unsigned long long ncand, const uint32_t* cand_c, const uint32_t* cand_row,
                           const uint32_t* cid, uint32_t nc, unsigned long long* keys, uint32_t* vals) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < ncand; k += stride) {
        const uint32_t src = cid[cand_row[k]];
        keys[k] = (unsigned long long)cand_c[k] * (nc + 1ull) + (src < nc ? src : nc);
        vals[k] = (uint32_t)k;
    }
}

int launch_vis_keys(cudaStream_t st, unsigned long long ncand, const uint32_t* cand_c, const uint32_t* cand_row,
                    const uint32_t* cid, uint32_t nc, unsigned long long* keys, uint32_t* vals) {
    if (ncand == 0) return 0;
    k_vis_keys<<<grid_for(ncand, 256), 256, 0, st>>>(ncand, cand_c, cand_row, cid, nc, keys, vals);
    return 1;
}
void launch_closure(cudaStream_t st, BlobRef blob, SceneConsts sc, const float4* sp, const float4* sn,
                    uint32_t n, const uint32_t* order, uint16_t* clo, uint32_t* status, unsigned long long* counts,
                    unsigned long long* cursor) {
    const size_t sm = blob_smem(blob, 128);
    const unsigned long long items = (unsigned long long)n * 16ull;
    if (counts)
        k_closure<Counts><<<persistent_grid(k_closure<Counts>, 128, sm, items), 128, sm, st>>>(
            blob, sc, sp, sn, n, order, clo, status, counts, cursor);
    else if (blob.tree3)
        k_closure<NoCount3><<<persistent_grid(k_closure<NoCount3>, 128, sm, items), 128, sm, st>>>(
            blob, sc, sp, sn, n, order, clo, status, nullptr, cursor);
    else
        k_closure<NoCount><<<persistent_grid(k_closure<NoCount>, 128, sm, items), 128, sm, st>>>(
            blob, sc, sp, sn, n, order, clo, status, nullptr, cursor);
}

// Sort keys of the closure order: the row's cluster (nc when it has none),
// then the direction index; values: item indices (row * 16 + direction).
__global__ void k_clo_keys(uint32_t n, const uint32_t* cid, uint32_t nc, uint32_t* keys, uint32_t* vals) {
    const uint32_t total = n * 16u;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const uint32_t c = cid[t >> 4];
        keys[t] = (c < nc ? c : nc) * 16u + (t & 15u);
        vals[t] = t;
    }
}

int launch_clo_keys(cudaStream_t st, uint32_t n, const uint32_t* cid, uint32_t nc, uint32_t* keys, uint32_t* vals) {
    if (n == 0) return 0;
    k_clo_keys<<<grid_for((unsigned long long)n * 16ull, 256), 256, 0, st>>>(n, cid, nc, keys, vals);
    return 1;
}
void launch_row_finalize(cudaStream_t st, uint32_t n, const unsigned long long* cand_off, const float* cand_ff,
                         const float* cand_vis, const uint8_t* cand_steps, const uint16_t* clo, uint32_t* row_links,
                         float* row_scale, float* row_sum, float* row_sky, unsigned long long* row_evals) {
    k_row_finalize<<<grid_for((unsigned long long)n * 32ull, 256), 256, 0, st>>>(
        n, cand_off, cand_ff, cand_vis, cand_steps, clo, row_links, row_scale, row_sum, row_sky, row_evals);
}
void launch_row_fill(cudaStream_t st, uint32_t n, const unsigned long long* cand_off, const uint32_t* cand_c,
                     const float* cand_ff, const float* cand_vis, const float* row_scale, const uint32_t* starts,
                     uint32_t* idx, float* w) {
    k_row_fill<<<grid_for((unsigned long long)n * 32ull, 256), 256, 0, st>>>(n, cand_off, cand_c, cand_ff, cand_vis,
                                                                            row_scale, starts, idx, w);
}
void launch_mean_row_sum(cudaStream_t st, uint32_t n, const uint32_t* starts, const float* row_sum,
                         float* out_mean, unsigned long long* out_interior) {
    k_mean_row_sum<<<1, kMeanBlock, 0, st>>>(n, starts, row_sum, out_mean, out_interior);
}
void launch_sum_u64(cudaStream_t st, const unsigned long long* v, uint32_t n, unsigned long long* out) {
    k_sum_u64<<<grid_for(n, 256, 2), 256, 0, st>>>(v, n, out);
}

#ifdef IFX_CHECKED
// Bounds-checked build only: every structure the transfer build produced is
// validated before the solve reads it (CSR starts non-decreasing and ending
// at `links`, link columns below nc, cluster ranges inside the member list,
// member indices below n); a violation sets kStatusBounds.
__global__ void k_check_transfer(uint32_t n, uint32_t nc, unsigned long long links, const uint32_t* starts,
                                 const uint32_t* idx, const uint2* crange, const uint32_t* members,
                                 uint32_t* status) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    const unsigned long long t0 = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool bad = false;
    for (unsigned long long i = t0; i < n; i += stride) bad |= starts[i] > starts[i + 1] || members[i] >= n;
    if (t0 == 0) bad |= starts[0] != 0u || starts[n] != links;
    for (unsigned long long k = t0; k < links; k += stride) bad |= idx[k] >= nc;
    for (unsigned long long c = t0; c < nc; c += stride) bad |= crange[c].x > crange[c].y || crange[c].y > n;
    if (bad) atomicOr(status, kStatusBounds);
}
void launch_check_transfer(cudaStream_t st, uint32_t n, uint32_t nc, unsigned long long links,
                           const uint32_t* starts, const uint32_t* idx, const uint2* crange,
                           const uint32_t* members, uint32_t* status) {
    k_check_transfer<<<grid_for(links > n ? links : n, 256), 256, 0, st>>>(n, nc, links, starts, idx, crange,
                                                                          members, status);
}
#endif

void configure_transfer_kernels(int max_dyn_smem) {
    cudaFuncSetAttribute(k_visibility<NoCount>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_visibility<NoCount3>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_visibility<Counts>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_closure<NoCount>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_closure<NoCount3>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_closure<Counts>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
}

}  // namespace ifx
