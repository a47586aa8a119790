// Surfel generation (projection part), surfel clusters and the gather grid.
#include "kcommon.cuh"

namespace ifx {

// surfel.rs:190-211: Halton seed i (bases 2, 3, 5) across the scene bounds,
// Newton projection onto the zero level set (at most 10 steps), then the
// on-surface and in-bounds tests. Writes the projected point with w = 1 if
// the seed survives, w = 0 otherwise. The Poisson-disc thinning that follows
// (below) keeps the reference's seed-order semantics.
__global__ void __launch_bounds__(128) k_gen_project(BlobRef blob, SceneConsts sc, uint32_t seed0,
                                                      uint32_t count, float eps, float4* out, uint32_t* status) {
    IFX_SCENE_PROLOGUE(blob, status, sv);
    NoCount nc;
    const V lo{sc.lo[0], sc.lo[1], sc.lo[2]}, hi{sc.hi[0], sc.hi[1], sc.hi[2]};
    const float diag = sc.diag;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x) {
        uint32_t i = seed0 + j;
        V s{radical_inverse(i + 1, 2), radical_inverse(i + 1, 3), radical_inverse(i + 1, 5)};
        V p = lo + (hi - lo) * s;
        bool ok = false;
        for (int it = 0; it < 10; ++it) {
            float d = scene_dist(sv, p, nc);
            if (fabsf(d) < eps) {
                ok = true;
                break;
            }
            if (!isfinite(d) || fabsf(d) > diag) break;
            p = p - scene_normal(sv, p, nc) * d;
        }
        if (ok && fabsf(scene_dist(sv, p, nc)) >= eps) ok = false;
        if (ok && (p.x < lo.x || p.y < lo.y || p.z < lo.z || p.x > hi.x || p.y > hi.y || p.z > hi.z)) ok = false;
        out[j] = make_float4(p.x, p.y, p.z, ok ? 1.0f : 0.0f);
    }
}

// surfel.rs:233-246: material albedo and normal of each accepted point.
__global__ void __launch_bounds__(128) k_gen_finalize(BlobRef blob, const float4* pts, uint32_t n, float area,
                                                       SurfelArrays s, uint32_t* status) {
    IFX_SCENE_PROLOGUE(blob, status, sv);
    NoCount nc;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        V p = mk4(pts[i]);
        DistHit h = dist_mat(sv, p, nc);
        const DMaterial& m = sv.mat(h.mat);
        V nn = scene_normal(sv, p, nc);
        s.p[i] = f4(p, area);
        s.n[i] = f4(nn, 0.0f);
        s.albedo[i] = make_float4(m.kd[0], m.kd[1], m.kd[2], 0.0f);
        s.direct[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        s.irr[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        s.rad[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

// ------------------------------------------------- Poisson-disc thinning --
// surfel.rs:206-227 accepts seed i iff no earlier accepted surfel lies
// within d_min (squared distance in f32, glam's dot order) and the target is
// not yet reached; the occupancy grid there is only an accelerator, since
// cells are d_min wide, so "within d_min" is exactly the test. Here seeds are
// taken in batches of consecutive indices:
//   filter   drop seeds that an accepted point of an earlier batch rejects;
//   append   the rest become this batch's points, in seed order, linked into
//            the batch's occupancy lists;
//   resolve  rounds: a point is accepted once every earlier point of the
//            batch within d_min is rejected, and rejected as soon as one of
//            them is accepted. Decisions are final and only taken on final
//            information, so the fixed point is the sequential result and
//            does not depend on scheduling; each round decides at least the
//            earliest open point;
//   retire   the batch's accepted points join the accepted-point lists that
//            later filters walk, and the batch lists are emptied, so that no
//            walk ever passes a rejected point.
// Lists are walked with a bound (the point capacity); an over-long walk sets
// kStatusGenWalk.
__device__ __forceinline__ int gen_cell(const GenGrid& g, float v, int a) {
    return clampi(as_i32((v - g.lo[a]) * g.inv_cell), 0, g.dim[a] - 1);
}

__device__ __forceinline__ bool gen_close(float4 a, float4 b, float d2) {
    const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return dx * dx + dy * dy + dz * dz < d2;
}

__device__ __forceinline__ size_t gen_cell_index(const GenGrid& g, float4 p) {
    return (size_t)gen_cell(g, p.x, 0) +
           (size_t)g.dim[0] * ((size_t)gen_cell(g, p.y, 1) + (size_t)g.dim[1] * gen_cell(g, p.z, 2));
}

// Visits every point linked into the 27 cells around p in the lists
// (head, next): f(index) returns false to stop. Returns false if a walk hit
// the bound.
template <class F>
__device__ __forceinline__ bool gen_walk(const GenGrid& g, const uint32_t* head, const uint32_t* next, float4 p,
                                         F&& f) {
    const int cx = gen_cell(g, p.x, 0), cy = gen_cell(g, p.y, 1), cz = gen_cell(g, p.z, 2);
    for (int z = max(cz - 1, 0); z <= min(cz + 1, g.dim[2] - 1); ++z)
        for (int y = max(cy - 1, 0); y <= min(cy + 1, g.dim[1] - 1); ++y)
            for (int x = max(cx - 1, 0); x <= min(cx + 1, g.dim[0] - 1); ++x) {
                const size_t cell = (size_t)x + (size_t)g.dim[0] * ((size_t)y + (size_t)g.dim[1] * (size_t)z);
                uint32_t e = head[cell];
                for (uint32_t guard = 0; e != 0; ++guard) {
                    if (guard > g.cap) {
                        atomicOr(g.err, kStatusGenWalk);
                        return false;
                    }
                    const uint32_t idx = e - 1;
                    if (!f(idx)) return true;
                    e = next[idx];
                }
            }
    return true;
}

// A seed survives if no accepted point of an earlier batch lies within d_min
// (those are exactly the points in the accepted lists).
__global__ void k_gen_filter(GenGrid g, const float4* cand, uint32_t cnt, uint32_t* keep) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < cnt; j += gridDim.x * blockDim.x) {
        const float4 q = cand[j];
        bool close = false;
        if (q.w != 0.0f)
            gen_walk(g, g.head_acc, g.next_acc, q, [&](uint32_t idx) {
                if (gen_close(g.pts[idx], q, g.d_min_sq)) close = true;
                return !close;
            });
        keep[j] = (q.w != 0.0f && !close) ? 1u : 0u;
    }
}

__global__ void k_gen_append(GenGrid g, const float4* cand, const uint32_t* keep, const uint32_t* off, uint32_t cnt,
                             uint32_t base) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < cnt; j += gridDim.x * blockDim.x) {
        if (!keep[j]) continue;
        const uint32_t pid = base + off[j];
        if (pid >= g.cap) {
            atomicOr(g.err, kStatusGenWalk);
            continue;
        }
        const float4 q = cand[j];
        g.pts[pid] = q;
        g.state[pid] = 0u;
        g.next[pid] = atomicExch(&g.head[gen_cell_index(g, q)], pid + 1u);
    }
}

__global__ void k_gen_resolve(GenGrid g, uint32_t base, uint32_t count, uint32_t* undecided) {
    volatile uint32_t* state = g.state;
    uint32_t open = 0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t pid = base + k;
        if (state[pid] != 0u) continue;
        const float4 p = g.pts[pid];
        bool rej = false, pend = false;
        const bool ok = gen_walk(g, g.head, g.next, p, [&](uint32_t idx) {
            if (idx < base || idx >= pid || !gen_close(g.pts[idx], p, g.d_min_sq)) return true;
            const uint32_t s = state[idx];
            if (s == 1u) rej = true;
            else if (s == 0u) pend = true;
            return !rej;
        });
        if (!ok) continue;
        if (rej) state[pid] = 2u;
        else if (!pend) state[pid] = 1u;
        else ++open;
    }
    for (int o = 16; o >= 1; o >>= 1) open += __shfl_xor_sync(0xffffffffu, open, o);
    if ((threadIdx.x & 31) == 0 && open) atomicAdd(undecided, open);
}

__global__ void k_gen_accept_flags(GenGrid g, uint32_t base, uint32_t count, uint32_t* flags) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= count; k += gridDim.x * blockDim.x)
        flags[k] = k < count && g.state[base + k] == 1u ? 1u : 0u;
}

__global__ void k_gen_emit(GenGrid g, uint32_t base, uint32_t count, const uint32_t* rank, uint32_t quota,
                           float4* out) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x)
        if (g.state[base + k] == 1u && rank[k] < quota) out[rank[k]] = g.pts[base + k];
}

__global__ void k_gen_retire(GenGrid g, uint32_t base, uint32_t count) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t pid = base + k;
        const size_t cell = gen_cell_index(g, g.pts[pid]);
        g.head[cell] = 0u;
        if (g.state[pid] == 1u) g.next_acc[pid] = atomicExch(&g.head_acc[cell], pid + 1u);
    }
}

int launch_gen_retire(cudaStream_t st, const GenGrid& g, uint32_t base, uint32_t count) {
    k_gen_retire<<<grid_for(count, 256), 256, 0, st>>>(g, base, count);
    return 1;
}

int launch_gen_filter(cudaStream_t st, const GenGrid& g, const float4* cand, uint32_t cnt, uint32_t* keep) {
    k_gen_filter<<<grid_for(cnt, 256), 256, 0, st>>>(g, cand, cnt, keep);
    return 1;
}
int launch_gen_append(cudaStream_t st, const GenGrid& g, const float4* cand, const uint32_t* keep,
                      const uint32_t* off, uint32_t cnt, uint32_t base) {
    k_gen_append<<<grid_for(cnt, 256), 256, 0, st>>>(g, cand, keep, off, cnt, base);
    return 1;
}
int launch_gen_resolve(cudaStream_t st, const GenGrid& g, uint32_t base, uint32_t count, uint32_t* undecided) {
    k_gen_resolve<<<grid_for(count, 256), 256, 0, st>>>(g, base, count, undecided);
    return 1;
}
int launch_gen_accept_flags(cudaStream_t st, const GenGrid& g, uint32_t base, uint32_t count, uint32_t* flags) {
    k_gen_accept_flags<<<grid_for((unsigned long long)count + 1, 256), 256, 0, st>>>(g, base, count, flags);
    return 1;
}
int launch_gen_emit(cudaStream_t st, const GenGrid& g, uint32_t base, uint32_t count, const uint32_t* rank,
                    uint32_t quota, float4* out) {
    k_gen_emit<<<grid_for(count, 256), 256, 0, st>>>(g, base, count, rank, quota, out);
    return 1;
}

void launch_gen_project(cudaStream_t st, BlobRef blob, SceneConsts sc, uint32_t seed0, uint32_t count, float eps,
                        float4* out, uint32_t* status) {
    k_gen_project<<<grid_for(count, 128), 128, blob_smem(blob, 128), st>>>(blob, sc, seed0, count, eps, out, status);
}
void launch_gen_finalize(cudaStream_t st, BlobRef blob, const float4* pts, uint32_t n, float area, SurfelArrays s,
                         uint32_t* status) {
    k_gen_finalize<<<grid_for(n, 128), 128, blob_smem(blob, 128), st>>>(blob, pts, n, area, s, status);
}

// ------------------------------------------------------------ clusters ----
// formfactor.rs:70-89
__device__ __forceinline__ uint32_t normal_bucket(V n) {
    V a = vabs(n);
    if (a.x >= a.y && a.x >= a.z) return n.x >= 0.0f ? 0u : 1u;
    if (a.y >= a.z) return n.y >= 0.0f ? 2u : 3u;
    return n.z >= 0.0f ? 4u : 5u;
}

// formfactor.rs:100-110: key (x, y, z, bucket) packed so that integer order
// is the tuple order; the surfel index in the low word makes the sort
// stable (members ascend within a cluster, as the reference's push order).
__global__ void k_cluster_keys(const float4* p, const float4* n, uint32_t count, SceneConsts sc, int res,
                               unsigned long long* keys) {
    const V lo{sc.lo[0], sc.lo[1], sc.lo[2]};
    V ext = V{sc.hi[0], sc.hi[1], sc.hi[2]} - lo;
    V inv{(float)res / fmaxf(ext.x, 1e-6f), (float)res / fmaxf(ext.y, 1e-6f), (float)res / fmaxf(ext.z, 1e-6f)};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        V c = (mk4(p[i]) - lo) * inv;
        unsigned long long x = (unsigned long long)clampi(as_i32(c.x), 0, res - 1);
        unsigned long long y = (unsigned long long)clampi(as_i32(c.y), 0, res - 1);
        unsigned long long z = (unsigned long long)clampi(as_i32(c.z), 0, res - 1);
        unsigned long long key = ((x * (unsigned long long)res + y) * (unsigned long long)res + z) * 6ull +
                                 normal_bucket(mk4(n[i]));
        keys[i] = (key << 32) | (unsigned long long)i;
    }
}

__global__ void k_seg_heads(const unsigned long long* s, uint32_t count, uint32_t* heads) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x)
        heads[j] = (j == 0 || (s[j] >> 32) != (s[j - 1] >> 32)) ? 1u : 0u;
}

// head_scan is the inclusive scan of heads: the segment of position j is
// head_scan[j] - 1.
__global__ void k_seg_starts(const unsigned long long* s, const uint32_t* head_scan, uint32_t count,
                             uint32_t* seg_start, uint32_t* members) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x) {
        members[j] = (uint32_t)(s[j] & 0xffffffffull);
        uint32_t seg = head_scan[j] - 1u;
        if (j == 0 || head_scan[j] != head_scan[j - 1]) seg_start[seg] = j;
        if (j == count - 1) seg_start[seg + 1] = count;
    }
}

// formfactor.rs:119-145: sequential area-weighted sums in member order. One
// CTA per segment: the threads stage each member's p * area, n * area and
// area (each product rounds the same whoever forms it) in shared memory, a
// chunk at a time, and thread 0 adds them in member order.
static constexpr int kRedBlock = 128;
__global__ void __launch_bounds__(kRedBlock) k_cluster_reduce(const uint32_t* seg_start, const uint32_t* members,
                                                               uint32_t nseg, const float4* sp, const float4* sn,
                                                               float4* cp, float4* cn, uint32_t* valid) {
    __shared__ float4 bp[kRedBlock], bn[kRedBlock];
    for (uint32_t c = blockIdx.x; c < nseg; c += gridDim.x) {
        const uint32_t s0 = seg_start[c], s1 = seg_start[c + 1];
        V p{0.0f, 0.0f, 0.0f}, n{0.0f, 0.0f, 0.0f};
        float area = 0.0f;
        for (uint32_t k0 = s0; k0 < s1; k0 += kRedBlock) {
            const uint32_t k = k0 + threadIdx.x;
            if (k < s1) {
                const uint32_t m = members[k];
                const float4 a = __ldg(&sp[m]);
                const float4 b = __ldg(&sn[m]);
                bp[threadIdx.x] = make_float4(a.x * a.w, a.y * a.w, a.z * a.w, a.w);
                bn[threadIdx.x] = make_float4(b.x * a.w, b.y * a.w, b.z * a.w, 0.0f);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                const uint32_t cnt = min((uint32_t)kRedBlock, s1 - k0);
                for (uint32_t j = 0; j < cnt; ++j) {
                    const float4 u = bp[j], v = bn[j];
                    p = p + V{u.x, u.y, u.z};
                    n = n + V{v.x, v.y, v.z};
                    area += u.w;
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            bool ok = area > 1e-12f;
            valid[c] = ok ? 1u : 0u;
            V nn = dot(n, n) > 1e-12f ? nrm(n) : V{0.0f, 1.0f, 0.0f};
            cp[c] = f4(p / area, area);
            cn[c] = f4(nn, sqrtf(area / kPiF));
        }
    }
}

__global__ void k_cluster_compact(const uint32_t* valid, const uint32_t* valid_scan, uint32_t nseg,
                                  const uint32_t* seg_start, const float4* cp_in, const float4* cn_in, float4* cp,
                                  float4* cn, uint2* crange) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nseg; c += gridDim.x * blockDim.x) {
        if (!valid[c]) continue;
        uint32_t o = valid_scan[c];  // exclusive scan
        cp[o] = cp_in[c];
        cn[o] = cn_in[c];
        crange[o] = make_uint2(seg_start[c], seg_start[c + 1]);
    }
}

void launch_cluster_keys(cudaStream_t st, const float4* p, const float4* n, uint32_t count, SceneConsts sc,
                         int res, unsigned long long* keys) {
    k_cluster_keys<<<grid_for(count, 256), 256, 0, st>>>(p, n, count, sc, res, keys);
}
void launch_seg_heads(cudaStream_t st, const unsigned long long* sorted, uint32_t count, uint32_t* heads) {
    k_seg_heads<<<grid_for(count, 256), 256, 0, st>>>(sorted, count, heads);
}
void launch_seg_starts(cudaStream_t st, const unsigned long long* sorted, const uint32_t* head_scan,
                       uint32_t count, uint32_t* seg_start, uint32_t* members) {
    k_seg_starts<<<grid_for(count, 256), 256, 0, st>>>(sorted, head_scan, count, seg_start, members);
}
void launch_cluster_reduce(cudaStream_t st, const uint32_t* seg_start, const uint32_t* members, uint32_t nseg,
                           const float4* sp, const float4* sn, float4* cp, float4* cn, uint32_t* valid) {
    k_cluster_reduce<<<nseg < 65535u ? (nseg ? nseg : 1u) : 65535u, kRedBlock, 0, st>>>(seg_start, members, nseg, sp,
                                                                                       sn, cp, cn, valid);
}
void launch_cluster_compact(cudaStream_t st, const uint32_t* valid, const uint32_t* valid_scan, uint32_t nseg,
                            const uint32_t* seg_start, const float4* cp_in, const float4* cn_in, float4* cp,
                            float4* cn, uint2* crange) {
    k_cluster_compact<<<grid_for(nseg, 256), 256, 0, st>>>(valid, valid_scan, nseg, seg_start, cp_in, cn_in, cp, cn,
                                                           crange);
}

// ---------------------------------------------------------------- grid ----
// surfel.rs:262-269 cell index; key = (cell << 32) | surfel so that a sort
// reproduces the counting sort's stable order.
__global__ void k_grid_keys(const float4* p, uint32_t n, GridParams g, unsigned long long* keys) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 q = p[i];
        int cx = clampi(as_i32((q.x - g.lo[0]) * g.inv_cell), 0, g.dim[0] - 1);
        int cy = clampi(as_i32((q.y - g.lo[1]) * g.inv_cell), 0, g.dim[1] - 1);
        int cz = clampi(as_i32((q.z - g.lo[2]) * g.inv_cell), 0, g.dim[2] - 1);
        unsigned long long c =
            (unsigned long long)cx + (unsigned long long)g.dim[0] * ((unsigned long long)cy +
                                                                     (unsigned long long)g.dim[1] * (unsigned long long)cz);
        keys[i] = (c << 32) | (unsigned long long)i;
    }
}

// starts[c] = first sorted position whose cell is >= c (CSR offsets of the
// counting sort, surfel.rs:271-279), for every c in [0, ncells].
__global__ void k_grid_starts(const unsigned long long* s, uint32_t n, uint32_t ncells, uint32_t* starts) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j <= n; j += gridDim.x * blockDim.x) {
        unsigned long long lo_c = (j == 0) ? 0ull : (s[j - 1] >> 32) + 1ull;
        unsigned long long hi_c = (j == n) ? (unsigned long long)ncells : (s[j] >> 32);
        for (unsigned long long c = lo_c; c <= hi_c; ++c) starts[c] = j;
    }
}

__global__ void k_grid_scatter(const unsigned long long* s, uint32_t n, SurfelArrays sa, float4* gp, float4* gn,
                               float4* girr, uint32_t* items) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        uint32_t i = (uint32_t)(s[j] & 0xffffffffull);
        items[j] = i;
        gp[j] = sa.p[i];
        gn[j] = sa.n[i];
        girr[j] = sa.irr[i];
    }
}

void launch_grid_keys(cudaStream_t st, const float4* p, uint32_t n, GridParams g, unsigned long long* keys) {
    k_grid_keys<<<grid_for(n, 256), 256, 0, st>>>(p, n, g, keys);
}
void launch_grid_starts(cudaStream_t st, const unsigned long long* sorted, uint32_t n, uint32_t ncells,
                        uint32_t* starts) {
    k_grid_starts<<<grid_for((unsigned long long)n + 1, 256), 256, 0, st>>>(sorted, n, ncells, starts);
}
void launch_grid_scatter(cudaStream_t st, const unsigned long long* sorted, uint32_t n, SurfelArrays s,
                         float4* gp, float4* gn, float4* girr, uint32_t* items) {
    k_grid_scatter<<<grid_for(n, 256), 256, 0, st>>>(sorted, n, s, gp, gn, girr, items);
}

void configure_surfel_kernels(int max_dyn_smem) {
    cudaFuncSetAttribute(k_gen_project, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_gen_finalize, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
}

}  // namespace ifx
