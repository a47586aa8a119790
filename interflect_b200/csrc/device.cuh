// Device-side scene evaluation: SDF primitives, BVH nearest-distance query,
// sphere tracing, cone soft shadows, analytic area lights and the surfel
// gather. Every function keeps the reference's f32 operation order; the
// library is compiled with --fmad=false and IEEE division/square root, so
// each result is bit-identical to the unfused f32 arithmetic of the
// reference (acos reproduces glibc's acosf exactly; only the sphere-light extension calls CUDA's atanf).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "layout.h"
#include "libm_f32.h"
#include "sqcmp.h"

namespace ifx {

// ------------------------------------------------------------- vectors ----
struct V {
    float x, y, z;
};
__device__ __forceinline__ V mk(float x, float y, float z) { return V{x, y, z}; }
__device__ __forceinline__ V mk4(float4 a) { return V{a.x, a.y, a.z}; }
__device__ __forceinline__ V operator+(V a, V b) { return V{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V operator-(V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V operator*(V a, V b) { return V{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V operator*(V a, float s) { return V{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V operator/(V a, float s) { return V{a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ V operator-(V a) { return V{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len(V a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ V nrm(V a) { return a * (1.0f / len(a)); }
__device__ __forceinline__ V cross(V a, V b) {
    return V{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
__device__ __forceinline__ V vabs(V a) { return V{fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
__device__ __forceinline__ V vmax(V a, V b) { return V{fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
// Rust f32::clamp: NaN passes through.
__device__ __forceinline__ float clampr(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
__device__ __forceinline__ float signumr(float x) { return isnan(x) ? x : copysignf(1.0f, x); }
// Rust `f32 as i32`: truncating, saturating, NaN -> 0.
__device__ __forceinline__ int32_t as_i32(float x) {
    if (isnan(x)) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}
__device__ __forceinline__ int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ float4 f4(V a, float w) { return make_float4(a.x, a.y, a.z, w); }

static constexpr float kPiF = 3.14159265358979323846f;
static constexpr float kMaxF = 3.40282347e38f;

// --------------------------------------------------------- scene view -----
// Views of the program blob (layout.h) in shared or global memory.
// Device status word bits (written with integer atomicOr, read by the host).
static constexpr uint32_t kStatusStageTimeout = 1u;
static constexpr uint32_t kStatusStackOverflow = 2u;

// Index check of the bounds-checked build (-DIFX_CHECKED): an index outside
// [0, n) sets kStatusBounds and is replaced by 0, so the access stays inside
// the array and the host reports the failure; in the normal build it is the
// index itself.
#ifdef IFX_CHECKED
__device__ __forceinline__ uint32_t ck_index(uint32_t i, uint32_t n, uint32_t* status) {
    if (i >= n) {
        if (status) atomicOr(status, kStatusBounds);
        return 0u;
    }
    return i;
}
#define IFX_CK(i, n, status) ::ifx::ck_index((uint32_t)(i), (uint32_t)(n), (status))
#else
#define IFX_CK(i, n, status) (i)
#endif

struct SceneView {
    const DObject* objs;
    const DPrim* prims;
    const DNode* nodes;
    const DQuadLight* lights;
    const DSphereLight* slights;
    const DMaterial* mats;
    const uint32_t* linear;
    int n_planes, n_objects, n_nodes, n_lights, n_slights, use_bvh;
    int n_prims, n_mats;
    uint32_t* status;  // the kernel's status word (bounds checks of IFX_CHECKED builds)
    LeafGrid lg;       // per-cell candidate leaves (shadow marches in large BVHs)
    // This thread's BVH traversal stack in shared memory: entry i lives at
    // stk[i * stk_stride] (node index) and stkd[i * stk_stride] (the node's
    // box distance, computed when it was pushed); stk_depth entries (the tree
    // depth + 2, fixed by the host), so consecutive threads hit consecutive
    // banks.
    uint32_t* stk;
    float* stkd;
    int stk_stride, stk_depth;

    // Element access; bounds-checked in IFX_CHECKED builds.
    __device__ __forceinline__ const DObject& obj(int i) const { return objs[IFX_CK(i, n_planes + n_objects, status)]; }
    __device__ __forceinline__ const DPrim& prim(int i) const { return prims[IFX_CK(i, n_prims, status)]; }
    __device__ __forceinline__ const DNode& node(int i) const { return nodes[IFX_CK(i, n_nodes, status)]; }
    __device__ __forceinline__ const DQuadLight& light(int i) const { return lights[IFX_CK(i, n_lights, status)]; }
    __device__ __forceinline__ const DSphereLight& slight(int i) const {
        return slights[IFX_CK(i, n_slights, status)];
    }
    __device__ __forceinline__ const DMaterial& mat(uint32_t i) const { return mats[IFX_CK(i, n_mats, status)]; }
    __device__ __forceinline__ uint32_t lin(int i) const { return linear[IFX_CK(i, n_objects, status)]; }
};

__device__ __forceinline__ SceneView make_view(const uint8_t* base) {
    const BlobHeader* h = reinterpret_cast<const BlobHeader*>(base);
    SceneView v;
    v.stk = nullptr;
    v.stkd = nullptr;
    v.stk_stride = 0;
    v.stk_depth = 0;
    v.objs = reinterpret_cast<const DObject*>(base + h->off_objects);
    v.prims = reinterpret_cast<const DPrim*>(base + h->off_prims);
    v.nodes = reinterpret_cast<const DNode*>(base + h->off_nodes);
    v.lights = reinterpret_cast<const DQuadLight*>(base + h->off_lights);
    v.slights = reinterpret_cast<const DSphereLight*>(base + h->off_sphere_lights);
    v.mats = reinterpret_cast<const DMaterial*>(base + h->off_materials);
    v.linear = reinterpret_cast<const uint32_t*>(base + h->off_linear);
    v.n_planes = h->n_planes;
    v.n_objects = h->n_objects;
    v.n_nodes = h->n_nodes;
    v.n_lights = h->n_lights;
    v.n_slights = h->n_sphere_lights;
    v.use_bvh = h->use_bvh;
    v.n_prims = h->n_prims;
    v.n_mats = h->n_materials;
    v.status = nullptr;
    v.lg = LeafGrid{};
    return v;
}

// ------------------------------------------------------- work counters ----
// Tracing functions take a counter policy. NoCount compiles to nothing and is
// what the timed kernels use; Counts tallies the work of one thread so that
// a separate counting launch can derive the algorithmic FLOPs of a kernel
// (the per-item costs are in flop_model.h).
enum CounterId : int {
    CN_NODE = 0,       // BVH aabb_dist evaluations
    CN_PRIM = 1,       // CN_PRIM + kind: primitive distance evaluations (8 kinds)
    CN_SMOOTH = 9,     // smooth subtractions
    CN_HARD = 10,      // hard subtractions max(d, -s)
    CN_SDF = 11,       // scene distance queries
    CN_TSTEP = 12,     // sphere-tracing steps
    CN_SSTEP = 13,     // soft-shadow steps
    CN_FF = 14,        // quad form factors
    CN_FF_EDGE = 15,   // edges summed by quad form factors
    CN_LIGHT = 16,     // light evaluations past the form-factor cull
    CN_SPEC = 17,      // specular lobes
    CN_GVISIT = 18,    // surfels visited by gather
    CN_GACCEPT = 19,   // surfels accumulated by gather
    CN_SSTEP_HIT = 20, // (reserved)
    kNumCounters = 21
};

//
// kTree3: the scene's BVH is known (by the host, which picks the kernel) to
// be a root with two leaves, so the distance queries compile only that
// traversal; a kernel then carries a fraction of the code, which matters to
// instruction-fetch-bound ray marches. NoCount3 is NoCount for such scenes.
struct NoCount {
    static constexpr bool kTree3 = false;
    __device__ __forceinline__ void add(int, uint32_t = 1) {}
};
struct NoCount3 : NoCount {
    static constexpr bool kTree3 = true;
};

struct Counts {
    static constexpr bool kTree3 = false;
    uint32_t v[kNumCounters];
    __device__ __forceinline__ Counts() {
#pragma unroll
        for (int i = 0; i < kNumCounters; ++i) v[i] = 0;
    }
    __device__ __forceinline__ void add(int id, uint32_t k = 1) { v[id] += k; }
    // Warp-level sum, then one 64-bit atomic per counter per warp (integer,
    // so the totals do not depend on scheduling). All lanes must call.
    __device__ __forceinline__ void flush(unsigned long long* out) {
#pragma unroll 1
        for (int i = 0; i < kNumCounters; ++i) {
            unsigned long long x = v[i];
            for (int o = 16; o >= 1; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if ((threadIdx.x & 31) == 0 && x) atomicAdd(&out[i], x);
            v[i] = 0;
        }
    }
};

// Copies the program blob into dynamic shared memory with one bulk
// (non-multicast) async copy completed on an mbarrier, and returns a view of
// it. The wait is bounded by `polls`: on expiry the status word gets
// kStatusStageTimeout, the CTA still waits (again bounded, by
// kStageDrainPolls) for its copy in flight to land so that no copy writes
// shared memory after the CTA has left, and the caller must return without
// tracing. `bytes` is a multiple of 16 and both addresses are 16-byte aligned.
static constexpr uint32_t kStageDrainPolls = 1u << 22;
__device__ __forceinline__ uint32_t mbar_try_wait(uint32_t bar) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar)
        : "memory");
    return done;
}
__device__ __forceinline__ void bulk_copy(uint32_t dst, const uint8_t* src, uint32_t bytes, uint32_t bar) {
    const uint32_t kChunk = 32768u;
    for (uint32_t off = 0; off < bytes; off += kChunk) {
        uint32_t n = bytes - off < kChunk ? bytes - off : kChunk;
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst + off),
            "l"(src + off), "r"(n), "r"(bar)
            : "memory");
    }
}
__device__ __forceinline__ bool stage_scene(const uint8_t* gblob, uint32_t bytes, uint8_t* smem,
                                            uint64_t* mbar, uint32_t* status, uint32_t polls) {
    uint32_t bar = (uint32_t)__cvta_generic_to_shared(mbar);
    uint32_t dst = (uint32_t)__cvta_generic_to_shared(smem);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
        bulk_copy(dst, gblob, bytes, bar);
    }
    uint32_t done = 0;
    for (uint32_t spin = 0; spin < polls; ++spin) {
        done = mbar_try_wait(bar);
        if (done) break;
    }
    if (!done) {
        atomicOr(status, kStatusStageTimeout);
        for (uint32_t spin = 0; spin < kStageDrainPolls; ++spin)
            if (mbar_try_wait(bar)) break;
    }
    __syncthreads();
    return __syncthreads_and(done) != 0;
}

// ------------------------------------------------------------- sdf.rs -----
// sdf.rs:52-125 over a packed primitive (hoisted terms in layout.h).
template <class C>
__device__ __forceinline__ float prim_dist(const DPrim& pr, V p, C& cnt) {
    const float4* q = reinterpret_cast<const float4*>(&pr);
    const int kind = pr.kind;
    cnt.add(CN_PRIM + kind);
    const float4 a = q[1];
    switch (kind) {
        case K_SPHERE:
            return len(p - mk4(a)) - a.w;
        case K_BOX:
        case K_BOX_ROT: {
            const float4 b = q[2];
            V d = p - mk4(a);
            if (kind == K_BOX_ROT) {
                const float4 c = q[3];
                const float rc = b.w, rs = c.x;
                d = V{rc * d.x - rs * d.z, d.y, rs * d.x + rc * d.z};
            }
            V bq{a.w, b.x, b.y};
            V qq = vabs(d) - bq;
            return len(vmax(qq, V{0.0f, 0.0f, 0.0f})) + fminf(fmaxf(qq.x, fmaxf(qq.y, qq.z)), 0.0f) - b.z;
        }
        case K_PLANE:
            return dot(p, mk4(a)) - a.w;
        case K_CAPSULE: {
            const float4 b = q[2];
            V pa = p - mk4(a);
            V ba{a.w, b.x, b.y};
            float h = clampr(dot(pa, ba) / b.z, 0.0f, 1.0f);
            return len(pa - ba * h) - b.w;
        }
        case K_TORUS: {
            const float4 b = q[2];
            V t = p - mk4(a);
            float xz = sqrtf(t.x * t.x + t.z * t.z) - a.w;
            return sqrtf(xz * xz + t.y * t.y) - b.x;
        }
        case K_CYLINDER: {
            const float4 b = q[2];
            const float4 c = q[3];
            V ba{a.w, b.x, b.y};
            float baba = b.z;
            V pa = p - mk4(a);
            float paba = dot(pa, ba);
            float x = len(pa * baba - ba * paba) - c.x;
            float y = fabsf(paba - c.y) - c.y;
            float x2 = x * x;
            float y2 = y * y * baba;
            float d;
            if (fmaxf(x, y) < 0.0f) d = -fminf(x2, y2);
            else d = (x > 0.0f ? x2 : 0.0f) + (y > 0.0f ? y2 : 0.0f);
            return signumr(d) * sqrtf(fabsf(d)) / baba;
        }
        case K_CONE: {
            const float4 b = q[2];
            const float4 c = q[3];
            V ba{a.w, b.x, b.y};
            float baba = b.z, ra = b.w, rb = c.x, rba = c.y, kk = c.z;
            V pa = p - mk4(a);
            float papa = dot(pa, pa);
            float paba = dot(pa, ba) / baba;
            float x = sqrtf(fmaxf(papa - paba * paba * baba, 0.0f));
            float cax = fmaxf(0.0f, x - (paba < 0.5f ? ra : rb));
            float cay = fabsf(paba - 0.5f) - 0.5f;
            float f = clampr((rba * (x - ra) + paba * baba) / kk, 0.0f, 1.0f);
            float cbx = x - ra - f * rba;
            float cby = paba - f;
            float s = (cbx < 0.0f && cay < 0.0f) ? -1.0f : 1.0f;
            return s * sqrtf(fminf(cax * cax + cay * cay * baba, cbx * cbx + cby * cby * baba));
        }
    }
    return kMaxF;
}

// sdf.rs:166-172 with the smooth-subtraction extension. `best` is the
// caller's best distance so far, against which the result is only compared
// with a strict `<`. A subtraction never lowers the base primitive's
// distance: max(d, -s) >= d exactly, and the smooth form is above max(d, -s)
// but for rounding (a few ulps of its operands, far below the margin here).
// So in the uncounted kernels, a base at or beyond `best` (plus that margin
// for the smooth form) cannot win the comparison, and its subtractions are
// not evaluated; the returned value is then the base's, itself >= best. The
// counting kernels evaluate everything, as the reference does.
template <class C>
__device__ __forceinline__ float obj_dist(const SceneView& sv, const DObject& o, V p, C& cnt, float best = kMaxF) {
    float d = prim_dist(sv.prim(o.prim), p, cnt);
    if constexpr (sizeof(C) == 1) {
        if (o.nsub > 0 && d >= best + (o.smooth > 0.0f ? 1e-5f * (1.0f + fabsf(best) + o.smooth) : 0.0f)) return d;
    }
    for (int s = 1; s <= o.nsub; ++s) {
        float sd = prim_dist(sv.prim(o.prim + s), p, cnt);
        cnt.add(o.smooth > 0.0f ? CN_SMOOTH : CN_HARD);
        if (o.smooth > 0.0f) {
            float k = o.smooth;
            float hk = clampr(0.5f - 0.5f * (d + sd) / k, 0.0f, 1.0f);
            d = d * (1.0f - hk) + (-sd) * hk + k * hk * (1.0f - hk);
        } else {
            d = fmaxf(d, -sd);
        }
    }
    return d;
}

// bvh.rs:46-50 before its square root: the box distance is
// sqrtf(aabb_dist2(p, n)).
template <class C>
__device__ __forceinline__ float aabb_dist2(V p, const DNode& n, C& cnt) {
    cnt.add(CN_NODE);
    V lo{n.lo[0], n.lo[1], n.lo[2]}, hi{n.hi[0], n.hi[1], n.hi[2]};
    const V q = vmax(vmax(lo - p, p - hi), V{0.0f, 0.0f, 0.0f});
    return dot(q, q);
}

struct DistHit {
    float d;
    uint32_t mat;
};

// scene.rs:191-208 with bvh.rs:100-150 (query) or bvh.rs:155-163 (linear).
template <class C>
__device__ __forceinline__ DistHit dist_mat(const SceneView& sv, V p, C& cnt) {
    cnt.add(CN_SDF);
    DistHit best{kMaxF, 0u};
    for (int i = 0; i < sv.n_planes; ++i) {
        const DObject o = sv.obj(i);
        float d = obj_dist(sv, o, p, cnt, best.d);
        if (d < best.d) best = DistHit{d, o.mat};
    }
    if constexpr (C::kTree3) {
        // bvh.rs:100-150 on a root and two leaves: the same tests, prunes and
        // visit order as the stack traversal below.
        if (sq_ge(aabb_dist2(p, sv.node(0), cnt), best.d)) return best;
        const int r = sv.node(0).link;
        const float dl = aabb_dist2(p, sv.node(1), cnt), dr = aabb_dist2(p, sv.node(r), cnt);
        const bool lfirst = sq_lt(dl, dr);
#pragma unroll 1
        for (int pass = 0; pass < 2; ++pass) {
            const bool left = (pass == 0) == lfirst;
            if (sq_ge(left ? dl : dr, best.d)) continue;
            const DNode& nd = sv.node(left ? 1 : r);
            for (int k = nd.link; k < nd.link + nd.count; ++k) {
                const DObject o = sv.obj(k);
                const float d = obj_dist(sv, o, p, cnt, best.d);
                if (d < best.d) {
                    best.d = d;
                    best.mat = o.mat;
                }
            }
        }
        return best;
    }
    if (sv.use_bvh) {
        if (sv.n_nodes == 0) return best;
        // bvh.rs:100-150. A node's box distance is a pure function of p and
        // the node, so the value computed when it was pushed (bvh.rs:135-136)
        // is the one the reference recomputes when it pops it (:116); it is
        // kept on the stack and counted as the reference's test.
        // The stack holds squared box distances (see sq_ge / sq_lt).
        uint32_t* const stack = sv.stk;
        float* const stackd = sv.stkd;
        const int stride = sv.stk_stride;
        int sp = 0;
        stack[0] = 0;
        stackd[0] = aabb_dist2(p, sv.node(0), cnt);
        sp = 1;
        bool first = true;
        while (sp > 0) {
            --sp;
            const int ni = (int)stack[sp * stride];
            const DNode nd = sv.node(ni);
            if (!first) cnt.add(CN_NODE);
            first = false;
            if (sq_ge(stackd[sp * stride], best.d)) continue;
            if (nd.count > 0) {
                for (int k = nd.link; k < nd.link + nd.count; ++k) {
                    const DObject o = sv.obj(k);
                    float d = obj_dist(sv, o, p, cnt, best.d);
                    if (d < best.d) {
                        best.d = d;
                        best.mat = o.mat;
                    }
                }
            } else {
                const int l = ni + 1, r = nd.link;
                float dl = aabb_dist2(p, sv.node(l), cnt);
                float dr = aabb_dist2(p, sv.node(r), cnt);
                // Near-first DFS holds at most depth + 1 entries; the host
                // sizes the stack to depth + 2 (and rejects trees deeper
                // than the reference's 64-entry stack). The guard keeps an
                // unexpected overflow inside the stack: traversal stops.
                if (sp + 2 > sv.stk_depth) break;
                if (sq_lt(dl, dr)) {
                    stack[sp * stride] = (uint32_t)r;
                    stackd[sp * stride] = dr;
                    stack[(sp + 1) * stride] = (uint32_t)l;
                    stackd[(sp + 1) * stride] = dl;
                } else {
                    stack[sp * stride] = (uint32_t)l;
                    stackd[sp * stride] = dl;
                    stack[(sp + 1) * stride] = (uint32_t)r;
                    stackd[(sp + 1) * stride] = dr;
                }
                sp += 2;
            }
        }
    } else {
        for (int k = 0; k < sv.n_objects; ++k) {
            const DObject o = sv.obj(sv.lin(k));
            float d = obj_dist(sv, o, p, cnt, best.d);
            if (d < best.d) {
                best.d = d;
                best.mat = o.mat;
            }
        }
    }
    return best;
}

template <class C>
__device__ __forceinline__ float scene_dist(const SceneView& sv, V p, C& cnt) {
    return dist_mat(sv, p, cnt).d;
}

// Evaluates leaf `leaf`'s objects into `best` (bvh.rs:118-126).
template <class C>
__device__ __forceinline__ void leaf_eval(const SceneView& sv, int leaf, V p, DistHit& best, C& cnt) {
    const DNode nd = sv.node(leaf);
    for (int k = nd.link; k < nd.link + nd.count; ++k) {
        const DObject o = sv.obj(k);
        const float d = obj_dist(sv, o, p, cnt, best.d);
        if (d < best.d) {
            best.d = d;
            best.mat = o.mat;
        }
    }
}

// dist_mat_warp's traversal for a three-node tree (a root and two leaves):
// the same box tests, pruning decisions, visit order and counts, with the two
// pending leaves held in registers instead of the shared-memory stack. The
// root is popped first (not counted, as in dist_mat), then the nearer leaf,
// then the other; leaves are evaluated in warp rounds of one leaf each.
template <class C>
__device__ __forceinline__ DistHit dist_mat_warp3(const SceneView& sv, V p, bool active, DistHit best, C& cnt) {
    int next = -1, last = -1;  // leaves still to pop, in order
    float dnext = 0.0f, dlast = 0.0f;
    if (active) {
        const float d0 = aabb_dist2(p, sv.node(0), cnt);
        if (!sq_ge(d0, best.d)) {
            const int l = 1, r = sv.node(0).link;
            const float dl = aabb_dist2(p, sv.node(l), cnt);
            const float dr = aabb_dist2(p, sv.node(r), cnt);
            if (sq_lt(dl, dr)) {
                next = l, dnext = dl, last = r, dlast = dr;
            } else {
                next = r, dnext = dr, last = l, dlast = dl;
            }
        }
    }
    int pending = -1;
    while (true) {
        while (pending < 0 && next >= 0) {
            cnt.add(CN_NODE);
            if (!sq_ge(dnext, best.d)) pending = next;
            next = last, dnext = dlast, last = -1;
        }
        const unsigned waiting = __ballot_sync(0xffffffffu, pending >= 0);
        if (!waiting) break;
        const int leaf = __shfl_sync(0xffffffffu, pending, __ffs(waiting) - 1);
        if (pending == leaf) {
            leaf_eval(sv, leaf, p, best, cnt);
            pending = -1;
        }
    }
    return best;
}

// dist_mat for a whole warp (all 32 lanes call it; lanes with !active only
// take part in the votes). Each active lane runs its own near-first BVH
// traversal with the reference's pruning, but leaves are evaluated in
// warp-synchronous rounds: a lane advances through interior nodes until it
// reaches a leaf that passes the AABB test; then, once every lane has either
// found one or finished, either the lanes sharing the first waiting lane's
// leaf evaluate it together (the primitive code runs converged) or, in trees
// of more than four leaves when fewer than 7/8 of the waiting lanes share
// that leaf, every waiting lane evaluates its own leaf in the same round
// (lanes at different leaves then diverge only by primitive kind, instead of
// waiting a round per leaf). A lane's sequence of node
// tests, object evaluations and best-distance updates is exactly the one
// dist_mat() makes.
template <class C>
__device__ __forceinline__ DistHit dist_mat_warp(const SceneView& sv, V p, bool active, C& cnt) {
    DistHit best{kMaxF, 0u};
    if (active) {
        cnt.add(CN_SDF);
        for (int i = 0; i < sv.n_planes; ++i) {
            const DObject o = sv.obj(i);
            float d = obj_dist(sv, o, p, cnt, best.d);
            if (d < best.d) best = DistHit{d, o.mat};
        }
    }
    if constexpr (C::kTree3) return dist_mat_warp3(sv, p, active, best, cnt);
    if (!sv.use_bvh) {
        if (active) {
            for (int k = 0; k < sv.n_objects; ++k) {
                const DObject o = sv.obj(sv.lin(k));
                float d = obj_dist(sv, o, p, cnt, best.d);
                if (d < best.d) {
                    best.d = d;
                    best.mat = o.mat;
                }
            }
        }
        return best;
    }
    if (sv.n_nodes == 0) return best;
    if (sv.n_nodes == 3) return dist_mat_warp3(sv, p, active, best, cnt);
    uint32_t* const stack = sv.stk;
    float* const stackd = sv.stkd;
    const int stride = sv.stk_stride;
    int sp = 0;
    bool first = true;
    if (active) {
        stack[0] = 0;
        stackd[0] = aabb_dist2(p, sv.node(0), cnt);
        sp = 1;
    }
    int pending = -1;
    while (true) {
        while (pending < 0 && sp > 0) {
            --sp;
            const int ni = (int)stack[sp * stride];
            const DNode nd = sv.node(ni);
            // The box distance stored at push time (see dist_mat).
            if (!first) cnt.add(CN_NODE);
            first = false;
            if (sq_ge(stackd[sp * stride], best.d)) continue;
            if (nd.count > 0) {
                pending = ni;
                break;
            }
            const int l = ni + 1, r = nd.link;
            float dl = aabb_dist2(p, sv.node(l), cnt);
            float dr = aabb_dist2(p, sv.node(r), cnt);
            if (sp + 2 > sv.stk_depth) {
                sp = 0;
                break;
            }
            if (sq_lt(dl, dr)) {
                stack[sp * stride] = (uint32_t)r;
                stackd[sp * stride] = dr;
                stack[(sp + 1) * stride] = (uint32_t)l;
                stackd[(sp + 1) * stride] = dl;
            } else {
                stack[sp * stride] = (uint32_t)l;
                stackd[sp * stride] = dl;
                stack[(sp + 1) * stride] = (uint32_t)r;
                stackd[(sp + 1) * stride] = dr;
            }
            sp += 2;
        }
        const unsigned waiting = __ballot_sync(0xffffffffu, pending >= 0);
        if (!waiting) break;
        const int leaf = __shfl_sync(0xffffffffu, pending, __ffs(waiting) - 1);
        // Trees of at most four leaves: one leaf per round, converged. Larger
        // trees: the first waiting lane's leaf is evaluated alone when at
        // least 7/8 of the waiting lanes share it; otherwise every waiting
        // lane evaluates its own leaf in this round.
        const bool shared = sv.n_nodes <= 7 || 8 * __popc(__ballot_sync(0xffffffffu, pending == leaf)) >=
                                                   7 * __popc(waiting);
        if (pending >= 0 && (pending == leaf || !shared)) {
            leaf_eval(sv, pending, p, best, cnt);
            pending = -1;
        }
    }
    return best;
}

// scene.rs:218-236: tetrahedron taps K = (1,-1,-1), (-1,-1,1), (-1,1,-1), (1,1,1).
template <class C>
__device__ __forceinline__ V scene_normal(const SceneView& sv, V p, C& cnt) {
    const float H = 5e-4f;
    V n{0.0f, 0.0f, 0.0f};
    const V K[4] = {V{1.0f, -1.0f, -1.0f}, V{-1.0f, -1.0f, 1.0f}, V{-1.0f, 1.0f, -1.0f}, V{1.0f, 1.0f, 1.0f}};
#pragma unroll
    for (int i = 0; i < 4; ++i) n = n + K[i] * scene_dist(sv, p + K[i] * H, cnt);
    float l = len(n);
    if (l > 1e-12f) return n / l;
    return V{0.0f, 1.0f, 0.0f};
}

// ------------------------------------------------------------ trace.rs ----
static constexpr uint32_t kMaxSteps = 128;    // trace.rs:10
static constexpr uint32_t kShadowSteps = 96;  // trace.rs:11

struct TraceHit {
    bool hit;
    float t;
    V p;
    uint32_t mat;
    uint32_t steps;  // includes the +4 normal taps on a hit (trace.rs:48)
};

// trace.rs:27-58 without the normal; callers that need it call
// scene_normal(hit.p), which costs exactly the four counted taps.
template <class C>
__device__ __forceinline__ TraceHit trace(const SceneView& sv, V ro, V rd, float tmin, float tmax, C& cnt) {
    float t = tmin;
    uint32_t steps = 0;
    while (steps < kMaxSteps) {
        V p = ro + rd * t;
        DistHit h = dist_mat(sv, p, cnt);
        cnt.add(CN_TSTEP);
        steps += 1;
        float eps = 1e-4f * fmaxf(t, 1.0f);
        if (h.d < eps) return TraceHit{true, t, p, h.mat, steps + 4};
        t += h.d;
        if (t > tmax) break;
    }
    return TraceHit{false, 0.0f, V{0.0f, 0.0f, 0.0f}, 0u, steps};
}

// True when this step's cone term X = k * d / max(t - y, 1e-4)
// (trace.rs:84-124) is provably >= res, so that res = min(res, X) leaves res
// unchanged and X need not be formed: y = h^2 / (2 ph) < h / 2 when h < ph
// (else y = 0), so d = sqrt(h^2 - y^2) > 0.866 h, and max(t - y, 1e-4) <=
// max(t, 1e-4). The test uses products only, with a 1e-4 relative margin over
// their rounding; NaN operands fail it, and X is then formed as usual.
__device__ __forceinline__ bool cone_cannot_lower(float h, float t, float k, float res) {
    return k * h * 0.8660f >= res * fmaxf(t, 1e-4f) * 1.0001f;
}

// trace.rs:84-124
template <class C>
__device__ __forceinline__ float soft_shadow(const SceneView& sv, V ro, V rd, float tmin, float tmax, float k,
                                             uint32_t& steps_out, C& cnt) {
    float res = 1.0f;
    float t = tmin;
    uint32_t steps = 0;
    float ph = 1e20f;
    while (steps < kShadowSteps && t < tmax) {
        float h = scene_dist(sv, ro + rd * t, cnt);
        cnt.add(CN_SSTEP);
        steps += 1;
        if (h < 1e-4f) {
            steps_out = steps;
            return 0.0f;
        }
        if (!cone_cannot_lower(h, t, k, res)) {
            float y, d;
            if (h < ph) {
                y = h * h / (2.0f * ph);
                d = sqrtf(fmaxf(h * h - y * y, 0.0f));
            } else {
                y = 0.0f;
                d = h;
            }
            res = fminf(res, k * d / fmaxf(t - y, 1e-4f));
        }
        if (res < 1e-3f) {
            steps_out = steps;
            return 0.0f;
        }
        ph = h;
        t += clampr(h, 0.006f, 0.12f);
    }
    steps_out = steps;
    return clampr(res, 0.0f, 1.0f);
}

// ------------------------------------------------- resumable ray marches ----
// The loops of trace() and soft_shadow() split into single steps, so that a
// persistent kernel can advance many rays one SDF query at a time and refill
// lanes whose ray ended. The arithmetic per step is exactly the loop body's.

// trace.rs:84-124 as a state machine.
struct ShadowRay {
    V ro, rd;
    float t, tmax, k, res, ph;
    uint32_t steps;
};
__device__ __forceinline__ ShadowRay shadow_begin(V ro, V rd, float tmin, float tmax, float k) {
    return ShadowRay{ro, rd, tmin, tmax, k, 1.0f, 1e20f, 0u};
}
// True when the march cannot take a first step (the loop body never runs).
__device__ __forceinline__ bool shadow_done_before_start(const ShadowRay& s) { return !(s.t < s.tmax); }
// One loop iteration. Returns true when the march has ended, with `vis` set.
template <class C>
__device__ __forceinline__ bool shadow_step(const SceneView& sv, ShadowRay& s, float& vis, C& cnt) {
    float h = scene_dist(sv, s.ro + s.rd * s.t, cnt);
    cnt.add(CN_SSTEP);
    s.steps += 1;
    if (h < 1e-4f) {
        vis = 0.0f;
        return true;
    }
    if (!cone_cannot_lower(h, s.t, s.k, s.res)) {
        float y, d;
        if (h < s.ph) {
            y = h * h / (2.0f * s.ph);
            d = sqrtf(fmaxf(h * h - y * y, 0.0f));
        } else {
            y = 0.0f;
            d = h;
        }
        s.res = fminf(s.res, s.k * d / fmaxf(s.t - y, 1e-4f));
    }
    if (s.res < 1e-3f) {
        vis = 0.0f;
        return true;
    }
    s.ph = h;
    s.t += clampr(h, 0.006f, 0.12f);
    if (!(s.steps < kShadowSteps && s.t < s.tmax)) {
        vis = clampr(s.res, 0.0f, 1.0f);
        return true;
    }
    return false;
}

// trace.rs:27-58 as a state machine.
struct TraceRay {
    V ro, rd;
    float t, tmax;
    uint32_t steps;
};
enum : int { kMarching = 0, kHit = 1, kMiss = 2 };
// One loop iteration. On kHit, `p`/`mat` are the hit and r.t its distance;
// r.steps then includes the four normal taps (trace.rs:48).
template <class C>
__device__ __forceinline__ int trace_step(const SceneView& sv, TraceRay& r, V& p, uint32_t& mat, C& cnt) {
    p = r.ro + r.rd * r.t;
    DistHit h = dist_mat(sv, p, cnt);
    cnt.add(CN_TSTEP);
    r.steps += 1;
    float eps = 1e-4f * fmaxf(r.t, 1.0f);
    if (h.d < eps) {
        mat = h.mat;
        r.steps += 4;
        return kHit;
    }
    r.t += h.d;
    if (r.t > r.tmax || r.steps >= kMaxSteps) return kMiss;
    return kMarching;
}

// Scene::dist (scene.rs:211-213) for a cone-shadow step, through the cell's
// candidate leaves instead of the BVH: the planes, then each listed leaf whose
// box is nearer than best + tol, its objects' minimum taken with the same
// strict `<`. Returns that minimum G; `ok` says whether G is exactly the value
// the reference's pruned near-first query (bvh.rs:100-150) returns:
//  * a leaf not listed, or listed but skipped, lies at least best + tol away,
//    and every object's distance is at least its leaf box's distance less a
//    rounding error far below tol (exact SDFs; measured below 3e-7 on the
//    stress scene), so no object outside the evaluated leaves is below G;
//  * the reference evaluates every plane, and reaches the leaf L1 holding G
//    unless it prunes L1 or an ancestor, which needs a best <= box(L1) first;
//    so G is its answer when G is a plane's, when box(L1) <= G, or when no
//    other leaf or plane reaches box(L1) (then nothing can have pruned L1).
// At or inside a surface (G <= 0) the value may differ from the reference's
// but both are below every stopping threshold of the marches that use it
// (shadow 1e-4, trace 1e-4 * max(t, 1)), so the march ends at the same step.
// Otherwise (and outside the grid) ok is false and the caller asks the
// reference query.
__device__ __forceinline__ float dist_fast(const SceneView& sv, V p, bool& ok) {
    NoCount nc;
    const LeafGrid& g = sv.lg;
    float P = kMaxF;
    for (int i = 0; i < sv.n_planes; ++i) {
        const float d = obj_dist(sv, sv.obj(i), p, nc);
        if (d < P) P = d;
    }
    ok = false;
    const float fx = (p.x - g.lo[0]) * g.inv_cell, fy = (p.y - g.lo[1]) * g.inv_cell,
                fz = (p.z - g.lo[2]) * g.inv_cell;
    if (!(fx >= 0.0f && fy >= 0.0f && fz >= 0.0f && fx < (float)g.dim[0] && fy < (float)g.dim[1] &&
          fz < (float)g.dim[2]))
        return P;
    const uint32_t cell = (uint32_t)fx + (uint32_t)g.dim[0] * ((uint32_t)fy + (uint32_t)g.dim[1] * (uint32_t)fz);
    const uint32_t e = __ldg(&g.start[cell + 1]);
    float best = P, m1 = kMaxF, m2 = kMaxF, d2_1 = 0.0f;
    for (uint32_t k = __ldg(&g.start[cell]); k < e; ++k) {
        const DNode& nd = sv.node((int)__ldg(&g.leaf[k]));
        const float d2 = aabb_dist2(p, nd, nc);
        const float lim = best + g.tol;
        if (!(lim > 0.0f) || d2 >= lim * lim) continue;
        float m = kMaxF;
        for (int j = nd.link; j < nd.link + nd.count; ++j) {
            const float d = obj_dist(sv, sv.obj(j), p, nc);
            if (d < m) m = d;
        }
        if (m < m1) {
            m2 = m1;
            m1 = m;
            d2_1 = d2;
        } else if (m < m2) {
            m2 = m;
        }
        if (m < best) best = m;
    }
    const float G = P <= m1 ? P : m1;
    // At or inside a surface: the reference's value is <= 0 too, or within
    // rounding of it (a leaf can only be pruned against a best <= its box
    // distance, which is ~0 here), so both stop the march at this step.
    if (G <= 0.0f || P <= m1) {
        ok = true;
        return G;
    }
    const float v1 = sqrtf(d2_1);
    ok = v1 <= m1 || (m2 > v1 && P > v1);
    return m1;
}

// The distance a cone-shadow step needs, for a whole warp: dist_fast where
// the scene has a leaf grid (uncounted kernels), the reference query for the
// lanes it cannot answer exactly, dist_mat_warp everywhere else.
template <class C>
__device__ __forceinline__ float shadow_dist_w(const SceneView& sv, V p, bool active, C& cnt) {
    if constexpr (sizeof(C) == 1 && !C::kTree3) {
        if (sv.lg.enabled) {
            bool ok = true;
            float h = 0.0f;
            if (active) h = dist_fast(sv, p, ok);
            const bool need = active && !ok;
            if (__any_sync(0xffffffffu, need)) {
                const float r = dist_mat_warp(sv, p, need, cnt).d;
                if (need) h = r;
            }
            return h;
        }
    }
    return dist_mat_warp(sv, p, active, cnt).d;
}

// Warp-collective forms of the two steps above: all 32 lanes call them, the
// SDF query is dist_mat_warp (shadow_dist_w for the cone march), and lanes
// with !active change nothing.
template <class C>
__device__ __forceinline__ bool shadow_step_w(const SceneView& sv, ShadowRay& s, bool active, float& vis, C& cnt) {
    const float h = shadow_dist_w(sv, s.ro + s.rd * s.t, active, cnt);
    if (!active) return false;
    cnt.add(CN_SSTEP);
    s.steps += 1;
    if (h < 1e-4f) {
        vis = 0.0f;
        return true;
    }
    if (!cone_cannot_lower(h, s.t, s.k, s.res)) {
        float y, d;
        if (h < s.ph) {
            y = h * h / (2.0f * s.ph);
            d = sqrtf(fmaxf(h * h - y * y, 0.0f));
        } else {
            y = 0.0f;
            d = h;
        }
        s.res = fminf(s.res, s.k * d / fmaxf(s.t - y, 1e-4f));
    }
    if (s.res < 1e-3f) {
        vis = 0.0f;
        return true;
    }
    s.ph = h;
    s.t += clampr(h, 0.006f, 0.12f);
    if (!(s.steps < kShadowSteps && s.t < s.tmax)) {
        vis = clampr(s.res, 0.0f, 1.0f);
        return true;
    }
    return false;
}

template <class C>
__device__ __forceinline__ int trace_step_w(const SceneView& sv, TraceRay& r, bool active, V& p, uint32_t& mat,
                                            C& cnt) {
    p = r.ro + r.rd * r.t;
    const DistHit h = dist_mat_warp(sv, p, active, cnt);
    if (!active) return kMarching;
    cnt.add(CN_TSTEP);
    r.steps += 1;
    float eps = 1e-4f * fmaxf(r.t, 1.0f);
    if (h.d < eps) {
        mat = h.mat;
        r.steps += 4;
        return kHit;
    }
    r.t += h.d;
    if (r.t > r.tmax || r.steps >= kMaxSteps) return kMiss;
    return kMarching;
}

// trace_step_w for marches that need only hit or miss and the step count
// (the hemisphere closure, trace.rs:165-186): the query is shadow_dist_w's,
// whose value is the reference's exactly, so the march is the same.
template <class C>
__device__ __forceinline__ int trace_step_dist_w(const SceneView& sv, TraceRay& r, bool active, C& cnt) {
    const float hd = shadow_dist_w(sv, r.ro + r.rd * r.t, active, cnt);
    if (!active) return kMarching;
    cnt.add(CN_TSTEP);
    r.steps += 1;
    float eps = 1e-4f * fmaxf(r.t, 1.0f);
    if (hd < eps) {
        r.steps += 4;
        return kHit;
    }
    r.t += hd;
    if (r.t > r.tmax || r.steps >= kMaxSteps) return kMiss;
    return kMarching;
}

// scene.rs:218-236 with the four taps in a rolled loop (one query site).
template <class C>
__device__ __forceinline__ V scene_normal_rolled(const SceneView& sv, V p, C& cnt) {
    const float H = 5e-4f;
    V n{0.0f, 0.0f, 0.0f};
#pragma unroll 1
    for (int i = 0; i < 4; ++i) {
        V k{(i == 0 || i == 3) ? 1.0f : -1.0f, (i >= 2) ? 1.0f : -1.0f, (i == 1 || i == 3) ? 1.0f : -1.0f};
        n = n + k * scene_dist(sv, p + k * H, cnt);
    }
    float l = len(n);
    if (l > 1e-12f) return n / l;
    return V{0.0f, 1.0f, 0.0f};
}

// ltc.rs:88-96
__device__ __forceinline__ void frame(V n, V& t, V& b) {
    float s = n.z >= 0.0f ? 1.0f : -1.0f;
    float a = -1.0f / (s + n.z);
    float bb = n.x * n.y * a;
    t = V{1.0f + s * n.x * n.x * a, s * bb, -s * n.x};
    b = V{bb, s + n.y * n.y * a, -n.y};
}

// -------------------------------------------------------------- ltc.rs ----
// ltc.rs:25-83 on a quad already in the local frame.
template <class C>
__device__ __forceinline__ float quad_form_factor(const V l[4], C& cnt) {
    V c[5];
    int n = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        V a = l[i];
        V b = l[(i + 1) & 3];
        float da = a.z, db = b.z;
        if (n < 5 && da >= 0.0f) c[n++] = a;
        if (n < 5 && (da >= 0.0f) != (db >= 0.0f)) {
            float t = da / (da - db);
            c[n++] = a + (b - a) * t;
        }
    }
    cnt.add(CN_FF);
    if (n < 3) return 0.0f;
    cnt.add(CN_FF_EDGE, (uint32_t)n);
    for (int i = 0; i < n; ++i) {
        float ln = len(c[i]);
        if (ln > 1e-9f) c[i] = c[i] / ln;
    }
    float sum = 0.0f;
    for (int i = 0; i < n; ++i) {
        V a = c[i];
        V b = c[i + 1 == n ? 0 : i + 1];
        float cos_t = clampr(dot(a, b), -1.0f, 1.0f);
        float theta = acos_f32(cos_t);
        V cr = cross(a, b);
        float ln = len(cr);
        if (ln > 1e-9f) sum += theta * (cr.z / ln);
    }
    return fmaxf(sum * 0.15915494f, 0.0f);
}

// Quad light form factor at (p, n) in the frame (t, b, n): ltc.rs:108-115
// (to_local with the winding flip) then quad_form_factor.
template <class C>
__device__ __forceinline__ float quad_light_ff(const DQuadLight& L, V p, V t, V b, V n, C& cnt) {
    V loc[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        V d = V{L.v[3 - i][0], L.v[3 - i][1], L.v[3 - i][2]} - p;
        loc[i] = V{dot(d, t), dot(d, b), dot(d, n)};
    }
    return quad_form_factor(loc, cnt);
}

// Extension: horizon-clipped sphere-light form factor (Snyder 1996 closed
// form, as written by Lagarde & de Rousiers 2014). Its acos and atan are
// libm_f32.h's, equal to glibc's acosf/atanf, which the oracle calls: the
// horizon branch subtracts nearly equal terms, so an atan that differed by
// an ulp would show as a relative difference of up to 1e-3 in the result.
__device__ __forceinline__ float sphere_light_ff(V p, V n, V c, float r) {
    V d = c - p;
    float dist2 = dot(d, d);
    float r2 = r * r;
    if (dist2 <= r2) return 0.0f;
    float dist = sqrtf(dist2);
    float cos_t = dot(n, d) / dist;
    float sin_s2 = r2 / dist2;
    if (cos_t * cos_t > sin_s2) return sin_s2 * fmaxf(cos_t, 0.0f);
    float x = sqrtf(1.0f / sin_s2 - 1.0f);
    float sin_t = sqrtf(fmaxf(1.0f - cos_t * cos_t, 0.0f));
    float y = clampr(-x * (cos_t / sin_t), -1.0f, 1.0f);
    float sty = sin_t * sqrtf(1.0f - y * y);
    float ill = (cos_t * acos_f32(y) - x * sty) * sin_s2 + atan_f32(sty / x);
    return fmaxf(ill, 0.0f) * (1.0f / kPiF);
}

// ltc.rs:119-127
__device__ __forceinline__ V closest_on_quad(const DQuadLight& L, V q) {
    V o{L.v[0][0], L.v[0][1], L.v[0][2]};
    V e1{L.e1[0], L.e1[1], L.e1[2]};
    V e2{L.e2[0], L.e2[1], L.e2[2]};
    V d = q - o;
    float u = clampr(dot(d, e1) / L.e1[3], 0.0f, 1.0f);
    float v = clampr(dot(d, e2) / L.e2[3], 0.0f, 1.0f);
    return o + e1 * u + e2 * v;
}

// ------------------------------------------------------------ shade.rs ----
__device__ __forceinline__ V fresnel_schlick(float cos_theta, V f0) {  // shade.rs:10-14
    float m = clampr(1.0f - cos_theta, 0.0f, 1.0f);
    float m2 = m * m;
    return f0 + (V{1.0f, 1.0f, 1.0f} - f0) * (m2 * m2 * m);
}
__device__ __forceinline__ float d_ggx(float n_dot_h, float alpha) {  // shade.rs:18-22
    float a2 = alpha * alpha;
    float d = n_dot_h * n_dot_h * (a2 - 1.0f) + 1.0f;
    return a2 / fmaxf(kPiF * d * d, 1e-9f);
}
__device__ __forceinline__ float v_smith(float n_dot_v, float n_dot_l, float alpha) {  // shade.rs:26-31
    float a2 = alpha * alpha;
    float gv = n_dot_l * sqrtf(n_dot_v * n_dot_v * (1.0f - a2) + a2);
    float gl = n_dot_v * sqrtf(n_dot_l * n_dot_l * (1.0f - a2) + a2);
    return 0.5f / fmaxf(gv + gl, 1e-9f);
}

// shade.rs:104-121: representative-point GGX lobe.
template <class C>
__device__ __forceinline__ void add_specular(V& out, V p, V n, V v, V rep, float radius, float alpha,
                                             float n_dot_v, V f0, V radiance, C& cnt) {
    cnt.add(CN_SPEC);
    V l = nrm(rep - p);
    float n_dot_l = dot(n, l);
    if (n_dot_l <= 0.0f) return;
    float rep_dist = fmaxf(len(rep - p), 1e-4f);
    float wide = clampr(alpha + radius / (2.0f * rep_dist), alpha, 1.0f);
    float energy = (alpha / wide) * (alpha / wide);
    V h = nrm(l + v);
    float d = d_ggx(fmaxf(dot(n, h), 0.0f), wide);
    float vis_s = v_smith(n_dot_v, n_dot_l, wide);
    V f = fresnel_schlick(fmaxf(dot(l, h), 0.0f), f0);
    out = out + f * (d * vis_s * energy * n_dot_l) * radiance;
}

// shade.rs:50-125
template <class C>
__device__ __forceinline__ V direct(const SceneView& sv, V p, V n, V v, const DMaterial& m, uint32_t& steps_out,
                                    C& cnt) {
    V out{0.0f, 0.0f, 0.0f};
    uint32_t steps = 0;
    V tan, bit;
    frame(n, tan, bit);
    float n_dot_v = fmaxf(dot(n, v), 1e-4f);
    float alpha = m.kd[3];
    V f0{m.f0[0], m.f0[1], m.f0[2]};
    V kd{m.kd[0], m.kd[1], m.kd[2]};
    for (int li = 0; li < sv.n_lights; ++li) {
        const DQuadLight& L = sv.light(li);
        V lc{L.center[0], L.center[1], L.center[2]};
        V ln{L.normal[0], L.normal[1], L.normal[2]};
        V to_light = lc - p;
        if (dot(ln, -nrm(to_light)) <= 0.0f) continue;
        float ff = quad_light_ff(L, p, tan, bit, n, cnt);
        if (ff <= 1e-6f) continue;
        cnt.add(CN_LIGHT);
        float dist = len(to_light);
        float radius = L.center[3];
        float k = clampr(dist / radius, 1.5f, 96.0f);
        V ldir = to_light / dist;
        float shadow_end = fmaxf(dist - radius * 1.25f, 0.05f);
        uint32_t s;
        float vis = soft_shadow(sv, p + n * 3e-3f, ldir, 0.015f, shadow_end, k, s, cnt);
        steps += s;
        if (vis <= 1e-4f) continue;
        V radiance = V{L.emit[0], L.emit[1], L.emit[2]} * vis;
        out = out + kd * radiance * ff;
        V r = (-v) - n * (2.0f * dot(n, -v));
        float denom = dot(r, ln);
        V rep = lc;
        if (fabsf(denom) > 1e-6f) {
            float t = dot(V{L.v[0][0], L.v[0][1], L.v[0][2]} - p, ln) / denom;
            if (t > 0.0f) rep = closest_on_quad(L, p + r * t);
        }
        add_specular(out, p, n, v, rep, radius, alpha, n_dot_v, f0, radiance, cnt);
    }
    for (int li = 0; li < sv.n_slights; ++li) {  // extension: sphere lights
        const DSphereLight& L = sv.slight(li);
        V c{L.c[0], L.c[1], L.c[2]};
        V to_light = c - p;
        float ff = sphere_light_ff(p, n, c, L.c[3]);
        if (ff <= 1e-6f) continue;
        cnt.add(CN_LIGHT);
        float dist = len(to_light);
        float radius = fmaxf(L.c[3], 1e-4f);
        float k = clampr(dist / radius, 1.5f, 96.0f);
        V ldir = to_light / dist;
        float shadow_end = fmaxf(dist - radius * 1.25f, 0.05f);
        uint32_t s;
        float vis = soft_shadow(sv, p + n * 3e-3f, ldir, 0.015f, shadow_end, k, s, cnt);
        steps += s;
        if (vis <= 1e-4f) continue;
        V radiance = V{L.emit[0], L.emit[1], L.emit[2]} * vis;
        out = out + kd * radiance * ff;
        V r = (-v) - n * (2.0f * dot(n, -v));
        V ctr = r * dot(to_light, r) - to_light;
        float cl = len(ctr);
        V rep = p + to_light + ctr * clampr(radius / fmaxf(cl, 1e-9f), 0.0f, 1.0f);
        add_specular(out, p, n, v, rep, radius, alpha, n_dot_v, f0, radiance, cnt);
    }
    steps_out = steps;
    return out;
}

// shade.rs:133-164
// terms (nullable): per light, the factor ff * vis this point receives, or
// -1 where the light is skipped (the emission-free part of each term).
template <class C>
__device__ __forceinline__ V direct_diffuse(const SceneView& sv, V p, V n, V albedo, uint32_t& steps_out, C& cnt,
                                            float* terms = nullptr) {
    V out{0.0f, 0.0f, 0.0f};
    uint32_t steps = 0;
    V tan, bit;
    frame(n, tan, bit);
    if (terms)
        for (int li = 0; li < sv.n_lights + sv.n_slights; ++li) terms[li] = -1.0f;
    for (int li = 0; li < sv.n_lights; ++li) {
        const DQuadLight& L = sv.light(li);
        V lc{L.center[0], L.center[1], L.center[2]};
        V ln{L.normal[0], L.normal[1], L.normal[2]};
        V to_light = lc - p;
        if (dot(ln, -nrm(to_light)) <= 0.0f) continue;
        float ff = quad_light_ff(L, p, tan, bit, n, cnt);
        if (ff <= 1e-6f) continue;
        cnt.add(CN_LIGHT);
        float dist = len(to_light);
        float radius = L.center[3];
        float k = clampr(dist / radius, 1.5f, 96.0f);
        float shadow_end = fmaxf(dist - radius * 1.25f, 0.05f);
        uint32_t s;
        float vis = soft_shadow(sv, p + n * 3e-3f, to_light / dist, 0.015f, shadow_end, k, s, cnt);
        steps += s;
        if (vis <= 1e-4f) continue;
        out = out + albedo * V{L.emit[0], L.emit[1], L.emit[2]} * (ff * vis);
        if (terms) terms[li] = ff * vis;
    }
    for (int li = 0; li < sv.n_slights; ++li) {  // extension: sphere lights
        const DSphereLight& L = sv.slight(li);
        V c{L.c[0], L.c[1], L.c[2]};
        V to_light = c - p;
        float ff = sphere_light_ff(p, n, c, L.c[3]);
        if (ff <= 1e-6f) continue;
        cnt.add(CN_LIGHT);
        float dist = len(to_light);
        float radius = fmaxf(L.c[3], 1e-4f);
        float k = clampr(dist / radius, 1.5f, 96.0f);
        float shadow_end = fmaxf(dist - radius * 1.25f, 0.05f);
        uint32_t s;
        float vis = soft_shadow(sv, p + n * 3e-3f, to_light / dist, 0.015f, shadow_end, k, s, cnt);
        steps += s;
        if (vis <= 1e-4f) continue;
        out = out + albedo * V{L.emit[0], L.emit[1], L.emit[2]} * (ff * vis);
        if (terms) terms[sv.n_lights + li] = ff * vis;
    }
    steps_out = steps;
    return out;
}

// shade.rs:168-181 with trace.rs:128-148 (and sphere-light entry points).
// `which` (nullable) receives the index of the light picked (quad lights,
// then sphere lights).
// quads_only: the quad lights alone (reference.rs passes &sc.lights).
__device__ __forceinline__ bool emitter_hit(const SceneView& sv, V ro, V rd, float tmax, V& emit,
                                            int* which = nullptr, bool quads_only = false) {
    bool found = false;
    float best = 0.0f;
    for (int li = 0; li < sv.n_lights; ++li) {
        const DQuadLight& L = sv.light(li);
        V nc{L.ncross[0], L.ncross[1], L.ncross[2]};
        float denom = dot(nc, rd);
        if (fabsf(denom) < 1e-9f) continue;
        V v0{L.v[0][0], L.v[0][1], L.v[0][2]};
        float t = dot(v0 - ro, nc) / denom;
        if (t < 1e-4f) continue;
        V q = ro + rd * t - v0;
        float u = dot(q, V{L.e1[0], L.e1[1], L.e1[2]}) / L.e1[3];
        float w = dot(q, V{L.e2[0], L.e2[1], L.e2[2]}) / L.e2[3];
        if (!(u >= 0.0f && u <= 1.0f && w >= 0.0f && w <= 1.0f)) continue;
        if (t < tmax && dot(V{L.normal[0], L.normal[1], L.normal[2]}, rd) < 0.0f && (!found || t < best)) {
            found = true;
            best = t;
            emit = V{L.emit[0], L.emit[1], L.emit[2]};
            if (which) *which = li;
        }
    }
    if (quads_only) return found;
    for (int li = 0; li < sv.n_slights; ++li) {
        const DSphereLight& L = sv.slight(li);
        V oc = ro - V{L.c[0], L.c[1], L.c[2]};
        float b = dot(oc, rd);
        float cc = dot(oc, oc) - L.c[3] * L.c[3];
        float disc = b * b - cc;
        if (disc < 0.0f) continue;
        float t = -b - sqrtf(disc);
        if (t < 1e-4f) continue;
        if (t < tmax && (!found || t < best)) {
            found = true;
            best = t;
            emit = V{L.emit[0], L.emit[1], L.emit[2]};
            if (which) *which = sv.n_lights + li;
        }
    }
    return found;
}

// Emission of light l (quad lights, then sphere lights).
__device__ __forceinline__ V light_emit(const SceneView& sv, int l) {
    if (l < sv.n_lights) return V{sv.light(l).emit[0], sv.light(l).emit[1], sv.light(l).emit[2]};
    const DSphereLight& S = sv.slight(l - sv.n_lights);
    return V{S.emit[0], S.emit[1], S.emit[2]};
}

// ------------------------------------------------------------ halton ------
__device__ __forceinline__ float radical_inverse(uint32_t i, uint32_t base) {  // trace.rs:189-199
    float f = 1.0f, r = 0.0f;
    float inv = 1.0f / (float)base;
    while (i > 0) {
        f *= inv;
        r += f * (float)(i % base);
        i /= base;
    }
    return r;
}

// ------------------------------------------------------------ gather ------
// Surfel grid in item order: gp/gn/girr are the surfels' p, n, irr copied
// in the grid's cell order, so each cell is a contiguous run.
struct GatherView {
    const float4* gp;
    const float4* gn;
    const float4* girr;
    const uint32_t* starts;
    int dim[3];
    float lo[3];
    float inv_cell;
    float radius;
};

// surfel.rs:262-293 with the cell walk of surfel.rs:127-140.
template <class C>
__device__ __forceinline__ V gather(const GatherView& g, V p, V n, C& cnt) {
    V acc{0.0f, 0.0f, 0.0f};
    float wsum = 0.0f;
    float r2 = g.radius * g.radius;
    int cx = clampi(as_i32((p.x - g.lo[0]) * g.inv_cell), 0, g.dim[0] - 1);
    int cy = clampi(as_i32((p.y - g.lo[1]) * g.inv_cell), 0, g.dim[1] - 1);
    int cz = clampi(as_i32((p.z - g.lo[2]) * g.inv_cell), 0, g.dim[2] - 1);
    for (int z = max(cz - 1, 0); z <= min(cz + 1, g.dim[2] - 1); ++z)
        for (int y = max(cy - 1, 0); y <= min(cy + 1, g.dim[1] - 1); ++y) {
            // Cells x-1..x+1 of one row are adjacent in the cell order, so
            // their items form one contiguous run.
            size_t row = (size_t)g.dim[0] * ((size_t)y + (size_t)g.dim[1] * (size_t)z);
            int x0 = max(cx - 1, 0), x1 = min(cx + 1, g.dim[0] - 1);
            uint32_t s = __ldg(&g.starts[row + x0]);
            uint32_t e = __ldg(&g.starts[row + x1 + 1]);
            for (uint32_t k = s; k < e; ++k) {
                float4 sp = __ldg(&g.gp[k]);
                cnt.add(CN_GVISIT);
                float d2 = dot(mk4(sp) - p, mk4(sp) - p);
                if (d2 > r2) continue;
                float4 sn = __ldg(&g.gn[k]);
                float align = dot(mk4(sn), n);
                if (align <= 0.15f) continue;
                float t = 1.0f - d2 / r2;
                float w = t * t * align;
                cnt.add(CN_GACCEPT);
                float4 ir = __ldg(&g.girr[k]);
                acc = acc + mk4(ir) * w;
                wsum += w;
            }
        }
    if (wsum > 1e-6f) return acc / wsum;
    return V{0.0f, 0.0f, 0.0f};
}

}  // namespace ifx
