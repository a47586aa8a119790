// Per-pixel shading (main.rs:229-367) with the film encode (film.rs:8-61)
// as a wavefront of kernels, so that every ray march runs in a persistent
// kernel with one SDF query site and full warps:
//
//   k_primary    camera rays (one lane per pixel, refilled)      -> hit 1
//   k_setup      emitter / sky / debug modes, normal, per-light
//                form factors; queues shadow rays and mirror rays
//   k_shadow     cone shadows of the primary hits               -> vis 1
//   k_reflect    mirror rays of glossy pixels                    -> hit 2
//   k_setup2     emitter test, normal and form factors at hit 2
//   k_shadow     cone shadows of the mirror hits                -> vis 2
//   k_compose    direct() recomputed from the stored form factors and
//                visibilities in the reference's operation order, the
//                gathers, the mirror term, then the sRGB encode
//
// Queue order depends on scheduling, but every result is written to a slot
// fixed by pixel and light, and every float sum is formed in k_compose in
// the reference's order, so the image is bit-identical across runs.
#include "shade.cuh"
#include "pixorder.h"

namespace ifx {

static constexpr uint32_t kFlagHit = kPixHit;
static constexpr uint32_t kFlagDone = kPixDone;
static constexpr uint32_t kFlagEmit = kPixEmit;
static constexpr uint32_t kMatMask = kPixMatMask;

// ------------------------------------------------------------ kernels ----
// Camera rays: trace.rs:27-58 from the eye (main.rs:261), pixels taken in
// 8 x 4 tiles (pixorder.h). hn1 keeps the march's step count in x until
// k_setup replaces it with the normal.
template <class C>
__global__ void __launch_bounds__(128) k_primary(ShadeParams P) {
    IFX_SCENE_PROLOGUE(P.blob, P.status, sv);
    C cnt;
    const unsigned long long total = (unsigned long long)P.w * P.h;
    WarpQueue q(total);
    const V org{P.cam.origin[0], P.cam.origin[1], P.cam.origin[2]};
    uint32_t item = ~0u;
    TraceRay ray{};
    unsigned long long ev = 0;
    while (true) {
        const uint32_t got = q.refill(item == ~0u, total, &P.cursors[0]);
        if (got != ~0u) {
            const uint32_t pix = tile_pixel(got, P.w, P.h);
            ray = TraceRay{org, camera_ray(P, pix), 1e-3f, P.tmax, 0u};
            item = pix;
        }
        if (!__any_sync(kFull, item != ~0u)) {
            if (q.empty()) break;
            continue;
        }
        const bool active = item != ~0u;
        V hp;
        uint32_t hm = 0;
        const int st = trace_step_w(sv, ray, active, hp, hm, cnt);
        if (active && st != kMarching) {
            ev += ray.steps;
            const bool hit = st == kHit;
            P.hp1[item] = make_float4(hit ? hp.x : 0.0f, hit ? hp.y : 0.0f, hit ? hp.z : 0.0f, ray.t);
            P.hn1[item] = make_float4(__uint_as_float(ray.steps), 0.0f, 0.0f,
                                      __uint_as_float((hit ? kFlagHit : 0u) | (hm & kMatMask)));
            item = ~0u;
        }
    }
    add_evals(ev, P.evals);
    if constexpr (sizeof(C) > 1) cnt.flush(P.counts);
}

// main.rs:264-296 up to the direct-light call: emitter and sky pixels, the
// debug modes, the hit normal, and the per-light form factors whose cones
// k_shadow traces. Glossy hits are queued for a mirror ray (main.rs:322).
template <class C>
__global__ void __launch_bounds__(128) k_setup(ShadeParams P) {
    IFX_SCENE_PROLOGUE(P.blob, P.status, sv);
    C cnt;
    __shared__ float t8[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) t8[i] = P.srgb_t[i];
    __syncthreads();
    const uint32_t total = P.w * P.h;
    const V org{P.cam.origin[0], P.cam.origin[1], P.cam.origin[2]};
    const bool tonemapped = P.mode <= 2;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const uint32_t pix = tile_pixel(t, P.w, P.h);  // the queues then fill in tile order
        const float4 a = P.hp1[pix];
        const float4 b = P.hn1[pix];
        const uint32_t flags = __float_as_uint(b.w);
        const bool hit = (flags & kFlagHit) != 0;
        const V rd = camera_ray(P, pix);
        V e;
        int which = 0;
        if (emitter_hit(sv, org, rd, fminf(hit ? a.w : kMaxF, P.tmax), e, &which)) {
            write_pixel(P, t8, pix, tonemapped ? e : V{0.9f, 0.9f, 0.9f});
            // The light's index stays with the pixel for re-composition.
            P.hn1[pix] = make_float4(b.x, __uint_as_float((uint32_t)which), 0.0f,
                                     __uint_as_float(flags | kFlagDone | kFlagEmit));
            continue;
        }
        if (!hit) {
            write_pixel(P, t8, pix, sky());
            P.hn1[pix].w = __uint_as_float(flags | kFlagDone);
            continue;
        }
        if (P.mode == 4) {  // depth
            float d = 1.0f - clampr(a.w / P.tmax, 0.0f, 1.0f);
            write_pixel(P, t8, pix, V{d * d, d * d, d * d});
            P.hn1[pix].w = __uint_as_float(flags | kFlagDone);
            continue;
        }
        if (P.mode == 5) {  // steps
            float f = (float)__float_as_uint(b.x) / 128.0f;
            write_pixel(P, t8, pix, V{f, 1.0f - f, 0.2f});
            P.hn1[pix].w = __uint_as_float(flags | kFlagDone);
            continue;
        }
        const V p = mk4(a);
        const V n = scene_normal_rolled(sv, p, cnt);
        if (P.mode == 3) {  // normals
            write_pixel(P, t8, pix, n * 0.5f + V{0.5f, 0.5f, 0.5f});
            P.hn1[pix].w = __uint_as_float(flags | kFlagDone);
            continue;
        }
        P.hn1[pix] = f4(n, b.w);
        if (P.mode != 2) {
            V tan, bit;
            frame(n, tan, bit);
            for (int l = 0; l < P.nl; ++l) {
                const float ff = light_ff(sv, l, p, n, tan, bit, cnt);
                const uint32_t slot = pix * (uint32_t)P.nl + (uint32_t)l;
                P.ff1[slot] = ff;
                if (ff > 1e-6f) enqueue(P.q1, &P.qlen[0], slot);
            }
        }
        if (P.has_gi && sv.mat(flags & kMatMask).f0[3] != 0.0f) enqueue(P.qr, &P.qlen[1], pix);
    }
    if constexpr (sizeof(C) > 1) cnt.flush(P.counts);
}

// shade.rs:75-84: the cone shadow toward each queued light.
template <class C>
__global__ void __launch_bounds__(128) k_shadow(ShadeParams P, const float4* hp, const float4* hn,
                                                 const uint32_t* queue, const uint32_t* qlen, float* vis_out,
                                                 unsigned long long* cursor) {
    IFX_SCENE_PROLOGUE(P.blob, P.status, sv);
    C cnt;
    const unsigned long long total = *qlen;
    WarpQueue q(total);
    uint32_t item = ~0u;
    ShadowRay ray{};
    unsigned long long ev = 0;
    while (true) {
        const uint32_t got = q.refill(item == ~0u, total, cursor);
        if (got != ~0u) {
            const uint32_t slot = queue[got];
            const uint32_t pix = slot / (uint32_t)P.nl;
            const int l = (int)(slot - pix * (uint32_t)P.nl);
            const V p = mk4(hp[pix]), n = mk4(hn[pix]);
            const LightGeom g = light_geom(sv, l, p);
            float dist = len(g.to_light);
            float k = clampr(dist / g.radius, 1.5f, 96.0f);
            V ldir = g.to_light / dist;
            float shadow_end = fmaxf(dist - g.radius * 1.25f, 0.05f);
            ray = shadow_begin(p + n * 3e-3f, ldir, 0.015f, shadow_end, k);
            if (shadow_done_before_start(ray)) vis_out[slot] = clampr(ray.res, 0.0f, 1.0f);
            else item = slot;
        }
        if (!__any_sync(kFull, item != ~0u)) {
            if (q.empty()) break;
            continue;
        }
        const bool active = item != ~0u;
        float vis;
        if (shadow_step_w(sv, ray, active, vis, cnt) && active) {
            vis_out[item] = vis;
            ev += ray.steps;
            item = ~0u;
        }
    }
    add_evals(ev, P.evals);
    if constexpr (sizeof(C) > 1) cnt.flush(P.counts);
}

// main.rs:323-326: the mirror ray of each queued glossy pixel.
template <class C>
__global__ void __launch_bounds__(128) k_reflect(ShadeParams P) {
    IFX_SCENE_PROLOGUE(P.blob, P.status, sv);
    C cnt;
    const unsigned long long total = P.qlen[1];
    WarpQueue q(total);
    uint32_t item = ~0u, pix = 0;
    TraceRay ray{};
    unsigned long long ev = 0;
    while (true) {
        const uint32_t got = q.refill(item == ~0u, total, &P.cursors[1]);
        if (got != ~0u) {
            pix = P.qr[got];
            const V rd = camera_ray(P, pix);
            const V p = mk4(P.hp1[pix]), n = mk4(P.hn1[pix]);
            const V refl = rd - n * (2.0f * dot(n, rd));
            ray = TraceRay{p + n * 1e-3f, refl, 1e-3f, P.tmax, 0u};
            item = got;
        }
        if (!__any_sync(kFull, item != ~0u)) {
            if (q.empty()) break;
            continue;
        }
        const bool active = item != ~0u;
        V hp;
        uint32_t hm = 0;
        const int st = trace_step_w(sv, ray, active, hp, hm, cnt);
        if (active && st != kMarching) {
            ev += ray.steps;
            const bool hit = st == kHit;
            P.hp2[pix] = make_float4(hit ? hp.x : 0.0f, hit ? hp.y : 0.0f, hit ? hp.z : 0.0f, ray.t);
            P.hn2[pix] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float((hit ? kFlagHit : 0u) | (hm & kMatMask)));
            item = ~0u;
        }
    }
    add_evals(ev, P.evals);
    if constexpr (sizeof(C) > 1) cnt.flush(P.counts);
}

// main.rs:328-340 up to the direct-light call at the mirror hit.
template <class C>
__global__ void __launch_bounds__(128) k_setup2(ShadeParams P) {
    IFX_SCENE_PROLOGUE(P.blob, P.status, sv);
    C cnt;
    const uint32_t total = P.qlen[1];
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < total; j += gridDim.x * blockDim.x) {
        const uint32_t pix = P.qr[j];
        const V rd = camera_ray(P, pix);
        const V p = mk4(P.hp1[pix]), n = mk4(P.hn1[pix]);
        const V refl = rd - n * (2.0f * dot(n, rd));
        const float4 a = P.hp2[pix];
        const uint32_t flags = __float_as_uint(P.hn2[pix].w);
        const bool hit = (flags & kFlagHit) != 0;
        V e;
        int which = 0;
        if (emitter_hit(sv, p, refl, fminf(hit ? a.w : kMaxF, P.tmax), e, &which)) {
            P.hn2[pix] = make_float4(__uint_as_float((uint32_t)which), 0.0f, 0.0f,
                                     __uint_as_float(flags | kFlagEmit));
            continue;
        }
        if (!hit) continue;
        const V p2 = mk4(a);
        const V n2 = scene_normal_rolled(sv, p2, cnt);
        P.hn2[pix] = f4(n2, __uint_as_float(flags));
        V tan, bit;
        frame(n2, tan, bit);
        for (int l = 0; l < P.nl; ++l) {
            const float ff = light_ff(sv, l, p2, n2, tan, bit, cnt);
            const uint32_t slot = pix * (uint32_t)P.nl + (uint32_t)l;
            P.ff2[slot] = ff;
            if (ff > 1e-6f) enqueue(P.q2, &P.qlen[2], slot);
        }
    }
    if constexpr (sizeof(C) > 1) cnt.flush(P.counts);
}

// main.rs:289-358: the pixel's colour from the stored hits, form factors and
// visibilities, in the reference's order of operations, then film.rs encode.
template <class C>
__global__ void __launch_bounds__(128) k_compose(ShadeParams P) {
    IFX_SCENE_PROLOGUE(P.blob, P.status, sv);
    C cnt;
    __shared__ float t8[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) t8[i] = P.srgb_t[i];
    __syncthreads();
    const uint32_t end = P.pix1 ? P.pix1 : P.w * P.h;
    const GatherView g = gview(P.grid);
    for (uint32_t pix = P.pix0 + blockIdx.x * blockDim.x + threadIdx.x; pix < end; pix += gridDim.x * blockDim.x)
        compose_pixel(sv, P, t8, g, pix, cnt);
    if constexpr (sizeof(C) > 1) cnt.flush(P.counts);
}

// ev (nullable): kShadeEvents events recorded around the kernels, in
// pairs: [0,1] primary, [2,3] shadow, [4,5] reflect, [6,7] shadow2, and the
// rest as [8,9] setup, [10,11] setup2, [12,13] compose. Work counters go to
// slots (kNumCounters u64 each) 0 primary, 1 shadow, 2 reflect, 3 shadow2,
// 4 the rest.
template <class C>
static void launch_all(cudaStream_t st, const ShadeParams& p, cudaEvent_t* ev, int part) {
    const size_t sm = blob_smem(p.blob, 128);
    const unsigned long long px = (unsigned long long)p.w * p.h;
    const unsigned long long slots = px * (unsigned long long)(p.nl > 0 ? p.nl : 1);
    auto with = [&](int slot) {
        ShadeParams q = p;
        q.counts = p.counts ? p.counts + (size_t)slot * kNumCounters : nullptr;
        return q;
    };
    auto rec = [&](int i) {
        if (ev) cudaEventRecord(ev[i], st);
    };
    if (part & kShadeFront) {
        rec(0);
        k_primary<C><<<persistent_grid(k_primary<C>, 128, sm, px), 128, sm, st>>>(with(0));
        rec(1);
        rec(8);
        k_setup<C><<<grid_for(px, 128, 16), 128, sm, st>>>(with(4));
        rec(9);
        rec(2);
        k_shadow<C><<<persistent_grid(k_shadow<C>, 128, sm, slots), 128, sm, st>>>(
            with(1), p.hp1, p.hn1, p.q1, &p.qlen[0], p.vis1, &p.cursors[2]);
        rec(3);
        rec(4);
        if (p.has_gi) k_reflect<C><<<persistent_grid(k_reflect<C>, 128, sm, px), 128, sm, st>>>(with(2));
        rec(5);
        rec(10);
        if (p.has_gi) k_setup2<C><<<grid_for(px, 128, 16), 128, sm, st>>>(with(4));
        rec(11);
        rec(6);
        if (p.has_gi)
            k_shadow<C><<<persistent_grid(k_shadow<C>, 128, sm, slots), 128, sm, st>>>(
                with(3), p.hp2, p.hn2, p.q2, &p.qlen[2], p.vis2, &p.cursors[3]);
        rec(7);
    }
    if (part & kShadeCompose) {
        rec(12);
        const unsigned long long cpx = p.pix1 ? (unsigned long long)(p.pix1 - p.pix0) : px;
        k_compose<C><<<grid_for(cpx, 128, 16), 128, sm, st>>>(with(4));
        rec(13);
    }
}

int launch_shade(cudaStream_t st, const ShadeParams& p, cudaEvent_t* ev, int part) {
    if (p.counts) launch_all<Counts>(st, p, ev, part);
    else if (p.blob.tree3) launch_all<NoCount3>(st, p, ev, part);
    else launch_all<NoCount>(st, p, ev, part);
    return ((part & kShadeFront) ? (p.has_gi ? 6 : 3) : 0) + ((part & kShadeCompose) ? 1 : 0);
}

// ---------------------------------------------------------------------------
// solve.rs:27-39 (light_surfels) as three passes over (surfel, light) slots:
// k_light_setup stores each slot's form factor (shade.rs:60-73) and queues
// the slots that pass the 1e-6 cut; k_shadow marches their cones (the same
// march, origin offset and end as the light stage's); k_light_compose sums
// the lights per surfel in the reference's order. Slot = surfel * nl + light
// (quad lights, then sphere lights).
template <class C>
__global__ void __launch_bounds__(128) k_light_setup(ShadeParams P, const float4* sp, const float4* sn, uint32_t n,
                                                     float* ff_out) {
    IFX_SCENE_PROLOGUE(P.blob, P.status, sv);
    C cnt;
    const int nl = P.nl;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V p = mk4(sp[i]), nn = mk4(sn[i]);
        V tan, bit;
        frame(nn, tan, bit);
        for (int l = 0; l < nl; ++l) {
            const float ff = light_ff(sv, l, p, nn, tan, bit, cnt);
            const uint32_t slot = i * (uint32_t)nl + (uint32_t)l;
            ff_out[slot] = ff;
            if (!(ff <= 1e-6f)) {  // shade.rs:65: a light is skipped when ff <= 1e-6
                cnt.add(CN_LIGHT);
                enqueue(P.q1, &P.qlen[0], slot);
            }
        }
    }
    if constexpr (sizeof(C) > 1) cnt.flush(P.counts);
}

__global__ void __launch_bounds__(128) k_light_compose(ShadeParams P, SurfelArrays s, uint32_t n, const float* ff,
                                                       const float* vis, float* terms) {
    IFX_SCENE_PROLOGUE(P.blob, P.status, sv);
    const int nl = P.nl;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V albedo = mk4(s.albedo[i]);
        V out{0.0f, 0.0f, 0.0f};
        for (int l = 0; l < nl; ++l) {
            const size_t slot = (size_t)i * nl + l;
            if (terms) terms[slot] = -1.0f;
            const float f = ff[slot];
            if (f <= 1e-6f) continue;
            const float v = vis[slot];
            if (v <= 1e-4f) continue;
            const float* e = l < sv.n_lights ? sv.light(l).emit : sv.slight(l - sv.n_lights).emit;
            out = out + albedo * V{e[0], e[1], e[2]} * (f * v);
            if (terms) terms[slot] = f * v;
        }
        s.direct[i] = f4(out, 0.0f);
        s.rad[i] = f4(out, 0.0f);
        s.irr[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

int launch_light_slots(cudaStream_t st, const ShadeParams& p, const SurfelArrays& s, uint32_t n, float* ff,
                       float* vis, float* terms, unsigned long long* cursor) {
    const size_t sm = blob_smem(p.blob, 128);
    const unsigned long long slots = (unsigned long long)n * (unsigned long long)(p.nl > 0 ? p.nl : 1);
    if (p.counts) {
        k_light_setup<Counts><<<grid_for(n, 128, 16), 128, sm, st>>>(p, s.p, s.n, n, ff);
        k_shadow<Counts><<<persistent_grid(k_shadow<Counts>, 128, sm, slots), 128, sm, st>>>(
            p, s.p, s.n, p.q1, &p.qlen[0], vis, cursor);
    } else if (p.blob.tree3) {
        k_light_setup<NoCount3><<<grid_for(n, 128, 16), 128, sm, st>>>(p, s.p, s.n, n, ff);
        k_shadow<NoCount3><<<persistent_grid(k_shadow<NoCount3>, 128, sm, slots), 128, sm, st>>>(
            p, s.p, s.n, p.q1, &p.qlen[0], vis, cursor);
    } else {
        k_light_setup<NoCount><<<grid_for(n, 128, 16), 128, sm, st>>>(p, s.p, s.n, n, ff);
        k_shadow<NoCount><<<persistent_grid(k_shadow<NoCount>, 128, sm, slots), 128, sm, st>>>(
            p, s.p, s.n, p.q1, &p.qlen[0], vis, cursor);
    }
    k_light_compose<<<grid_for(n, 128, 16), 128, sm, st>>>(p, s, n, ff, vis, terms);
    return 3;
}

int launch_compose(cudaStream_t st, const ShadeParams& p) {
    const size_t sm = blob_smem(p.blob, 128);
    ShadeParams q = p;
    q.counts = nullptr;
    if (p.blob.tree3)
        k_compose<NoCount3><<<grid_for((unsigned long long)p.w * p.h, 128, 16), 128, sm, st>>>(q);
    else
        k_compose<NoCount><<<grid_for((unsigned long long)p.w * p.h, 128, 16), 128, sm, st>>>(q);
    return 1;
}

template <class C>
static void configure_one(int max_dyn_smem) {
    cudaFuncSetAttribute(k_primary<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_setup<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_shadow<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_reflect<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_setup2<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_compose<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
}

void configure_shade_kernels(int max_dyn_smem) {
    configure_one<NoCount>(max_dyn_smem);
    configure_one<NoCount3>(max_dyn_smem);
    configure_one<Counts>(max_dyn_smem);
    cudaFuncSetAttribute(k_light_setup<NoCount>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_light_setup<NoCount3>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_light_setup<Counts>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_light_compose, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
}

}  // namespace ifx
