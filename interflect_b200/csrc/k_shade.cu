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
#include "kcommon.cuh"

namespace ifx {

static constexpr uint32_t kFlagHit = kPixHit;
static constexpr uint32_t kFlagDone = kPixDone;
static constexpr uint32_t kFlagEmit = kPixEmit;
static constexpr uint32_t kMatMask = kPixMatMask;

__device__ __forceinline__ V sky() { return V{0.02f, 0.03f, 0.05f}; }

// film.rs:8-17
__device__ __forceinline__ V aces(V x) {
    const float A = 2.51f, B = 0.03f, C = 2.43f, D = 0.59f, E = 0.14f;
    V num = x * (x * A + V{B, B, B});
    V den = x * (x * C + V{D, D, D}) + V{E, E, E};
    V r = V{num.x / den.x, num.y / den.y, num.z / den.z};
    return V{fminf(fmaxf(r.x, 0.0f), 1.0f), fminf(fmaxf(r.y, 0.0f), 1.0f), fminf(fmaxf(r.z, 0.0f), 1.0f)};
}

// film.rs:23-31 via the host-computed step thresholds: the byte is the
// number of thresholds t[1..255] not above the clamped input (NaN -> 0).
__device__ __forceinline__ uint8_t srgb8(const float* t, float c) {
    c = clampr(c, 0.0f, 1.0f);
    int lo = 0;
#pragma unroll
    for (int step = 128; step >= 1; step >>= 1)
        if (lo + step <= 255 && t[lo + step] <= c) lo += step;
    return (uint8_t)lo;
}

__device__ __forceinline__ void write_pixel(const ShadeParams& P, const float* t8, uint32_t pix, V c) {
    const size_t o = (size_t)pix * 3;
    if (P.film) {
        P.film[o] = c.x;
        P.film[o + 1] = c.y;
        P.film[o + 2] = c.z;
    }
    V s = c * P.exposure;
    V m = P.tonemap ? aces(s) : s;
    P.out8[o] = srgb8(t8, m.x);
    P.out8[o + 1] = srgb8(t8, m.y);
    P.out8[o + 2] = srgb8(t8, m.z);
}

// main.rs:213-217
__device__ __forceinline__ V camera_ray(const ShadeParams& P, uint32_t pix) {
    const CamParams& c = P.cam;
    const uint32_t x = pix % P.w, y = pix / P.w;
    float px = (2.0f * ((float)x + 0.5f) / (float)P.w - 1.0f) * c.aspect * c.tan_half;
    float py = (1.0f - 2.0f * ((float)y + 0.5f) / (float)P.h) * c.tan_half;
    return nrm(V{c.fwd[0], c.fwd[1], c.fwd[2]} + V{c.right[0], c.right[1], c.right[2]} * px +
               V{c.up[0], c.up[1], c.up[2]} * py);
}

__device__ __forceinline__ GatherView gview(const GridParams& g) {
    GatherView v;
    v.gp = g.gp;
    v.gn = g.gn;
    v.girr = g.girr;
    v.starts = g.starts;
    v.dim[0] = g.dim[0]; v.dim[1] = g.dim[1]; v.dim[2] = g.dim[2];
    v.lo[0] = g.lo[0]; v.lo[1] = g.lo[1]; v.lo[2] = g.lo[2];
    v.inv_cell = g.inv_cell;
    v.radius = g.radius;
    return v;
}

// Appends v to a queue; the active lanes of the warp take consecutive slots
// with one atomic.
__device__ __forceinline__ void enqueue(uint32_t* q, uint32_t* len, uint32_t v) {
    const unsigned m = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(len, (uint32_t)__popc(m));
    base = __shfl_sync(m, base, leader);
    q[base + __popc(m & ((1u << lane) - 1u))] = v;
}

__device__ __forceinline__ void add_evals(unsigned long long ev, unsigned long long* out) {
    for (int o = 16; o >= 1; o >>= 1) ev += __shfl_xor_sync(kFull, ev, o);
    if ((threadIdx.x & 31) == 0 && ev) atomicAdd(out, ev);
}

// Light l of the scene's light list (quad lights, then sphere lights): the
// centre-to-point vector and cone radius as shade.rs:61-79 computes them.
struct LightGeom {
    V to_light;
    float radius;
};
__device__ __forceinline__ LightGeom light_geom(const SceneView& sv, int l, V p) {
    if (l < sv.n_lights) {
        const DQuadLight& L = sv.lights[l];
        return LightGeom{V{L.center[0], L.center[1], L.center[2]} - p, L.center[3]};
    }
    const DSphereLight& S = sv.slights[l - sv.n_lights];
    return LightGeom{V{S.c[0], S.c[1], S.c[2]} - p, fmaxf(S.c[3], 1e-4f)};
}

// shade.rs:60-73: the back-face cull and the exact diffuse form factor of
// light l (sphere lights: the horizon-clipped sphere form factor); -1 when
// the light is culled.
template <class C>
__device__ __forceinline__ float light_ff(const SceneView& sv, int l, V p, V n, V tan, V bit, C& cnt) {
    if (l < sv.n_lights) {
        const DQuadLight& L = sv.lights[l];
        V to_light = V{L.center[0], L.center[1], L.center[2]} - p;
        if (dot(V{L.normal[0], L.normal[1], L.normal[2]}, -nrm(to_light)) <= 0.0f) return -1.0f;
        return quad_light_ff(L, p, tan, bit, n, cnt);
    }
    const DSphereLight& S = sv.slights[l - sv.n_lights];
    return sphere_light_ff(p, n, V{S.c[0], S.c[1], S.c[2]}, S.c[3]);
}

// shade.rs:50-125 with the form factors and visibilities of this point's
// lights read from its slots (ff <= 1e-6 or a culled light skip, as there).
template <class C>
__device__ __forceinline__ V direct_from_slots(const SceneView& sv, V p, V n, V v, const DMaterial& m,
                                               const float* ffs, const float* viss, C& cnt) {
    V out{0.0f, 0.0f, 0.0f};
    float n_dot_v = fmaxf(dot(n, v), 1e-4f);
    float alpha = m.kd[3];
    V f0{m.f0[0], m.f0[1], m.f0[2]};
    V kd{m.kd[0], m.kd[1], m.kd[2]};
    for (int li = 0; li < sv.n_lights; ++li) {
        const DQuadLight& L = sv.lights[li];
        V lc{L.center[0], L.center[1], L.center[2]};
        V ln{L.normal[0], L.normal[1], L.normal[2]};
        V to_light = lc - p;
        if (dot(ln, -nrm(to_light)) <= 0.0f) continue;
        float ff = ffs[li];
        if (ff <= 1e-6f) continue;
        float radius = L.center[3];
        float vis = viss[li];
        if (vis <= 1e-4f) continue;
        cnt.add(CN_LIGHT);
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
    for (int si = 0; si < sv.n_slights; ++si) {
        const int li = sv.n_lights + si;
        const DSphereLight& S = sv.slights[si];
        V to_light = V{S.c[0], S.c[1], S.c[2]} - p;
        float ff = ffs[li];
        if (ff <= 1e-6f) continue;
        float radius = fmaxf(S.c[3], 1e-4f);
        float vis = viss[li];
        if (vis <= 1e-4f) continue;
        cnt.add(CN_LIGHT);
        V radiance = V{S.emit[0], S.emit[1], S.emit[2]} * vis;
        out = out + kd * radiance * ff;
        V r = (-v) - n * (2.0f * dot(n, -v));
        V ctr = r * dot(to_light, r) - to_light;
        float cl = len(ctr);
        V rep = p + to_light + ctr * clampr(radius / fmaxf(cl, 1e-9f), 0.0f, 1.0f);
        add_specular(out, p, n, v, rep, radius, alpha, n_dot_v, f0, radiance, cnt);
    }
    return out;
}

// ------------------------------------------------------------ kernels ----
// Camera rays: trace.rs:27-58 from the eye (main.rs:261). hn1 keeps the
// march's step count in x until k_setup replaces it with the normal.
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
            ray = TraceRay{org, camera_ray(P, got), 1e-3f, P.tmax, 0u};
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
    for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < total; pix += gridDim.x * blockDim.x) {
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
        if (P.has_gi && sv.mats[flags & kMatMask].f0[3] != 0.0f) enqueue(P.qr, &P.qlen[1], pix);
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
    const uint32_t total = P.w * P.h;
    const GatherView g = gview(P.grid);
    const int nl = P.nl;
    for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < total; pix += gridDim.x * blockDim.x) {
        const float4 b = P.hn1[pix];
        const uint32_t flags = __float_as_uint(b.w);
        if (flags & kFlagDone) {
            // Sky and debug pixels are final; an emitter pixel follows its
            // light's current emission when the frame is re-composed.
            if (P.recompose && (flags & kFlagEmit)) write_pixel(P, t8, pix, light_emit(sv, (int)__float_as_uint(b.y)));
            continue;
        }
        const V rd = camera_ray(P, pix);
        const V p = mk4(P.hp1[pix]), n = mk4(b);
        const DMaterial& m = sv.mats[flags & kMatMask];
        V col{0.0f, 0.0f, 0.0f};
        if (P.mode != 2) {
            V d = direct_from_slots(sv, p, n, -rd, m, P.ff1 + (size_t)pix * nl, P.vis1 + (size_t)pix * nl, cnt);
            col = col + (d + V{m.emissive[0], m.emissive[1], m.emissive[2]});
        }
        if (P.has_gi) {
            V irr = gather(g, p, n, cnt);
            col = col + V{m.kd[0], m.kd[1], m.kd[2]} * irr;
            if (m.f0[3] != 0.0f) {
                const V refl = rd - n * (2.0f * dot(n, rd));
                const float4 a2 = P.hp2[pix];
                const float4 b2 = P.hn2[pix];
                const uint32_t f2 = __float_as_uint(b2.w);
                V rc;
                if (f2 & kFlagEmit) {
                    rc = light_emit(sv, (int)__float_as_uint(b2.x));
                } else if (f2 & kFlagHit) {
                    const V p2 = mk4(a2), n2 = mk4(b2);
                    const DMaterial& m2 = sv.mats[f2 & kMatMask];
                    V d2 = direct_from_slots(sv, p2, n2, -refl, m2, P.ff2 + (size_t)pix * nl,
                                             P.vis2 + (size_t)pix * nl, cnt);
                    V i2 = gather(g, p2, n2, cnt);
                    rc = d2 + V{m2.kd[0], m2.kd[1], m2.kd[2]} * i2 +
                         V{m2.emissive[0], m2.emissive[1], m2.emissive[2]};
                } else {
                    rc = sky();
                }
                V f = fresnel_schlick(fmaxf(dot(n, -rd), 0.0f), V{m.f0[0], m.f0[1], m.f0[2]});
                float gloss = clampr(1.0f - m.albedo[3] / 0.45f, 0.0f, 1.0f);
                gloss = gloss * gloss;
                col = col + f * rc * gloss;
            }
        }
        write_pixel(P, t8, pix, col);
    }
    if constexpr (sizeof(C) > 1) cnt.flush(P.counts);
}

// ev (nullable): kShadeEvents events recorded around the kernels, in
// pairs: [0,1] primary, [2,3] shadow, [4,5] reflect, [6,7] shadow2, and the
// rest as [8,9] setup, [10,11] setup2, [12,13] compose. Work counters go to
// slots (kNumCounters u64 each) 0 primary, 1 shadow, 2 reflect, 3 shadow2,
// 4 the rest.
template <class C>
static void launch_all(cudaStream_t st, const ShadeParams& p, cudaEvent_t* ev) {
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
    rec(0);
    k_primary<C><<<persistent_grid(k_primary<C>, 128, sm, px), 128, sm, st>>>(with(0));
    rec(1);
    rec(8);
    k_setup<C><<<grid_for(px, 128, 16), 128, sm, st>>>(with(4));
    rec(9);
    rec(2);
    k_shadow<C><<<persistent_grid(k_shadow<C>, 128, sm, slots), 128, sm, st>>>(with(1), p.hp1, p.hn1, p.q1,
                                                                                &p.qlen[0], p.vis1, &p.cursors[2]);
    rec(3);
    rec(4);
    if (p.has_gi) k_reflect<C><<<persistent_grid(k_reflect<C>, 128, sm, px), 128, sm, st>>>(with(2));
    rec(5);
    rec(10);
    if (p.has_gi) k_setup2<C><<<grid_for(px, 128, 16), 128, sm, st>>>(with(4));
    rec(11);
    rec(6);
    if (p.has_gi)
        k_shadow<C><<<persistent_grid(k_shadow<C>, 128, sm, slots), 128, sm, st>>>(with(3), p.hp2, p.hn2, p.q2,
                                                                                    &p.qlen[2], p.vis2,
                                                                                    &p.cursors[3]);
    rec(7);
    rec(12);
    k_compose<C><<<grid_for(px, 128, 16), 128, sm, st>>>(with(4));
    rec(13);
}

int launch_shade(cudaStream_t st, const ShadeParams& p, cudaEvent_t* ev) {
    if (p.counts) launch_all<Counts>(st, p, ev);
    else launch_all<NoCount>(st, p, ev);
    return p.has_gi ? 7 : 4;
}

int launch_compose(cudaStream_t st, const ShadeParams& p) {
    const size_t sm = blob_smem(p.blob, 128);
    ShadeParams q = p;
    q.counts = nullptr;
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
    configure_one<Counts>(max_dyn_smem);
}

}  // namespace ifx
