// Per-pixel shading helpers shared by the wavefront kernels (k_shade.cu)
// and the packed multi-scene frame (k_multi.cu): film encode, camera rays,
// direct light from stored form factors and visibilities, and the final
// composition of a pixel (main.rs:289-358, film.rs:8-61).
#pragma once

#include "kcommon.cuh"

namespace ifx {

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
        const DQuadLight& L = sv.light(l);
        return LightGeom{V{L.center[0], L.center[1], L.center[2]} - p, L.center[3]};
    }
    const DSphereLight& S = sv.slight(l - sv.n_lights);
    return LightGeom{V{S.c[0], S.c[1], S.c[2]} - p, fmaxf(S.c[3], 1e-4f)};
}

// shade.rs:60-73: the back-face cull and the exact diffuse form factor of
// light l (sphere lights: the horizon-clipped sphere form factor); -1 when
// the light is culled.
template <class C>
__device__ __forceinline__ float light_ff(const SceneView& sv, int l, V p, V n, V tan, V bit, C& cnt) {
    if (l < sv.n_lights) {
        const DQuadLight& L = sv.light(l);
        V to_light = V{L.center[0], L.center[1], L.center[2]} - p;
        if (dot(V{L.normal[0], L.normal[1], L.normal[2]}, -nrm(to_light)) <= 0.0f) return -1.0f;
        return quad_light_ff(L, p, tan, bit, n, cnt);
    }
    const DSphereLight& S = sv.slight(l - sv.n_lights);
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
        const DQuadLight& L = sv.light(li);
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
        const DSphereLight& S = sv.slight(si);
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

// main.rs:289-358: pixel `pix`'s colour from the stored hits, form factors
// and visibilities, in the reference's order of operations, then film.rs
// encode. Sky and debug pixels were written when their hits were set up; an
// emitter pixel is rewritten from its light's current emission when the
// frame is re-composed.
template <class C>
__device__ __forceinline__ void compose_pixel(const SceneView& sv, const ShadeParams& P, const float* t8,
                                              const GatherView& g, uint32_t pix, C& cnt) {
    const int nl = P.nl;
    const float4 b = P.hn1[pix];
    const uint32_t flags = __float_as_uint(b.w);
    if (flags & kPixDone) {
        // Sky and debug pixels are final; an emitter pixel follows its
        // light's current emission when the frame is re-composed.
        if (P.recompose && (flags & kPixEmit)) write_pixel(P, t8, pix, light_emit(sv, (int)__float_as_uint(b.y)));
        return;
    }
    const V rd = camera_ray(P, pix);
    const V p = mk4(P.hp1[pix]), n = mk4(b);
    const DMaterial& m = sv.mat(flags & kPixMatMask);
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
            if (f2 & kPixEmit) {
                rc = light_emit(sv, (int)__float_as_uint(b2.x));
            } else if (f2 & kPixHit) {
                const V p2 = mk4(a2), n2 = mk4(b2);
                const DMaterial& m2 = sv.mat(f2 & kPixMatMask);
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

}  // namespace ifx
