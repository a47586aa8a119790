// Oracle (test infrastructure only): camera, per-pixel shading and film
// encoding, restated from the reference's main.rs (Cam, render_frame) and
// film.rs. Compiled with -ffp-contract=off; see ovec.h.
#include <algorithm>
#include <thread>

#include "oracle.h"

namespace orc {

void counters_flush();

// main.rs:198-210
Cam::Cam(V3 pos, V3 look, V3 up_hint, float fov, uint32_t w, uint32_t h) {
    origin = pos;
    fwd = normalize(look - pos);
    right = normalize(cross(fwd, up_hint));
    up = cross(right, fwd);
    const float rads_per_deg = PI_F / 180.0f;  // f32::to_radians
    tan_half = std::tan(fov * rads_per_deg * 0.5f);
    aspect = (float)w / (float)h;
}

// main.rs:213-217
V3 Cam::ray(uint32_t x, uint32_t y, uint32_t w, uint32_t h) const {
    float px = (2.0f * ((float)x + 0.5f) / (float)w - 1.0f) * aspect * tan_half;
    float py = (1.0f - 2.0f * ((float)y + 0.5f) / (float)h) * tan_half;
    return normalize(fwd + right * px + up * py);
}

static const V3 SKY(0.02f, 0.03f, 0.05f);

// reference.rs:31-46
Pcg::Pcg(uint64_t seed) : s(seed * 6364136223846793005ull + 1ull) {}
float Pcg::next_f32() {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    const uint64_t x = ((s >> 18) ^ s) >> 27;
    const uint32_t rot = (uint32_t)(s >> 59);
    const uint32_t v0 = (uint32_t)x;
    const uint32_t v = (v0 >> rot) | (v0 << ((32u - rot) & 31u));
    return (float)(v >> 8) * (1.0f / 16777216.0f);
}

// reference.rs:48-57
static V3 cosine_hemisphere(V3 n, Pcg& rng) {
    V3 t, b;
    frame(n, t, b);
    const float u1 = rng.next_f32();
    const float u2 = rng.next_f32();
    const float r = std::sqrt(u1);
    const float phi = TAU_F * u2;
    return normalize(t * (r * std::cos(phi)) + b * (r * std::sin(phi)) + n * std::sqrt(fmaxr(1.0f - u1, 0.0f)));
}

// reference.rs:61-137
V3 path(const Scene& sc, V3 ro, V3 rd, float tmax, uint32_t max_depth, Pcg& rng) {
    V3 radiance(0.0f, 0.0f, 0.0f), throughput(1.0f, 1.0f, 1.0f);
    V3 origin = ro, dir = rd;
    for (uint32_t depth = 0; depth < max_depth; ++depth) {
        Hit h;
        uint32_t steps;
        const bool hit = trace(sc, origin, dir, 1e-3f, tmax, h, steps);
        const float surf_t = hit ? h.t : 3.40282347e38f;
        float et;
        V3 e;
        if (emitter_hit(sc, origin, dir, fminr(surf_t, tmax), et, e, true)) {
            if (depth == 0) radiance += throughput * e;
            break;
        }
        if (!hit) break;
        const Material m = sc.material(h.mat);
        const V3 albedo = diffuse_albedo(m);
        radiance += throughput * m.emissive;
        for (const QuadLight& light : sc.lights) {
            const V3 e1 = light.verts[1] - light.verts[0];
            const V3 e2 = light.verts[3] - light.verts[0];
            const float r1 = rng.next_f32();
            const float r2 = rng.next_f32();
            const V3 lp = light.verts[0] + e1 * r1 + e2 * r2;
            const V3 to = lp - h.p;
            const float dist2 = length_squared(to);
            if (dist2 < 1e-9f) continue;
            const float dist = std::sqrt(dist2);
            const V3 l = to / dist;
            const float cos_s = dot(h.n, l);
            const float cos_l = dot(light.normal(), -l);
            if (cos_s <= 0.0f || cos_l <= 0.0f) continue;
            Hit occ;
            uint32_t s2;
            if (trace(sc, h.p + h.n * 1e-3f, l, 1e-3f, dist - 1e-2f, occ, s2)) continue;
            const float pdf = dist2 / (cos_l * light.area());
            radiance += throughput * albedo * light.emit * (cos_s / (PI_F * pdf));
        }
        throughput = throughput * albedo;
        dir = cosine_hemisphere(h.n, rng);
        origin = h.p + h.n * 1e-3f;
        if (depth >= 3) {
            const float q = clampf(max_element(throughput), 0.05f, 0.95f);
            if (rng.next_f32() > q) break;
            throughput = throughput / q;
        }
    }
    return radiance;
}

// One pixel of main.rs:247-361.
static V3 shade_pixel(const Scene& sc, const Cam& cam, int32_t mode, const Gi* gi, float tmax, uint32_t x,
                      uint32_t y, uint32_t w, uint32_t h, uint64_t& local, uint32_t spp) {
    V3 rd = cam.ray(x, y, w, h);
    if (mode == M_REFERENCE) {  // main.rs:249-259
        Pcg rng(((uint64_t)y << 32) | (uint64_t)x);
        V3 acc(0.0f, 0.0f, 0.0f);
        for (uint32_t i = 0; i < spp; ++i) acc += path(sc, cam.origin, rd, tmax, 12, rng);
        return acc / (float)spp;
    }
    Hit hh;
    uint32_t steps;
    bool hit = trace(sc, cam.origin, rd, 1e-3f, tmax, hh, steps);
    local += steps;
    float surf_t = hit ? hh.t : 3.40282347e38f;
    bool tonemapped = (mode == M_BEAUTY || mode == M_DIRECT || mode == M_INDIRECT || mode == M_REFERENCE);
    float et;
    V3 e;
    if (emitter_hit(sc, cam.origin, rd, fminr(surf_t, tmax), et, e)) return tonemapped ? e : V3::splat(0.9f);
    if (!hit) return SKY;
    switch (mode) {
        case M_NORMALS:
            return hh.n * 0.5f + V3::splat(0.5f);
        case M_DEPTH: {
            float d = 1.0f - clampf(hh.t / tmax, 0.0f, 1.0f);
            return V3::splat(d * d);
        }
        case M_STEPS: {
            float f = (float)steps / 128.0f;
            return V3(f, 1.0f - f, 0.2f);
        }
        default:
            break;
    }
    Material m = sc.material(hh.mat);
    V3 c(0.0f, 0.0f, 0.0f);
    if (mode != M_INDIRECT) {
        uint32_t s;
        V3 d = direct(sc, hh.p, hh.n, -rd, m, s);
        local += s;
        c += d + m.emissive;
    }
    if (gi) {
        V3 irr = gather(*gi->surfels, *gi->grid, hh.p, hh.n, gi->radius);
        c += diffuse_albedo(m) * irr;
        if (m.roughness < 0.45f || m.metallic > 0.05f) {
            V3 refl = rd - hh.n * (2.0f * dot(hh.n, rd));
            Hit rh;
            uint32_t s;
            bool rhit = trace(sc, hh.p + hh.n * 1e-3f, refl, 1e-3f, tmax, rh, s);
            local += s;
            float rt = rhit ? rh.t : 3.40282347e38f;
            V3 refl_col;
            float et2;
            V3 e2;
            if (emitter_hit(sc, hh.p, refl, fminr(rt, tmax), et2, e2)) {
                refl_col = e2;
            } else if (rhit) {
                Material m2 = sc.material(rh.mat);
                uint32_t s2;
                V3 d2 = direct(sc, rh.p, rh.n, -refl, m2, s2);
                local += s2;
                V3 i2 = gather(*gi->surfels, *gi->grid, rh.p, rh.n, gi->radius);
                refl_col = d2 + diffuse_albedo(m2) * i2 + m2.emissive;
            } else {
                refl_col = SKY;
            }
            V3 f = fresnel_schlick(fmaxr(dot(hh.n, -rd), 0.0f), f0_of(m));
            float gloss = clampf(1.0f - m.roughness / 0.45f, 0.0f, 1.0f);
            gloss = gloss * gloss;
            c += f * refl_col * gloss;
        }
    }
    return c;
}

// main.rs:229-367
uint64_t render_frame(const Scene& sc, const Cam& cam, int32_t mode, const Gi* gi, float tmax, uint32_t w,
                      uint32_t h, std::vector<V3>& film, int threads, uint32_t y0, uint32_t y1, uint32_t spp) {
    film.assign((size_t)w * (size_t)h, V3());
    if (y1 <= y0) {
        y0 = 0;
        y1 = h;
    }
    uint32_t nrows = y1 - y0;
    std::vector<uint64_t> row_evals(nrows, 0);
    auto do_row = [&](uint32_t r) {
        uint32_t y = y0 + r;
        uint64_t local = 0;
        for (uint32_t x = 0; x < w; ++x)
            film[(size_t)y * w + x] = shade_pixel(sc, cam, mode, gi, tmax, x, y, w, h, local, spp);
        row_evals[r] = local;
    };
    if (threads <= 1) {
        for (uint32_t r = 0; r < nrows; ++r) do_row(r);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t) {
            pool.emplace_back([&, t]() {
                for (uint32_t r = (uint32_t)t; r < nrows; r += (uint32_t)threads) do_row(r);
                counters_flush();
            });
        }
        for (auto& th : pool) th.join();
    }
    uint64_t total = 0;
    for (uint64_t e : row_evals) total += e;
    return total;
}

// film.rs:8-17
V3 aces(V3 x) {
    const float A = 2.51f, B = 0.03f, C = 2.43f, D = 0.59f, E = 0.14f;
    V3 num = x * (x * A + V3::splat(B));
    V3 den = x * (x * C + V3::splat(D)) + V3::splat(E);
    return vclamp(num / den, V3::splat(0.0f), V3::splat(1.0f));
}

// film.rs:23-31
uint8_t srgb(float c) {
    c = clampf(c, 0.0f, 1.0f);
    float v = (c <= 0.0031308f) ? c * 12.92f : 1.055f * std::pow(c, 1.0f / 2.4f) - 0.055f;
    return as_u8(v * 255.0f + 0.5f);
}

// film.rs:51-61
void encode(const std::vector<V3>& film, float exposure, bool tonemap, std::vector<uint8_t>& out) {
    out.resize(film.size() * 3);
    for (size_t i = 0; i < film.size(); ++i) {
        V3 scaled = film[i] * exposure;
        V3 m = tonemap ? aces(scaled) : scaled;
        out[3 * i + 0] = srgb(m.x);
        out[3 * i + 1] = srgb(m.y);
        out[3 * i + 2] = srgb(m.z);
    }
}

}  // namespace orc
