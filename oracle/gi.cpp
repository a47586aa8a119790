// Oracle (test infrastructure only): ray operations, analytic lighting,
// surfels, clusters, the transfer matrix and the Jacobi solve, restated from
// the reference's trace.rs, ltc.rs, shade.rs, surfel.rs, formfactor.rs and
// solve.rs. Compiled with -ffp-contract=off; see ovec.h.
#include <algorithm>
#include <map>
#include <thread>
#include <tuple>

#include "oracle.h"

namespace orc {

void counters_flush();

// Static row partition over `threads` workers. Every row is computed by the
// same code regardless of the partition, so results do not depend on it.
template <class F>
static void parallel_rows(size_t n, int threads, F f) {
    if (threads <= 1 || n < 2) {
        for (size_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::vector<std::thread> pool;
    size_t nt = (size_t)threads;
    for (size_t t = 0; t < nt; ++t) {
        pool.emplace_back([&, t]() {
            // Interleaved blocks of 16 rows balance uneven per-row cost.
            for (size_t b = t * 16; b < n; b += nt * 16) {
                size_t e = std::min(n, b + 16);
                for (size_t i = b; i < e; ++i) f(i);
            }
            counters_flush();
        });
    }
    for (auto& th : pool) th.join();
}

// -------------------------------------------------------------- trace.rs --
static const uint32_t MAX_STEPS = 128;    // trace.rs:10
static const uint32_t SHADOW_STEPS = 96;  // trace.rs:11

// trace.rs:27-58
bool trace(const Scene& sc, V3 ro, V3 rd, float tmin, float tmax, Hit& hit, uint32_t& steps_out) {
    float t = tmin;
    uint32_t steps = 0;
    while (steps < MAX_STEPS) {
        V3 p = ro + rd * t;
        DistHit h = sc.dist_mat(p);
        steps += 1;
        float eps = 1e-4f * fmaxr(t, 1.0f);
        if (h.d < eps) {
            hit.t = t;
            hit.p = p;
            hit.n = sc.normal(p);
            hit.mat = h.mat;
            steps_out = steps + 4;
            return true;
        }
        t += h.d;
        if (t > tmax) break;
    }
    steps_out = steps;
    return false;
}

// trace.rs:84-124
float soft_shadow(const Scene& sc, V3 ro, V3 rd, float tmin, float tmax, float k, uint32_t& steps_out) {
    float res = 1.0f;
    float t = tmin;
    uint32_t steps = 0;
    float ph = 1e20f;
    while (steps < SHADOW_STEPS && t < tmax) {
        float h = sc.dist(ro + rd * t);
        steps += 1;
        if (h < 1e-4f) {
            steps_out = steps;
            return 0.0f;
        }
        float y, d;
        if (h < ph) {
            y = h * h / (2.0f * ph);
            d = std::sqrt(fmaxr(h * h - y * y, 0.0f));
        } else {
            y = 0.0f;
            d = h;
        }
        res = fminr(res, k * d / fmaxr(t - y, 1e-4f));
        if (res < 1e-3f) {
            steps_out = steps;
            return 0.0f;
        }
        ph = h;
        t += clampf(h, 0.006f, 0.12f);
    }
    steps_out = steps;
    return clampf(res, 0.0f, 1.0f);
}

// trace.rs:128-148
bool intersect_quad(const V3 verts[4], V3 ro, V3 rd, float& t_out) {
    V3 e1 = verts[1] - verts[0];
    V3 e2 = verts[3] - verts[0];
    V3 n = cross(e1, e2);
    float denom = dot(n, rd);
    if (std::fabs(denom) < 1e-9f) return false;
    float t = dot(verts[0] - ro, n) / denom;
    if (t < 1e-4f) return false;
    V3 p = ro + rd * t - verts[0];
    float u = dot(p, e1) / dot(e1, e1);
    float v = dot(p, e2) / dot(e2, e2);
    if (u >= 0.0f && u <= 1.0f && v >= 0.0f && v <= 1.0f) {
        t_out = t;
        return true;
    }
    return false;
}

// trace.rs:189-199 (identical to surfel.rs:44-54)
float radical_inverse(uint32_t i, uint32_t base) {
    float f = 1.0f, r = 0.0f;
    float inv = 1.0f / (float)base;
    while (i > 0) {
        f *= inv;
        r += f * (float)(i % base);
        i /= base;
    }
    return r;
}

// trace.rs:165-186
float hemisphere_closure(const Scene& sc, V3 p, V3 n, float tmax, uint32_t dirs, uint32_t& steps_out) {
    V3 t, b;
    frame(n, t, b);
    uint32_t open = 0, steps = 0;
    for (uint32_t k = 0; k < dirs; ++k) {
        float u1 = radical_inverse(k + 1, 2);
        float u2 = radical_inverse(k + 1, 3);
        float r = std::sqrt(u1);
        float phi = TAU_F * u2;
        V3 d = t * (r * std::cos(phi)) + b * (r * std::sin(phi)) + n * std::sqrt(fmaxr(1.0f - u1, 0.0f));
        Hit hit;
        uint32_t s;
        bool h = trace(sc, p + n * 1e-3f, normalize(d), 1e-3f, tmax, hit, s);
        steps += s;
        if (!h) open += 1;
    }
    steps_out = steps;
    return (float)open / (float)dirs;
}

// ---------------------------------------------------------------- ltc.rs --
static const float INV_2PI = 0.15915494f;  // ltc.rs:23

// ltc.rs:25-46
static int clip_to_horizon(const V3 l[4], V3 out[5]) {
    int n = 0;
    for (int i = 0; i < 4; ++i) {
        V3 a = l[i];
        V3 b = l[(i + 1) % 4];
        float da = a.z, db = b.z;
        if (da >= 0.0f) out[n++] = a;
        if ((da >= 0.0f) != (db >= 0.0f)) {
            float t = da / (da - db);
            out[n++] = a + (b - a) * t;
        }
        if (n >= 5) break;
    }
    return n;
}

// ltc.rs:54-83
float quad_form_factor(const V3 l[4]) {
    V3 clipped[5];
    int n = clip_to_horizon(l, clipped);
    if (n < 3) return 0.0f;
    for (int i = 0; i < n; ++i) {
        float len = length(clipped[i]);
        if (len > 1e-9f) clipped[i] = clipped[i] / len;
    }
    float sum = 0.0f;
    for (int i = 0; i < n; ++i) {
        V3 a = clipped[i];
        V3 b = clipped[(i + 1) % n];
        float cos_t = clampf(dot(a, b), -1.0f, 1.0f);
        float theta = std::acos(cos_t);
        V3 c = cross(a, b);
        float len = length(c);
        if (len > 1e-9f) sum += theta * (c.z / len);
    }
    return fmaxr(sum * INV_2PI, 0.0f);
}

// ltc.rs:88-96
void frame(V3 n, V3& t, V3& b) {
    float s = n.z >= 0.0f ? 1.0f : -1.0f;
    float a = -1.0f / (s + n.z);
    float bb = n.x * n.y * a;
    t = V3(1.0f + s * n.x * n.x * a, s * bb, -s * n.x);
    b = V3(bb, s + n.y * n.y * a, -n.y);
}

// ltc.rs:108-115
void to_local(const V3 verts[4], V3 p, V3 t, V3 b, V3 n, V3 out[4]) {
    for (int i = 0; i < 4; ++i) {
        V3 d = verts[3 - i] - p;
        out[i] = V3(dot(d, t), dot(d, b), dot(d, n));
    }
}

// ltc.rs:119-127
V3 closest_on_quad(const V3 verts[4], V3 q) {
    V3 o = verts[0];
    V3 e1 = verts[1] - o;
    V3 e2 = verts[3] - o;
    V3 d = q - o;
    float u = clampf(dot(d, e1) / dot(e1, e1), 0.0f, 1.0f);
    float v = clampf(dot(d, e2) / dot(e2, e2), 0.0f, 1.0f);
    return o + e1 * u + e2 * v;
}

// [ext] Form factor from a receiver (p, n) to a sphere of radius r at c:
// the cosine-weighted solid angle over pi, with the horizon-clipped closed
// form of Snyder (1996), as given by Lagarde & de Rousiers (2014, eq. 15-16).
float sphere_form_factor(V3 p, V3 n, V3 c, float r) {
    V3 d = c - p;
    float dist2 = dot(d, d);
    float r2 = r * r;
    if (dist2 <= r2) return 0.0f;
    float dist = std::sqrt(dist2);
    float cos_t = dot(n, d) / dist;
    float sin_s2 = r2 / dist2;
    if (cos_t * cos_t > sin_s2) return sin_s2 * fmaxr(cos_t, 0.0f);
    float x = std::sqrt(1.0f / sin_s2 - 1.0f);
    float sin_t = std::sqrt(fmaxr(1.0f - cos_t * cos_t, 0.0f));
    float y = clampf(-x * (cos_t / sin_t), -1.0f, 1.0f);
    float sty = sin_t * std::sqrt(1.0f - y * y);
    float ill = (cos_t * std::acos(y) - x * sty) * sin_s2 + std::atan(sty / x);
    return fmaxr(ill, 0.0f) * (1.0f / PI_F);
}

// -------------------------------------------------------------- shade.rs --
// shade.rs:10-14
V3 fresnel_schlick(float cos_theta, V3 f0) {
    float m = clampf(1.0f - cos_theta, 0.0f, 1.0f);
    float m2 = m * m;
    return f0 + (V3::splat(1.0f) - f0) * (m2 * m2 * m);
}
// shade.rs:18-22
static float d_ggx(float n_dot_h, float alpha) {
    float a2 = alpha * alpha;
    float d = n_dot_h * n_dot_h * (a2 - 1.0f) + 1.0f;
    return a2 / fmaxr(PI_F * d * d, 1e-9f);
}
// shade.rs:26-31
static float v_smith(float n_dot_v, float n_dot_l, float alpha) {
    float a2 = alpha * alpha;
    float gv = n_dot_l * std::sqrt(n_dot_v * n_dot_v * (1.0f - a2) + a2);
    float gl = n_dot_v * std::sqrt(n_dot_l * n_dot_l * (1.0f - a2) + a2);
    return 0.5f / fmaxr(gv + gl, 1e-9f);
}
V3 f0_of(const Material& m) { return lerp(V3::splat(0.04f), m.albedo, m.metallic); }
V3 diffuse_albedo(const Material& m) { return m.albedo * (1.0f - m.metallic); }

// Specular lobe shared by both light kinds: shade.rs:104-121.
static void add_specular(V3& out, V3 p, V3 n, V3 v, V3 rep, float radius, float alpha, float n_dot_v, V3 f0,
                         V3 radiance) {
    V3 l = normalize(rep - p);
    float n_dot_l = dot(n, l);
    if (n_dot_l <= 0.0f) return;
    float rep_dist = fmaxr(length(rep - p), 1e-4f);
    float wide = clampf(alpha + radius / (2.0f * rep_dist), alpha, 1.0f);
    float energy = (alpha / wide) * (alpha / wide);
    V3 h = normalize(l + v);
    float d = d_ggx(fmaxr(dot(n, h), 0.0f), wide);
    float vis_s = v_smith(n_dot_v, n_dot_l, wide);
    V3 f = fresnel_schlick(fmaxr(dot(l, h), 0.0f), f0);
    out += f * (d * vis_s * energy * n_dot_l) * radiance;
}

// shade.rs:50-125
V3 direct(const Scene& sc, V3 p, V3 n, V3 v, const Material& m, uint32_t& steps_out) {
    V3 out(0.0f, 0.0f, 0.0f);
    uint32_t steps = 0;
    V3 tan, bit;
    frame(n, tan, bit);
    float n_dot_v = fmaxr(dot(n, v), 1e-4f);
    float alpha = fmaxr(m.roughness * m.roughness, 1e-3f);
    V3 f0 = f0_of(m);
    V3 kd = diffuse_albedo(m);
    for (const QuadLight& light : sc.lights) {
        V3 lc = light.center();
        V3 to_light = lc - p;
        if (dot(light.normal(), -normalize(to_light)) <= 0.0f) continue;
        V3 local[4];
        to_local(light.verts, p, tan, bit, n, local);
        float ff = quad_form_factor(local);
        if (ff <= 1e-6f) continue;
        float dist = length(to_light);
        float radius = fmaxr(std::sqrt(light.area() / PI_F), 1e-4f);
        float k = clampf(dist / radius, 1.5f, 96.0f);
        V3 ldir = to_light / dist;
        float shadow_end = fmaxr(dist - radius * 1.25f, 0.05f);
        uint32_t s;
        float vis = soft_shadow(sc, p + n * 3e-3f, ldir, 0.015f, shadow_end, k, s);
        steps += s;
        if (vis <= 1e-4f) continue;
        V3 radiance = light.emit * vis;
        out += kd * radiance * ff;
        V3 r = (-v) - n * (2.0f * dot(n, -v));
        V3 plane_n = light.normal();
        float denom = dot(r, plane_n);
        V3 rep = lc;
        if (std::fabs(denom) > 1e-6f) {
            float t = dot(light.verts[0] - p, plane_n) / denom;
            if (t > 0.0f) rep = closest_on_quad(light.verts, p + r * t);
        }
        add_specular(out, p, n, v, rep, radius, alpha, n_dot_v, f0, radiance);
    }
    for (const SphereLight& light : sc.sphere_lights) {  // [ext]
        V3 to_light = light.c - p;
        float ff = sphere_form_factor(p, n, light.c, light.r);
        if (ff <= 1e-6f) continue;
        float dist = length(to_light);
        float radius = fmaxr(light.r, 1e-4f);
        float k = clampf(dist / radius, 1.5f, 96.0f);
        V3 ldir = to_light / dist;
        float shadow_end = fmaxr(dist - radius * 1.25f, 0.05f);
        uint32_t s;
        float vis = soft_shadow(sc, p + n * 3e-3f, ldir, 0.015f, shadow_end, k, s);
        steps += s;
        if (vis <= 1e-4f) continue;
        V3 radiance = light.emit * vis;
        out += kd * radiance * ff;
        // Representative point: the point of the sphere closest to the
        // mirror ray (Karis 2013).
        V3 r = (-v) - n * (2.0f * dot(n, -v));
        V3 ctr = r * dot(to_light, r) - to_light;
        float cl = length(ctr);
        V3 rep = p + to_light + ctr * clampf(radius / fmaxr(cl, 1e-9f), 0.0f, 1.0f);
        add_specular(out, p, n, v, rep, radius, alpha, n_dot_v, f0, radiance);
    }
    steps_out = steps;
    return out;
}

// shade.rs:133-164
V3 direct_diffuse(const Scene& sc, V3 p, V3 n, V3 albedo, uint32_t& steps_out) {
    V3 out(0.0f, 0.0f, 0.0f);
    uint32_t steps = 0;
    V3 tan, bit;
    frame(n, tan, bit);
    for (const QuadLight& light : sc.lights) {
        V3 lc = light.center();
        V3 to_light = lc - p;
        if (dot(light.normal(), -normalize(to_light)) <= 0.0f) continue;
        V3 local[4];
        to_local(light.verts, p, tan, bit, n, local);
        float ff = quad_form_factor(local);
        if (ff <= 1e-6f) continue;
        float dist = length(to_light);
        float radius = fmaxr(std::sqrt(light.area() / PI_F), 1e-4f);
        float k = clampf(dist / radius, 1.5f, 96.0f);
        float shadow_end = fmaxr(dist - radius * 1.25f, 0.05f);
        uint32_t s;
        float vis = soft_shadow(sc, p + n * 3e-3f, to_light / dist, 0.015f, shadow_end, k, s);
        steps += s;
        if (vis <= 1e-4f) continue;
        out += albedo * light.emit * (ff * vis);
    }
    for (const SphereLight& light : sc.sphere_lights) {  // [ext]
        V3 to_light = light.c - p;
        float ff = sphere_form_factor(p, n, light.c, light.r);
        if (ff <= 1e-6f) continue;
        float dist = length(to_light);
        float radius = fmaxr(light.r, 1e-4f);
        float k = clampf(dist / radius, 1.5f, 96.0f);
        float shadow_end = fmaxr(dist - radius * 1.25f, 0.05f);
        uint32_t s;
        float vis = soft_shadow(sc, p + n * 3e-3f, to_light / dist, 0.015f, shadow_end, k, s);
        steps += s;
        if (vis <= 1e-4f) continue;
        out += albedo * light.emit * (ff * vis);
    }
    steps_out = steps;
    return out;
}

// [ext] nearest entry point of a ray into a sphere, t >= 1e-4.
static bool intersect_sphere(V3 c, float r, V3 ro, V3 rd, float& t_out) {
    V3 oc = ro - c;
    float b = dot(oc, rd);
    float cc = dot(oc, oc) - r * r;
    float disc = b * b - cc;
    if (disc < 0.0f) return false;
    float sq = std::sqrt(disc);
    float t = -b - sq;
    if (t < 1e-4f) return false;
    t_out = t;
    return true;
}

// shade.rs:168-181
bool emitter_hit(const Scene& sc, V3 ro, V3 rd, float tmax, float& t_best, V3& emit, bool quads_only) {
    bool found = false;
    for (const QuadLight& l : sc.lights) {
        float t;
        if (intersect_quad(l.verts, ro, rd, t)) {
            if (t < tmax && dot(l.normal(), rd) < 0.0f && (!found || t < t_best)) {
                found = true;
                t_best = t;
                emit = l.emit;
            }
        }
    }
    if (quads_only) return found;
    for (const SphereLight& l : sc.sphere_lights) {  // [ext]
        float t;
        if (intersect_sphere(l.c, l.r, ro, rd, t)) {
            if (t < tmax && (!found || t < t_best)) {
                found = true;
                t_best = t;
                emit = l.emit;
            }
        }
    }
    return found;
}

int emitter_index(const Scene& sc, V3 ro, V3 rd, float tmax) {
    int best = -1, li = 0;
    float t_best = 0.0f;
    for (const QuadLight& l : sc.lights) {
        float t;
        if (intersect_quad(l.verts, ro, rd, t) && t < tmax && dot(l.normal(), rd) < 0.0f &&
            (best < 0 || t < t_best)) {
            best = li;
            t_best = t;
        }
        ++li;
    }
    for (const SphereLight& l : sc.sphere_lights) {
        float t;
        if (intersect_sphere(l.c, l.r, ro, rd, t) && t < tmax && (best < 0 || t < t_best)) {
            best = li;
            t_best = t;
        }
        ++li;
    }
    return best;
}

// ------------------------------------------------------------- surfel.rs --
void Surfels::resize(size_t k) {
    p.resize(k);
    n.resize(k);
    albedo.resize(k);
    direct.resize(k);
    irr.resize(k);
    rad.resize(k);
    area.resize(k);
}

float halton(uint32_t i, uint32_t base) { return radical_inverse(i, base); }  // surfel.rs:44-54

// surfel.rs:71-114
void Grid::build(const std::vector<V3>& pts, V3 lo_, V3 hi, float cell) {
    lo = lo_;
    inv_cell = 1.0f / cell;
    V3 ext = hi - lo;
    dim[0] = clampi(as_i32(std::ceil(ext.x * inv_cell)), 1, 512);
    dim[1] = clampi(as_i32(std::ceil(ext.y * inv_cell)), 1, 512);
    dim[2] = clampi(as_i32(std::ceil(ext.z * inv_cell)), 1, 512);
    size_t ncells = (size_t)dim[0] * (size_t)dim[1] * (size_t)dim[2];
    std::vector<uint32_t> counts(ncells + 1, 0);
    std::vector<size_t> cidx(pts.size());
    for (size_t i = 0; i < pts.size(); ++i) {
        int32_t c[3];
        cell_of(pts[i], c);
        cidx[i] = (size_t)c[0] + (size_t)dim[0] * ((size_t)c[1] + (size_t)dim[1] * (size_t)c[2]);
        counts[cidx[i] + 1] += 1;
    }
    for (size_t i = 0; i < ncells; ++i) counts[i + 1] += counts[i];
    starts = counts;
    std::vector<uint32_t> cursor = counts;
    items.assign(pts.size(), 0);
    for (size_t i = 0; i < pts.size(); ++i) {
        size_t c = cidx[i];
        items[cursor[c]] = (uint32_t)i;
        cursor[c] += 1;
    }
}

// surfel.rs:127-133
void Grid::cell_of(V3 p, int32_t c[3]) const {
    c[0] = clampi(as_i32((p.x - lo.x) * inv_cell), 0, dim[0] - 1);
    c[1] = clampi(as_i32((p.y - lo.y) * inv_cell), 0, dim[1] - 1);
    c[2] = clampi(as_i32((p.z - lo.z) * inv_cell), 0, dim[2] - 1);
}

// surfel.rs:147-255
void generate(const Scene& sc, uint64_t target, Surfels& out) {
    V3 lo = sc.lo, hi = sc.hi;
    float diag = length(hi - lo);
    float d_min = fmaxr(diag / std::sqrt((float)target), 1e-4f);
    float cell = d_min;
    std::vector<V3> pts;
    out.resize(0);
    float inv_cell = 1.0f / cell;
    int32_t dim[3] = {clampi(as_i32(std::ceil((hi.x - lo.x) * inv_cell)), 1, 512),
                      clampi(as_i32(std::ceil((hi.y - lo.y) * inv_cell)), 1, 512),
                      clampi(as_i32(std::ceil((hi.z - lo.z) * inv_cell)), 1, 512)};
    size_t ncells = (size_t)dim[0] * (size_t)dim[1] * (size_t)dim[2];
    std::vector<std::vector<uint32_t>> occ(ncells);
    auto cell_idx = [&](V3 p, int32_t c[3]) {
        c[0] = clampi(as_i32((p.x - lo.x) * inv_cell), 0, dim[0] - 1);
        c[1] = clampi(as_i32((p.y - lo.y) * inv_cell), 0, dim[1] - 1);
        c[2] = clampi(as_i32((p.z - lo.z) * inv_cell), 0, dim[2] - 1);
    };
    float eps = d_min * 0.02f;
    float d_min_sq = d_min * d_min;
    uint64_t seeds64 = (uint64_t)(uint32_t)target * 24ull;
    uint32_t seeds = (uint32_t)std::min<uint64_t>(std::min<uint64_t>(seeds64, 0xffffffffull), 6000000ull);
    for (uint32_t i = 0; i < seeds; ++i) {
        if (out.size() >= target) break;
        V3 s(halton(i + 1, 2), halton(i + 1, 3), halton(i + 1, 5));
        V3 p = lo + (hi - lo) * s;
        bool ok = false;
        for (int it = 0; it < 10; ++it) {
            float d = sc.dist(p);
            if (std::fabs(d) < eps) {
                ok = true;
                break;
            }
            if (!std::isfinite(d) || std::fabs(d) > diag) break;
            p -= sc.normal(p) * d;
        }
        if (!ok || std::fabs(sc.dist(p)) >= eps) continue;
        if (any_lt(p, lo) || any_gt(p, hi)) continue;
        int32_t c[3];
        cell_idx(p, c);
        bool too_close = false;
        for (int32_t z = std::max(c[2] - 1, 0); z <= std::min(c[2] + 1, dim[2] - 1) && !too_close; ++z)
            for (int32_t y = std::max(c[1] - 1, 0); y <= std::min(c[1] + 1, dim[1] - 1) && !too_close; ++y)
                for (int32_t x = std::max(c[0] - 1, 0); x <= std::min(c[0] + 1, dim[0] - 1) && !too_close; ++x) {
                    size_t ci = (size_t)x + (size_t)dim[0] * ((size_t)y + (size_t)dim[1] * (size_t)z);
                    for (uint32_t j : occ[ci]) {
                        if (length_squared(pts[j] - p) < d_min_sq) {
                            too_close = true;
                            break;
                        }
                    }
                }
        if (too_close) continue;
        DistHit hit = sc.dist_mat(p);
        Material m = sc.material(hit.mat);
        V3 n = sc.normal(p);
        size_t ci = (size_t)c[0] + (size_t)dim[0] * ((size_t)c[1] + (size_t)dim[1] * (size_t)c[2]);
        occ[ci].push_back((uint32_t)out.size());
        pts.push_back(p);
        out.p.push_back(p);
        out.n.push_back(n);
        out.albedo.push_back(diffuse_albedo(m));
        out.area.push_back(d_min * d_min / 0.65f);
        out.direct.push_back(V3());
        out.irr.push_back(V3());
        out.rad.push_back(V3());
    }
}

// surfel.rs:262-293
V3 gather(const Surfels& s, const Grid& g, V3 p, V3 n, float radius) {
    V3 acc(0.0f, 0.0f, 0.0f);
    float wsum = 0.0f;
    float r2 = radius * radius;
    int32_t c[3];
    g.cell_of(p, c);
    for (int32_t z = std::max(c[2] - 1, 0); z <= std::min(c[2] + 1, g.dim[2] - 1); ++z)
        for (int32_t y = std::max(c[1] - 1, 0); y <= std::min(c[1] + 1, g.dim[1] - 1); ++y)
            for (int32_t x = std::max(c[0] - 1, 0); x <= std::min(c[0] + 1, g.dim[0] - 1); ++x) {
                size_t ci = (size_t)x + (size_t)g.dim[0] * ((size_t)y + (size_t)g.dim[1] * (size_t)z);
                for (uint32_t k = g.starts[ci]; k < g.starts[ci + 1]; ++k) {
                    uint32_t i = g.items[k];
                    float d2 = length_squared(s.p[i] - p);
                    if (d2 > r2) continue;
                    float align = dot(s.n[i], n);
                    if (align <= 0.15f) continue;
                    float t = 1.0f - d2 / r2;
                    float w = t * t * align;
                    acc += s.irr[i] * w;
                    wsum += w;
                }
            }
    if (wsum > 1e-6f) return acc / wsum;
    return V3(0.0f, 0.0f, 0.0f);
}

// --------------------------------------------------------- formfactor.rs --
static const float MAX_CALIBRATION = 8.0f;  // formfactor.rs:28

// formfactor.rs:70-89
uint32_t normal_bucket(V3 n) {
    V3 a = vabs(n);
    if (a.x >= a.y && a.x >= a.z) return n.x >= 0.0f ? 0u : 1u;
    if (a.y >= a.z) return n.y >= 0.0f ? 2u : 3u;
    return n.z >= 0.0f ? 4u : 5u;
}

// formfactor.rs:91-147
void build_clusters(const Scene& sc, const Surfels& s, int32_t res, std::vector<Cluster>& out) {
    V3 lo = sc.lo, hi = sc.hi;
    V3 ext = hi - lo;
    V3 inv((float)res / fmaxr(ext.x, 1e-6f), (float)res / fmaxr(ext.y, 1e-6f), (float)res / fmaxr(ext.z, 1e-6f));
    std::map<std::tuple<int32_t, int32_t, int32_t, uint32_t>, std::vector<uint32_t>> map;
    for (size_t i = 0; i < s.size(); ++i) {
        V3 c = (s.p[i] - lo) * inv;
        auto key = std::make_tuple(clampi(as_i32(c.x), 0, res - 1), clampi(as_i32(c.y), 0, res - 1),
                                   clampi(as_i32(c.z), 0, res - 1), normal_bucket(s.n[i]));
        map[key].push_back((uint32_t)i);
    }
    out.clear();
    for (auto& kv : map) {  // std::map iterates in sorted key order
        const std::vector<uint32_t>& members = kv.second;
        V3 p(0.0f, 0.0f, 0.0f), n(0.0f, 0.0f, 0.0f);
        float area = 0.0f;
        for (uint32_t m : members) {
            p += s.p[m] * s.area[m];
            n += s.n[m] * s.area[m];
            area += s.area[m];
        }
        if (area <= 1e-12f) continue;
        n = length_squared(n) > 1e-12f ? normalize(n) : V3(0.0f, 1.0f, 0.0f);
        Cluster c;
        c.p = p / area;
        c.n = n;
        c.area = area;
        c.radius = std::sqrt(area / PI_F);
        c.members = members;
        out.push_back(c);
    }
}

// formfactor.rs:153-277
uint64_t build_transfer(const Scene& sc, const Surfels& s, std::vector<Cluster> clusters, Transfer& t,
                        int threads, size_t stride) {
    size_t nc = clusters.size();
    float diag = length(sc.hi - sc.lo);
    size_t N = s.size();
    std::vector<std::vector<uint32_t>> ridx(N);
    std::vector<std::vector<float>> rw(N);
    t.row_sum.assign(N, 0.0f);
    t.row_sky.assign(N, 0.0f);
    t.row_evals.assign(N, 0);
    t.cand_count.assign(N, 0);
    if (stride < 1) stride = 1;
    parallel_rows((N + stride - 1) / stride, threads, [&](size_t row) {
        size_t i = row * stride;
        V3 sp = s.p[i], sn = s.n[i];
        uint64_t evals = 0;
        float sum = 0.0f;
        uint32_t cands = 0;
        for (size_t ci = 0; ci < nc; ++ci) {
            const Cluster& c = clusters[ci];
            V3 d = c.p - sp;
            float r2 = length_squared(d);
            if (r2 < 1e-9f) continue;
            float r = std::sqrt(r2);
            V3 dir = d / r;
            float cos_i = dot(sn, dir);
            float cos_c = dot(c.n, -dir);
            if (cos_i <= 1e-3f || cos_c <= 1e-3f) continue;
            float ff = cos_i * cos_c * c.area / (PI_F * r2 + c.area);
            if (ff < 2e-5f) continue;
            cands += 1;
            float k = clampf(r / fmaxr(c.radius, 1e-4f), 1.5f, 32.0f);
            uint32_t e;
            float vis = soft_shadow(sc, sp + sn * (diag * 5e-4f), dir, diag * 1e-3f, r - c.radius * 0.75f, k, e);
            evals += e;
            if (vis <= 1e-3f) continue;
            float v = ff * vis;
            ridx[i].push_back((uint32_t)ci);
            rw[i].push_back(v);
            sum += v;
        }
        uint32_t e;
        float sky = hemisphere_closure(sc, sp, sn, diag * 2.0f, 16, e);
        evals += e;
        float target = clampf(1.0f - sky, 0.0f, 1.0f);
        if (sum > 1e-5f) {
            float scale = fminr(target / sum, MAX_CALIBRATION);
            for (float& v : rw[i]) v *= scale;
            sum *= scale;
        }
        t.row_sum[i] = fminr(sum, 1.0f);
        t.row_sky[i] = sky;
        t.row_evals[i] = evals;
        t.cand_count[i] = cands;
    });
    size_t links = 0, interior = 0;
    uint64_t evals = 0;
    for (size_t i = 0; i < N; ++i) {
        links += ridx[i].size();
        evals += t.row_evals[i];
        if (!ridx[i].empty()) interior += 1;
    }
    float mean = 0.0f;
    if (interior > 0) {
        float acc = -0.0f;
        for (size_t i = 0; i < N; ++i)
            if (!ridx[i].empty()) acc += t.row_sum[i];
        mean = acc / (float)interior;
    }
    t.starts.assign(1, 0u);
    t.idx.clear();
    t.w.clear();
    t.idx.reserve(links);
    t.w.reserve(links);
    for (size_t i = 0; i < N; ++i) {
        t.idx.insert(t.idx.end(), ridx[i].begin(), ridx[i].end());
        t.w.insert(t.w.end(), rw[i].begin(), rw[i].end());
        t.starts.push_back((uint32_t)t.idx.size());
    }
    t.clusters = std::move(clusters);
    t.mean_row_sum = mean;
    t.nc = nc;
    t.links = links;
    return evals;
}

// ------------------------------------------------------------- solve.rs ---
// solve.rs:27-39
uint64_t light_surfels(const Scene& sc, Surfels& s, int threads, size_t stride) {
    std::vector<uint64_t> ev(s.size(), 0);
    if (stride < 1) stride = 1;
    parallel_rows((s.size() + stride - 1) / stride, threads, [&](size_t row) {
        size_t i = row * stride;
        uint32_t e;
        V3 c = direct_diffuse(sc, s.p[i], s.n[i], s.albedo[i], e);
        s.direct[i] = c;
        s.rad[i] = c;
        s.irr[i] = V3(0.0f, 0.0f, 0.0f);
        ev[i] = e;
    });
    uint64_t total = 0;
    for (uint64_t e : ev) total += e;
    return total;
}

// solve.rs:47-108
SolveStats solve(Surfels& s, const Transfer& t, uint32_t max_bounces, int threads, bool no_exit) {
    size_t nc = t.nc;
    if (nc == 0) return SolveStats{0, 0.0f};
    std::vector<V3> cluster_rad(nc);
    float residual = 0.0f;
    uint32_t iterations = 0;
    std::vector<float> deltas(s.size());
    for (uint32_t it = 0; it < max_bounces; ++it) {
        for (size_t c = 0; c < nc; ++c) {
            V3 acc(0.0f, 0.0f, 0.0f);
            for (uint32_t m : t.clusters[c].members) acc += s.rad[m] * s.area[m];
            cluster_rad[c] = acc / fmaxr(t.clusters[c].area, 1e-12f);
        }
        parallel_rows(s.size(), threads, [&](size_t i) {
            V3 irr(0.0f, 0.0f, 0.0f);
            for (uint32_t k = t.starts[i]; k < t.starts[i + 1]; ++k) irr += cluster_rad[t.idx[k]] * t.w[k];
            V3 new_rad = s.direct[i] + s.albedo[i] * irr;
            float d = max_element(vabs(new_rad - s.rad[i]));
            s.irr[i] = irr;
            s.rad[i] = new_rad;
            deltas[i] = d;
        });
        residual = 0.0f;
        for (float d : deltas) residual = fmaxr(residual, d);
        iterations = it + 1;
        if (residual < 1e-4f && !no_exit) break;
    }
    return SolveStats{iterations, residual};
}

}  // namespace orc
