// Oracle (test infrastructure only): an FP64 reference of the differentiable
// model the GPU adjoint implements, used to check its gradients.
//
// With geometry and visibility held fixed, the rendered image is an affine
// function of the per-light emissions e_l and of the irradiance after K
// bounces, and the bounces are linear in E = rho * sum_l e_l a_il:
//   E_i   = rho_i * sum_l e_l * a_il          shade.rs:133-164, a_il = ff * vis
//   B_0 = E;  irr_k = F (A B_{k-1});  B_k = E + rho * irr_k     solve.rs:60-102
//   image = sum_l D_l e_l + em + kd * G irr_K
//           + Fg * (sky | e_light | sum_l D2_l e_l + em2 + kd2 * G2 irr_K)
//                                                    main.rs:289-356
// with A the area-weighted cluster mean (solve.rs:61-73), F the transfer,
// G the normalised gather weights (surfel.rs:262-293), D the per-light
// direct coefficients (shade.rs:50-125 with the emission factored out) and
// Fg = fresnel * gloss^2 of a glossy pixel's mirror term. Every coefficient
// is the f32 value the forward pass computes, taken along the same code path;
// the model and its reverse-mode gradient are evaluated in f64.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "oracle.h"

namespace orc {

struct PixelLin {
    int kind = 0;                   // 0 sky, 1 emitter (light `light`), 2 surface
    int light = -1;
    std::vector<double> D;          // nl x 3
    double em[3] = {0, 0, 0}, kd[3] = {0, 0, 0};
    std::vector<uint32_t> g_idx;    // gathered surfels and normalised weights
    std::vector<double> g_w;
    bool mirror = false;
    double Fg[3] = {0, 0, 0};
    int mkind = 0, mlight = -1;     // mirror: 0 sky, 1 emitter, 2 surface
    std::vector<double> D2;
    double em2[3] = {0, 0, 0}, kd2[3] = {0, 0, 0};
    std::vector<uint32_t> g2_idx;
    std::vector<double> g2_w;
};

struct DiffModel {
    int nl = 0;
    size_t N = 0;
    std::vector<float> a;  // N x nl: ff * vis of surfel i and light l, 0 where skipped
    std::vector<PixelLin> px;
    std::vector<uint32_t> starts, idx;
    std::vector<double> w;
    std::vector<std::vector<uint32_t>> members;
    std::vector<double> carea, sarea;
};

static const V3 SKY_C(0.02f, 0.03f, 0.05f);

template <class F>
static void par_for(size_t n, int threads, F f) {
    if (threads <= 1 || n < 2) {
        for (size_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t]() {
            for (size_t b = (size_t)t * 16; b < n; b += (size_t)threads * 16)
                for (size_t i = b; i < std::min(n, b + 16); ++i) f(i);
        });
    for (auto& th : pool) th.join();
}

static int n_lights(const Scene& sc) { return (int)(sc.lights.size() + sc.sphere_lights.size()); }

// Form factor and visibility of each light at (p, n) as shade.rs:60-84 and
// :133-164 compute them; `on` is false where the light is skipped
// (back-facing, ff <= 1e-6 or vis <= 1e-4).
struct LightTerm {
    bool on = false;
    float ff = 0.0f, vis = 0.0f, radius = 0.0f;
    V3 rep;
};

static void light_terms(const Scene& sc, V3 p, V3 n, const V3* v, std::vector<LightTerm>& out) {
    out.assign((size_t)n_lights(sc), LightTerm());
    V3 tan, bit;
    frame(n, tan, bit);
    int li = 0;
    for (const QuadLight& light : sc.lights) {
        LightTerm& T = out[(size_t)li++];
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
        if (vis <= 1e-4f) continue;
        T = LightTerm{true, ff, vis, radius, lc};
        if (v) {  // shade.rs:95-103: the representative point of the specular lobe
            V3 r = (-*v) - n * (2.0f * dot(n, -*v));
            V3 plane_n = light.normal();
            float denom = dot(r, plane_n);
            if (std::fabs(denom) > 1e-6f) {
                float t = dot(light.verts[0] - p, plane_n) / denom;
                if (t > 0.0f) T.rep = closest_on_quad(light.verts, p + r * t);
            }
        }
    }
    for (const SphereLight& light : sc.sphere_lights) {
        LightTerm& T = out[(size_t)li++];
        V3 to_light = light.c - p;
        float ff = sphere_form_factor(p, n, light.c, light.r);
        if (ff <= 1e-6f) continue;
        float dist = length(to_light);
        float radius = fmaxr(light.r, 1e-4f);
        float k = clampf(dist / radius, 1.5f, 96.0f);
        float shadow_end = fmaxr(dist - radius * 1.25f, 0.05f);
        uint32_t s;
        float vis = soft_shadow(sc, p + n * 3e-3f, to_light / dist, 0.015f, shadow_end, k, s);
        if (vis <= 1e-4f) continue;
        T = LightTerm{true, ff, vis, radius, V3()};
        if (v) {
            V3 r = (-*v) - n * (2.0f * dot(n, -*v));
            V3 ctr = r * dot(to_light, r) - to_light;
            float cl = length(ctr);
            T.rep = p + to_light + ctr * clampf(radius / fmaxr(cl, 1e-9f), 0.0f, 1.0f);
        }
    }
}

// shade.rs:50-125 per light with the emission factored out.
static void direct_coeffs(const Scene& sc, V3 p, V3 n, V3 v, const Material& m, std::vector<double>& D) {
    std::vector<LightTerm> T;
    light_terms(sc, p, n, &v, T);
    D.assign(T.size() * 3, 0.0);
    float n_dot_v = fmaxr(dot(n, v), 1e-4f);
    float alpha = fmaxr(m.roughness * m.roughness, 1e-3f);
    V3 f0 = f0_of(m);
    V3 kd = diffuse_albedo(m);
    for (size_t l = 0; l < T.size(); ++l) {
        if (!T[l].on) continue;
        double* d = &D[l * 3];
        for (int c = 0; c < 3; ++c) d[c] = (double)kd[c] * (double)T[l].ff * (double)T[l].vis;
        // shade.rs:104-121
        V3 L = normalize(T[l].rep - p);
        float n_dot_l = dot(n, L);
        if (n_dot_l <= 0.0f) continue;
        float rep_dist = fmaxr(length(T[l].rep - p), 1e-4f);
        float wide = clampf(alpha + T[l].radius / (2.0f * rep_dist), alpha, 1.0f);
        float energy = (alpha / wide) * (alpha / wide);
        V3 h = normalize(L + v);
        float a2 = wide * wide;
        float nh = fmaxr(dot(n, h), 0.0f);
        float dd = nh * nh * (a2 - 1.0f) + 1.0f;
        float dg = a2 / fmaxr(PI_F * dd * dd, 1e-9f);
        float gv = n_dot_l * std::sqrt(n_dot_v * n_dot_v * (1.0f - a2) + a2);
        float gl = n_dot_v * std::sqrt(n_dot_l * n_dot_l * (1.0f - a2) + a2);
        float vis_s = 0.5f / fmaxr(gv + gl, 1e-9f);
        V3 f = fresnel_schlick(fmaxr(dot(L, h), 0.0f), f0);
        float s = dg * vis_s * energy * n_dot_l;
        for (int c = 0; c < 3; ++c) d[c] += (double)f[c] * (double)s * (double)T[l].vis;
    }
}

// surfel.rs:262-293 as normalised weights (empty when the weight sum is
// below the reference's 1e-6 cut).
static void gather_weights(const Surfels& s, const Grid& g, V3 p, V3 n, float radius, std::vector<uint32_t>& idx,
                           std::vector<double>& wt) {
    idx.clear();
    wt.clear();
    float r2 = radius * radius;
    int32_t c[3];
    g.cell_of(p, c);
    double wsum = 0.0;
    float wsum_f = 0.0f;
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
                    idx.push_back(i);
                    wt.push_back((double)w);
                    wsum += (double)w;
                    wsum_f += w;
                }
            }
    if (!(wsum_f > 1e-6f)) {
        idx.clear();
        wt.clear();
        return;
    }
    for (double& w : wt) w /= wsum;
}

DiffModel* diff_build(const Scene& sc, const Surfels& s, const Transfer& t, const Grid& grid, float radius,
                      const Cam& cam, float tmax, uint32_t w, uint32_t h, int threads) {
    DiffModel* M = new DiffModel();
    M->nl = n_lights(sc);
    M->N = s.size();
    const size_t nl = (size_t)M->nl;
    M->a.assign(M->N * nl, 0.0f);
    par_for(M->N, threads, [&](size_t i) {
        std::vector<LightTerm> T;
        light_terms(sc, s.p[i], s.n[i], nullptr, T);
        for (size_t l = 0; l < nl; ++l)
            if (T[l].on) M->a[i * nl + l] = T[l].ff * T[l].vis;
    });
    M->starts = t.starts;
    M->idx = t.idx;
    M->w.assign(t.w.begin(), t.w.end());
    for (const Cluster& c : t.clusters) {
        M->members.push_back(c.members);
        M->carea.push_back((double)fmaxr(c.area, 1e-12f));
    }
    M->sarea.assign(s.area.begin(), s.area.end());
    M->px.assign((size_t)w * h, PixelLin());
    par_for(h, threads, [&](size_t y) {
        for (uint32_t x = 0; x < w; ++x) {
            PixelLin& L = M->px[y * w + x];
            V3 rd = cam.ray(x, (uint32_t)y, w, h);
            Hit hh;
            uint32_t steps;
            bool hit = trace(sc, cam.origin, rd, 1e-3f, tmax, hh, steps);
            float surf_t = hit ? hh.t : 3.40282347e38f;
            int el = emitter_index(sc, cam.origin, rd, fminr(surf_t, tmax));
            if (el >= 0) {
                L.kind = 1;
                L.light = el;
                continue;
            }
            if (!hit) continue;
            L.kind = 2;
            Material m = sc.material(hh.mat);
            direct_coeffs(sc, hh.p, hh.n, -rd, m, L.D);
            V3 kd = diffuse_albedo(m);
            for (int c = 0; c < 3; ++c) {
                L.em[c] = m.emissive[c];
                L.kd[c] = kd[c];
            }
            gather_weights(s, grid, hh.p, hh.n, radius, L.g_idx, L.g_w);
            if (!(m.roughness < 0.45f || m.metallic > 0.05f)) continue;
            L.mirror = true;
            V3 refl = rd - hh.n * (2.0f * dot(hh.n, rd));
            Hit rh;
            uint32_t s2;
            bool rhit = trace(sc, hh.p + hh.n * 1e-3f, refl, 1e-3f, tmax, rh, s2);
            float rt = rhit ? rh.t : 3.40282347e38f;
            V3 f = fresnel_schlick(fmaxr(dot(hh.n, -rd), 0.0f), f0_of(m));
            float gloss = clampf(1.0f - m.roughness / 0.45f, 0.0f, 1.0f);
            gloss = gloss * gloss;
            for (int c = 0; c < 3; ++c) L.Fg[c] = (double)f[c] * (double)gloss;
            int e2 = emitter_index(sc, hh.p, refl, fminr(rt, tmax));
            if (e2 >= 0) {
                L.mkind = 1;
                L.mlight = e2;
            } else if (rhit) {
                L.mkind = 2;
                Material m2 = sc.material(rh.mat);
                direct_coeffs(sc, rh.p, rh.n, -refl, m2, L.D2);
                V3 kd2 = diffuse_albedo(m2);
                for (int c = 0; c < 3; ++c) {
                    L.em2[c] = m2.emissive[c];
                    L.kd2[c] = kd2[c];
                }
                gather_weights(s, grid, rh.p, rh.n, radius, L.g2_idx, L.g2_w);
            }
        }
    });
    return M;
}

void diff_free(DiffModel* m) { delete m; }

void diff_dims(const DiffModel& m, int64_t* n_surfels, int64_t* n_lights_out, int64_t* n_pixels) {
    *n_surfels = (int64_t)m.N;
    *n_lights_out = m.nl;
    *n_pixels = (int64_t)m.px.size();
}

// irr = F (A B)
static void apply_M(const DiffModel& M, const std::vector<double>& B, std::vector<double>& irr) {
    const size_t nc = M.members.size();
    std::vector<double> C(nc * 3, 0.0);
    for (size_t c = 0; c < nc; ++c) {
        for (uint32_t m : M.members[c])
            for (int k = 0; k < 3; ++k) C[c * 3 + k] += B[m * 3 + k] * M.sarea[m];
        for (int k = 0; k < 3; ++k) C[c * 3 + k] /= M.carea[c];
    }
    irr.assign(M.N * 3, 0.0);
    for (size_t i = 0; i < M.N; ++i)
        for (uint32_t q = M.starts[i]; q < M.starts[i + 1]; ++q)
            for (int k = 0; k < 3; ++k) irr[i * 3 + k] += C[M.idx[q] * 3 + k] * M.w[q];
}

// out = A^T (F^T t)
static void apply_MT(const DiffModel& M, const std::vector<double>& t, std::vector<double>& out) {
    const size_t nc = M.members.size();
    std::vector<double> y(nc * 3, 0.0);
    for (size_t i = 0; i < M.N; ++i)
        for (uint32_t q = M.starts[i]; q < M.starts[i + 1]; ++q)
            for (int k = 0; k < 3; ++k) y[M.idx[q] * 3 + k] += M.w[q] * t[i * 3 + k];
    out.assign(M.N * 3, 0.0);
    for (size_t c = 0; c < nc; ++c)
        for (uint32_t m : M.members[c])
            for (int k = 0; k < 3; ++k) out[m * 3 + k] = M.sarea[m] / M.carea[c] * y[c * 3 + k];
}

struct Forward {
    std::vector<double> S, image;
    std::vector<std::vector<double>> irr;  // irr_1 .. irr_K
};

static void forward(const DiffModel& M, const double* rho, const double* e, int K, Forward& F) {
    const size_t nl = (size_t)M.nl, N3 = M.N * 3;
    F.S.assign(N3, 0.0);
    for (size_t i = 0; i < M.N; ++i)
        for (size_t l = 0; l < nl; ++l)
            for (int k = 0; k < 3; ++k) F.S[i * 3 + k] += e[l * 3 + k] * (double)M.a[i * nl + l];
    std::vector<double> E(N3), B(N3), irr(N3, 0.0);
    for (size_t q = 0; q < N3; ++q) E[q] = rho[q] * F.S[q];
    B = E;
    F.irr.clear();
    for (int k = 1; k <= K; ++k) {
        apply_M(M, B, irr);
        for (size_t q = 0; q < N3; ++q) B[q] = E[q] + rho[q] * irr[q];
        F.irr.push_back(irr);
    }
    F.image.assign(M.px.size() * 3, 0.0);
    for (size_t p = 0; p < M.px.size(); ++p) {
        const PixelLin& L = M.px[p];
        double* o = &F.image[p * 3];
        if (L.kind == 0) {
            for (int c = 0; c < 3; ++c) o[c] = SKY_C[c];
            continue;
        }
        if (L.kind == 1) {
            for (int c = 0; c < 3; ++c) o[c] = e[(size_t)L.light * 3 + c];
            continue;
        }
        for (size_t l = 0; l < nl; ++l)
            for (int c = 0; c < 3; ++c) o[c] += L.D[l * 3 + c] * e[l * 3 + c];
        for (int c = 0; c < 3; ++c) o[c] += L.em[c];
        for (size_t j = 0; j < L.g_idx.size(); ++j)
            for (int c = 0; c < 3; ++c) o[c] += L.kd[c] * L.g_w[j] * irr[L.g_idx[j] * 3 + c];
        if (!L.mirror) continue;
        double rc[3] = {0, 0, 0};
        if (L.mkind == 0) {
            for (int c = 0; c < 3; ++c) rc[c] = SKY_C[c];
        } else if (L.mkind == 1) {
            for (int c = 0; c < 3; ++c) rc[c] = e[(size_t)L.mlight * 3 + c];
        } else {
            for (int c = 0; c < 3; ++c) {
                for (size_t l = 0; l < nl; ++l) rc[c] += L.D2[l * 3 + c] * e[l * 3 + c];
                rc[c] += L.em2[c];
            }
            for (size_t j = 0; j < L.g2_idx.size(); ++j)
                for (int c = 0; c < 3; ++c) rc[c] += L.kd2[c] * L.g2_w[j] * irr[L.g2_idx[j] * 3 + c];
        }
        for (int c = 0; c < 3; ++c) o[c] += L.Fg[c] * rc[c];
    }
}

double diff_loss(const DiffModel& M, const double* rho, const double* e, int K, const double* target,
                 double* image) {
    Forward F;
    forward(M, rho, e, K, F);
    double loss = 0.0;
    for (size_t q = 0; q < F.image.size(); ++q) {
        double d = F.image[q] - (target ? target[q] : 0.0);
        loss += d * d;
    }
    if (image) memcpy(image, F.image.data(), F.image.size() * sizeof(double));
    return loss;
}

double diff_grad(const DiffModel& M, const double* rho, const double* e, int K, const double* target,
                 double* g_rho, double* g_e) {
    const size_t nl = (size_t)M.nl, N3 = M.N * 3;
    Forward F;
    forward(M, rho, e, K, F);
    double loss = 0.0;
    std::vector<double> gi(F.image.size());
    for (size_t q = 0; q < F.image.size(); ++q) {
        double d = F.image[q] - (target ? target[q] : 0.0);
        loss += d * d;
        gi[q] = 2.0 * d;
    }
    // Pixels: emission terms directly, irradiance terms into h = dL/dirr_K.
    std::vector<double> ge(nl * 3, 0.0), h(N3, 0.0);
    for (size_t p = 0; p < M.px.size(); ++p) {
        const PixelLin& L = M.px[p];
        const double* g = &gi[p * 3];
        if (L.kind == 1) {
            for (int c = 0; c < 3; ++c) ge[(size_t)L.light * 3 + c] += g[c];
            continue;
        }
        if (L.kind != 2) continue;
        for (size_t l = 0; l < nl; ++l)
            for (int c = 0; c < 3; ++c) ge[l * 3 + c] += L.D[l * 3 + c] * g[c];
        for (size_t j = 0; j < L.g_idx.size(); ++j)
            for (int c = 0; c < 3; ++c) h[L.g_idx[j] * 3 + c] += L.g_w[j] * L.kd[c] * g[c];
        if (!L.mirror) continue;
        double gm[3];
        for (int c = 0; c < 3; ++c) gm[c] = L.Fg[c] * g[c];
        if (L.mkind == 1) {
            for (int c = 0; c < 3; ++c) ge[(size_t)L.mlight * 3 + c] += gm[c];
        } else if (L.mkind == 2) {
            for (size_t l = 0; l < nl; ++l)
                for (int c = 0; c < 3; ++c) ge[l * 3 + c] += L.D2[l * 3 + c] * gm[c];
            for (size_t j = 0; j < L.g2_idx.size(); ++j)
                for (int c = 0; c < 3; ++c) h[L.g2_idx[j] * 3 + c] += L.g2_w[j] * L.kd2[c] * gm[c];
        }
    }
    // Bounces in reverse: t_K = h; b_k = M^T t_k; Ebar += b_k; for k >= 2
    // rhobar += b_k * irr_{k-1} and t_{k-1} = rho * b_k.
    std::vector<double> Eb(N3, 0.0), rb(N3, 0.0), t = h, b;
    for (int k = K; k >= 1; --k) {
        apply_MT(M, t, b);
        for (size_t q = 0; q < N3; ++q) Eb[q] += b[q];
        if (k >= 2) {
            const std::vector<double>& irr = F.irr[(size_t)k - 2];
            for (size_t q = 0; q < N3; ++q) {
                rb[q] += b[q] * irr[q];
                t[q] = rho[q] * b[q];
            }
        }
    }
    // E = rho * S with S = sum_l e_l a_il.
    for (size_t i = 0; i < M.N; ++i)
        for (int c = 0; c < 3; ++c) {
            rb[i * 3 + c] += Eb[i * 3 + c] * F.S[i * 3 + c];
            for (size_t l = 0; l < nl; ++l)
                ge[l * 3 + c] += Eb[i * 3 + c] * rho[i * 3 + c] * (double)M.a[i * nl + l];
        }
    memcpy(g_rho, rb.data(), N3 * sizeof(double));
    memcpy(g_e, ge.data(), nl * 3 * sizeof(double));
    return loss;
}

}  // namespace orc
