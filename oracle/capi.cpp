// Oracle (test infrastructure only): a flat C interface over the oracle so
// the Python tests, the smoke check and the benchmark's CPU-baseline leg can
// drive it with ctypes. One context holds one scene and its pipeline state.
#include <chrono>
#include <cstring>
#include <string>

#include "oracle.h"

using namespace orc;

struct orc_ctx {
    Scene scene;
    bool has_scene = false;
    Surfels surfels;
    std::vector<Cluster> clusters;
    Transfer transfer;
    bool has_transfer = false;
    Grid grid;
    float gather_radius = 0.0f;
    bool has_grid = false;
    std::vector<V3> film;
    std::vector<uint8_t> srgb8;
    uint32_t fw = 0, fh = 0;
    int threads = 1;
    std::string err;
    SolveStats stats{0, 0.0f};
    uint32_t spp = 512;  // samples per pixel of the path-traced reference mode
    DiffModel* diff = nullptr;
    ~orc_ctx() { diff_free(diff); }
};

static void put3(float* dst, const std::vector<V3>& v) {
    for (size_t i = 0; i < v.size(); ++i) {
        dst[3 * i + 0] = v[i].x;
        dst[3 * i + 1] = v[i].y;
        dst[3 * i + 2] = v[i].z;
    }
}
static void get3(std::vector<V3>& v, const float* src, size_t n) {
    v.resize(n);
    for (size_t i = 0; i < n; ++i) v[i] = V3(src[3 * i], src[3 * i + 1], src[3 * i + 2]);
}

extern "C" {

orc_ctx* orc_create(void) { return new orc_ctx(); }
void orc_destroy(orc_ctx* c) { delete c; }
const char* orc_error(orc_ctx* c) { return c->err.c_str(); }
void orc_set_threads(orc_ctx* c, int n) { c->threads = n < 1 ? 1 : n; }
void orc_set_use_bvh(orc_ctx* c, int on) { c->scene.use_bvh = on != 0; }

int orc_parse(orc_ctx* c, const char* src) {
    c->has_scene = false;
    c->has_transfer = false;
    c->has_grid = false;
    if (!parse_scene(std::string(src), c->scene, c->err)) return 1;
    c->has_scene = true;
    return 0;
}

// out[0..9]: objects, planes, lights(quad), materials (excl. default), bvh
// nodes, width, height, surfels, bounces, sphere lights.
int orc_scene_info(orc_ctx* c, int64_t* out, float* bounds6, float* exposure) {
    if (!c->has_scene) return 1;
    const Scene& s = c->scene;
    out[0] = (int64_t)s.objects.size();
    out[1] = (int64_t)s.planes.size();
    out[2] = (int64_t)s.lights.size();
    out[3] = (int64_t)s.materials.size() - 1;
    out[4] = (int64_t)s.bvh.nodes.size();
    out[5] = s.cfg.width;
    out[6] = s.cfg.height;
    out[7] = (int64_t)s.cfg.surfels;
    out[8] = s.cfg.bounces;
    out[9] = (int64_t)s.sphere_lights.size();
    bounds6[0] = s.lo.x; bounds6[1] = s.lo.y; bounds6[2] = s.lo.z;
    bounds6[3] = s.hi.x; bounds6[4] = s.hi.y; bounds6[5] = s.hi.z;
    *exposure = s.cfg.exposure;
    return 0;
}

// BVH nodes as 9 words each: lo(3 f32), hi(3 f32), start, count, right (u32),
// and the object order.
int orc_bvh(orc_ctx* c, float* nodes9, uint32_t* order) {
    const Bvh& b = c->scene.bvh;
    for (size_t i = 0; i < b.nodes.size(); ++i) {
        const BvhNode& n = b.nodes[i];
        float* d = nodes9 + 9 * i;
        d[0] = n.lo.x; d[1] = n.lo.y; d[2] = n.lo.z;
        d[3] = n.hi.x; d[4] = n.hi.y; d[5] = n.hi.z;
        memcpy(&d[6], &n.start, 4);
        memcpy(&d[7], &n.count, 4);
        memcpy(&d[8], &n.right, 4);
    }
    for (size_t i = 0; i < b.order.size(); ++i) order[i] = b.order[i];
    return 0;
}

// Scene SDF at n points: distance and material.
int orc_dist_mat(orc_ctx* c, int64_t n, const float* p, float* d, uint32_t* mat) {
    for (int64_t i = 0; i < n; ++i) {
        DistHit h = c->scene.dist_mat(V3(p[3 * i], p[3 * i + 1], p[3 * i + 2]));
        d[i] = h.d;
        mat[i] = h.mat;
    }
    return 0;
}

int orc_normal(orc_ctx* c, int64_t n, const float* p, float* out) {
    for (int64_t i = 0; i < n; ++i) {
        V3 v = c->scene.normal(V3(p[3 * i], p[3 * i + 1], p[3 * i + 2]));
        out[3 * i] = v.x; out[3 * i + 1] = v.y; out[3 * i + 2] = v.z;
    }
    return 0;
}

// Individual ray operations, for the kernel-level parity tests.
int orc_soft_shadow(orc_ctx* c, int64_t n, const float* ro, const float* rd, const float* tmin, const float* tmax,
                    const float* k, float* vis, uint32_t* steps) {
    for (int64_t i = 0; i < n; ++i) {
        vis[i] = soft_shadow(c->scene, V3(ro[3 * i], ro[3 * i + 1], ro[3 * i + 2]),
                             V3(rd[3 * i], rd[3 * i + 1], rd[3 * i + 2]), tmin[i], tmax[i], k[i], steps[i]);
    }
    return 0;
}

int orc_trace(orc_ctx* c, int64_t n, const float* ro, const float* rd, float tmin, float tmax, float* t_out,
              float* n_out, uint32_t* mat, uint32_t* steps, uint8_t* hit) {
    for (int64_t i = 0; i < n; ++i) {
        Hit h;
        uint32_t s;
        bool ok = trace(c->scene, V3(ro[3 * i], ro[3 * i + 1], ro[3 * i + 2]),
                        V3(rd[3 * i], rd[3 * i + 1], rd[3 * i + 2]), tmin, tmax, h, s);
        hit[i] = ok ? 1 : 0;
        steps[i] = s;
        t_out[i] = ok ? h.t : 0.0f;
        n_out[3 * i] = ok ? h.n.x : 0.0f;
        n_out[3 * i + 1] = ok ? h.n.y : 0.0f;
        n_out[3 * i + 2] = ok ? h.n.z : 0.0f;
        mat[i] = ok ? h.mat : 0u;
    }
    return 0;
}

float orc_quad_form_factor(const float* l12) {
    V3 l[4];
    for (int i = 0; i < 4; ++i) l[i] = V3(l12[3 * i], l12[3 * i + 1], l12[3 * i + 2]);
    return quad_form_factor(l);
}

float orc_form_factor_at(const float* verts12, const float* p, const float* n) {
    V3 v[4], t, b, loc[4];
    for (int i = 0; i < 4; ++i) v[i] = V3(verts12[3 * i], verts12[3 * i + 1], verts12[3 * i + 2]);
    V3 pp(p[0], p[1], p[2]), nn(n[0], n[1], n[2]);
    frame(nn, t, b);
    to_local(v, pp, t, b, nn, loc);
    return quad_form_factor(loc);
}

uint8_t orc_srgb(float c) { return srgb(c); }
void orc_aces(const float* in3, float* out3) {
    V3 r = aces(V3(in3[0], in3[1], in3[2]));
    out3[0] = r.x; out3[1] = r.y; out3[2] = r.z;
}

int64_t orc_generate(orc_ctx* c, int64_t target) {
    if (!c->has_scene) return -1;
    generate(c->scene, (uint64_t)target, c->surfels);
    return (int64_t)c->surfels.size();
}

int orc_set_surfels(orc_ctx* c, int64_t n, const float* p, const float* nrm, const float* albedo,
                    const float* area) {
    c->surfels.resize(0);
    get3(c->surfels.p, p, (size_t)n);
    get3(c->surfels.n, nrm, (size_t)n);
    get3(c->surfels.albedo, albedo, (size_t)n);
    c->surfels.area.assign(area, area + n);
    c->surfels.direct.assign((size_t)n, V3());
    c->surfels.irr.assign((size_t)n, V3());
    c->surfels.rad.assign((size_t)n, V3());
    return 0;
}

int64_t orc_surfel_count(orc_ctx* c) { return (int64_t)c->surfels.size(); }

// Any pointer may be null.
int orc_get_surfels(orc_ctx* c, float* p, float* n, float* albedo, float* area, float* direct, float* irr,
                    float* rad) {
    const Surfels& s = c->surfels;
    if (p) put3(p, s.p);
    if (n) put3(n, s.n);
    if (albedo) put3(albedo, s.albedo);
    if (area) memcpy(area, s.area.data(), s.area.size() * 4);
    if (direct) put3(direct, s.direct);
    if (irr) put3(irr, s.irr);
    if (rad) put3(rad, s.rad);
    return 0;
}

int orc_set_surfel_state(orc_ctx* c, const float* direct, const float* irr, const float* rad) {
    size_t n = c->surfels.size();
    if (direct) get3(c->surfels.direct, direct, n);
    if (irr) get3(c->surfels.irr, irr, n);
    if (rad) get3(c->surfels.rad, rad, n);
    return 0;
}

int64_t orc_build_clusters(orc_ctx* c, int res) {
    if (res < 1) {
        c->err = "cluster resolution must be at least 1";
        return -1;
    }
    build_clusters(c->scene, c->surfels, res, c->clusters);
    return (int64_t)c->clusters.size();
}

// Clusters as p(3) n(3) area radius per cluster, plus member offsets and the
// flat member list (from the last transfer build if one exists).
int orc_get_clusters(orc_ctx* c, float* pnar8, uint32_t* offsets, uint32_t* members) {
    const std::vector<Cluster>& cl = c->has_transfer ? c->transfer.clusters : c->clusters;
    uint32_t off = 0;
    for (size_t i = 0; i < cl.size(); ++i) {
        float* d = pnar8 + 8 * i;
        d[0] = cl[i].p.x; d[1] = cl[i].p.y; d[2] = cl[i].p.z;
        d[3] = cl[i].n.x; d[4] = cl[i].n.y; d[5] = cl[i].n.z;
        d[6] = cl[i].area; d[7] = cl[i].radius;
        if (offsets) offsets[i] = off;
        if (members) memcpy(members + off, cl[i].members.data(), cl[i].members.size() * 4);
        off += (uint32_t)cl[i].members.size();
    }
    if (offsets) offsets[cl.size()] = off;
    return 0;
}

// Builds the transfer from the clusters of the last orc_build_clusters call.
// info[0..3]: nc, links, evals, interior rows; *mean_row_sum.
int orc_build_transfer_sampled(orc_ctx* c, int64_t stride, int64_t* info, float* mean_row_sum);

int orc_build_transfer(orc_ctx* c, int64_t* info, float* mean_row_sum) {
    return orc_build_transfer_sampled(c, 1, info, mean_row_sum);
}

// Rows i % stride == 0 only (stride 1: every row); the others stay empty.
int orc_build_transfer_sampled(orc_ctx* c, int64_t stride, int64_t* info, float* mean_row_sum) {
    uint64_t ev = build_transfer(c->scene, c->surfels, c->clusters, c->transfer, c->threads,
                                 (size_t)(stride < 1 ? 1 : stride));
    c->has_transfer = true;
    int64_t interior = 0;
    for (size_t i = 0; i + 1 < c->transfer.starts.size(); ++i)
        if (c->transfer.starts[i + 1] > c->transfer.starts[i]) interior++;
    info[0] = (int64_t)c->transfer.nc;
    info[1] = (int64_t)c->transfer.links;
    info[2] = (int64_t)ev;
    info[3] = interior;
    *mean_row_sum = c->transfer.mean_row_sum;
    return 0;
}

int orc_get_transfer(orc_ctx* c, uint32_t* starts, uint32_t* idx, float* w, float* row_sum, float* row_sky,
                     uint64_t* row_evals, uint32_t* cand_count) {
    const Transfer& t = c->transfer;
    if (starts) memcpy(starts, t.starts.data(), t.starts.size() * 4);
    if (idx) memcpy(idx, t.idx.data(), t.idx.size() * 4);
    if (w) memcpy(w, t.w.data(), t.w.size() * 4);
    if (row_sum) memcpy(row_sum, t.row_sum.data(), t.row_sum.size() * 4);
    if (row_sky) memcpy(row_sky, t.row_sky.data(), t.row_sky.size() * 4);
    if (row_evals) memcpy(row_evals, t.row_evals.data(), t.row_evals.size() * 8);
    if (cand_count) memcpy(cand_count, t.cand_count.data(), t.cand_count.size() * 4);
    return 0;
}

// Installs a transfer matrix (CSR) over the current clusters, e.g. the GPU's,
// so the solve can be checked in isolation.
int orc_set_transfer(orc_ctx* c, int64_t n, const uint32_t* starts, int64_t links, const uint32_t* idx,
                     const float* w) {
    c->transfer.clusters = c->clusters;
    c->transfer.nc = c->clusters.size();
    c->transfer.starts.assign(starts, starts + n + 1);
    c->transfer.idx.assign(idx, idx + links);
    c->transfer.w.assign(w, w + links);
    c->transfer.links = (size_t)links;
    c->has_transfer = true;
    return 0;
}

int64_t orc_light_surfels(orc_ctx* c) { return (int64_t)light_surfels(c->scene, c->surfels, c->threads); }

// Surfels i % stride == 0 only.
int64_t orc_light_surfels_sampled(orc_ctx* c, int64_t stride) {
    return (int64_t)light_surfels(c->scene, c->surfels, c->threads, (size_t)(stride < 1 ? 1 : stride));
}

int orc_solve_ex(orc_ctx* c, uint32_t max_bounces, int fixed, uint32_t* iterations, float* residual);

int orc_solve(orc_ctx* c, uint32_t max_bounces, uint32_t* iterations, float* residual) {
    return orc_solve_ex(c, max_bounces, 0, iterations, residual);
}

// fixed != 0: exactly max_bounces bounces, no residual exit.
int orc_solve_ex(orc_ctx* c, uint32_t max_bounces, int fixed, uint32_t* iterations, float* residual) {
    if (!c->has_transfer) {
        c->err = "no transfer";
        return 1;
    }
    c->stats = solve(c->surfels, c->transfer, max_bounces, c->threads, fixed != 0);
    *iterations = c->stats.iterations;
    *residual = c->stats.residual;
    return 0;
}

// Builds the gather grid exactly as main.rs:473-475 does.
int orc_build_grid(orc_ctx* c, float* radius_out, int32_t* dims_out) {
    float diag = c->scene.diag();
    float radius = (diag / std::sqrt((float)c->scene.cfg.surfels)) * 2.6f;
    c->grid.build(c->surfels.p, c->scene.lo, c->scene.hi, radius);
    c->gather_radius = radius;
    c->has_grid = true;
    if (radius_out) *radius_out = radius;
    if (dims_out) {
        dims_out[0] = c->grid.dim[0];
        dims_out[1] = c->grid.dim[1];
        dims_out[2] = c->grid.dim[2];
    }
    return 0;
}

int orc_get_grid(orc_ctx* c, uint32_t* starts, uint32_t* items) {
    if (starts) memcpy(starts, c->grid.starts.data(), c->grid.starts.size() * 4);
    if (items) memcpy(items, c->grid.items.data(), c->grid.items.size() * 4);
    return 0;
}

int orc_gather(orc_ctx* c, int64_t n, const float* p, const float* nrm, float* out) {
    for (int64_t i = 0; i < n; ++i) {
        V3 r = gather(c->surfels, c->grid, V3(p[3 * i], p[3 * i + 1], p[3 * i + 2]),
                      V3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]), c->gather_radius);
        out[3 * i] = r.x; out[3 * i + 1] = r.y; out[3 * i + 2] = r.z;
    }
    return 0;
}

// Camera basis as main.rs:198-210 computes it: origin, fwd, right, up (12
// floats), tan_half, aspect.
int orc_camera(const float* pos, const float* look, const float* up, float fov, uint32_t w, uint32_t h,
               float* out14) {
    Cam cam(V3(pos[0], pos[1], pos[2]), V3(look[0], look[1], look[2]), V3(up[0], up[1], up[2]), fov, w, h);
    V3 v[4] = {cam.origin, cam.fwd, cam.right, cam.up};
    for (int i = 0; i < 4; ++i) {
        out14[3 * i] = v[i].x; out14[3 * i + 1] = v[i].y; out14[3 * i + 2] = v[i].z;
    }
    out14[12] = cam.tan_half;
    out14[13] = cam.aspect;
    return 0;
}

// Renders the scene camera (or the given pose, if pos is non-null) into the
// context's film. Rows [y0, y1) only when y1 > y0. Returns SDF evaluations.
int64_t orc_render(orc_ctx* c, int mode, uint32_t w, uint32_t h, const float* pos, const float* look,
                   uint32_t y0, uint32_t y1) {
    const Scene& s = c->scene;
    V3 P = pos ? V3(pos[0], pos[1], pos[2]) : s.camera.pos;
    V3 L = look ? V3(look[0], look[1], look[2]) : s.camera.look;
    Cam cam(P, L, s.camera.up, s.camera.fov, w, h);
    float tmax = s.diag() * 4.0f;
    Gi gi{&c->surfels, &c->grid, c->gather_radius};
    bool needs_gi = (mode == M_BEAUTY || mode == M_INDIRECT);
    c->fw = w;
    c->fh = h;
    return (int64_t)render_frame(s, cam, mode, needs_gi && c->has_grid ? &gi : nullptr, tmax, w, h, c->film,
                                 c->threads, y0, y1, c->spp);
}

void orc_set_spp(orc_ctx* c, uint32_t spp) { c->spp = spp < 1 ? 1 : spp; }

int orc_get_film(orc_ctx* c, float* rgb) {
    put3(rgb, c->film);
    return 0;
}

int orc_encode(orc_ctx* c, float exposure, int tonemap, uint8_t* out) {
    encode(c->film, exposure, tonemap != 0, c->srgb8);
    memcpy(out, c->srgb8.data(), c->srgb8.size());
    return 0;
}

// Per-light emission, quad lights then sphere lights, nl x 3.
int orc_set_emission(orc_ctx* c, int64_t nl, const float* e) {
    Scene& s = c->scene;
    if (nl != (int64_t)(s.lights.size() + s.sphere_lights.size())) return 1;
    size_t k = 0;
    for (QuadLight& l : s.lights) { l.emit = V3(e[3 * k], e[3 * k + 1], e[3 * k + 2]); ++k; }
    for (SphereLight& l : s.sphere_lights) { l.emit = V3(e[3 * k], e[3 * k + 1], e[3 * k + 2]); ++k; }
    return 0;
}

int orc_get_emission(orc_ctx* c, float* e) {
    size_t k = 0;
    for (const QuadLight& l : c->scene.lights) { e[3 * k] = l.emit.x; e[3 * k + 1] = l.emit.y; e[3 * k + 2] = l.emit.z; ++k; }
    for (const SphereLight& l : c->scene.sphere_lights) {
        e[3 * k] = l.emit.x; e[3 * k + 1] = l.emit.y; e[3 * k + 2] = l.emit.z; ++k;
    }
    return 0;
}

// FP64 differentiable model (diff.cpp) of the scene camera at w x h over the
// current surfels, transfer and grid. dims: surfels, lights, pixels.
int orc_diff_build(orc_ctx* c, uint32_t w, uint32_t h, int64_t* dims) {
    if (!c->has_transfer || !c->has_grid) {
        c->err = "diff model needs a transfer and a grid";
        return 1;
    }
    const Scene& s = c->scene;
    Cam cam(s.camera.pos, s.camera.look, s.camera.up, s.camera.fov, w, h);
    diff_free(c->diff);
    c->diff = diff_build(s, c->surfels, c->transfer, c->grid, c->gather_radius, cam, s.diag() * 4.0f, w, h,
                         c->threads);
    diff_dims(*c->diff, &dims[0], &dims[1], &dims[2]);
    return 0;
}

double orc_diff_loss(orc_ctx* c, const double* rho, const double* e, int K, const double* target, double* image) {
    return diff_loss(*c->diff, rho, e, K, target, image);
}

double orc_diff_grad(orc_ctx* c, const double* rho, const double* e, int K, const double* target, double* g_rho,
                     double* g_e) {
    return diff_grad(*c->diff, rho, e, K, target, g_rho, g_e);
}

void orc_counters(int enable, int reset, uint64_t* out10) {
    if (reset) counters_reset();
    counters_enable(enable != 0);
    if (out10) {
        WorkCounters w = counters_read();
        out10[0] = w.node_visits;
        for (int i = 0; i < 8; ++i) out10[1 + i] = w.prim_evals[i];
        out10[9] = w.sdf_evals;
    }
}

}  // extern "C"
