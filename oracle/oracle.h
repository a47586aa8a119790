// Oracle (test infrastructure only): a CPU restatement of the reference's
// surfel-radiosity path, used by the tests, the smoke check and the CPU
// baseline leg of the benchmark to check the CUDA path. Nothing in the product
// links or calls it.
//
// Every function cites the reference file:line it restates (paths relative to
// the reference crate root). The restatement keeps the reference's loop order,
// constants, early exits and f32 operation order, so that on the same inputs
// it produces the same bits as the reference built with rustc on x86-64
// (SSE2, no FMA contraction) and glibc libm.
//
// Extensions marked [ext] are not in the reference; they exist only so the
// synthetic benchmark scenes can be expressed, and reduce to the reference
// behaviour when unused (rotation 0, smoothing 0, no sphere lights).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "ovec.h"

namespace orc {

// ---------------------------------------------------------------- sdf.rs ----
enum PrimType : int32_t {
    P_SPHERE = 0,
    P_ROUNDBOX = 1,
    P_PLANE = 2,
    P_CAPSULE = 3,
    P_TORUS = 4,
    P_CYLINDER = 5,
    P_CONE = 6,
};

// sdf.rs:10-48. Fields are shared across variants; unused ones stay zero.
struct Prim {
    int32_t type = P_SPHERE;
    V3 c, b, a, n;      // centre / half-size / end points / plane normal
    float r = 0.0f;     // radius, rounding, cone ra
    float r2 = 0.0f;    // cone rb, torus minor
    float h = 0.0f;     // plane height, torus major
    // [ext] rotation about +y applied to the box before evaluation (radians
    // as cos/sin pair); identity for every reference scene.
    float rot_c = 1.0f, rot_s = 0.0f;
    bool rotated = false;

    float dist(V3 p) const;                       // sdf.rs:52-125
    bool bounds(V3& lo, V3& hi) const;            // sdf.rs:128-148
};

// sdf.rs:156-172
struct Object {
    Prim prim;
    std::vector<Prim> subtract;
    uint32_t mat = 0;
    float blend = 0.0f;
    float smooth = 0.0f;  // [ext] smooth-subtraction radius; 0 = reference max(d,-s)
    float dist(V3 p) const;
};

// ---------------------------------------------------------------- scene.rs --
struct Material {  // scene.rs:12-28
    V3 albedo = V3::splat(0.8f);
    float roughness = 0.8f;
    float metallic = 0.0f;
    V3 emissive = V3(0.0f, 0.0f, 0.0f);
};

struct QuadLight {  // scene.rs:33-56
    V3 verts[4];
    V3 emit;
    V3 center() const;
    V3 normal() const;
    float area() const;
};

// [ext] spherical area light, emitting from its whole surface.
struct SphereLight {
    V3 c;
    float r = 0.0f;
    V3 emit;
};

struct Camera {  // scene.rs:59-75
    V3 pos = V3(0.0f, 2.0f, 6.0f);
    V3 look = V3(0.0f, 1.0f, 0.0f);
    V3 up = V3(0.0f, 1.0f, 0.0f);
    float fov = 40.0f;
};

struct RenderCfg {  // scene.rs:78-161
    uint32_t width = 800, height = 600;
    uint64_t surfels = 20000;
    uint32_t bounces = 12;
    float exposure = 1.0f;
    bool validate(std::string& err) const;
};

struct BvhNode {  // bvh.rs:27-36
    V3 lo, hi;
    uint32_t start = 0, count = 0, right = 0;
};

struct Bvh {  // bvh.rs:38-43
    std::vector<BvhNode> nodes;
    std::vector<uint32_t> order;
    bool empty = true;
    void build(const std::vector<Object>& objects);  // bvh.rs:53-91
};

struct DistHit {  // scene.rs:182-185
    float d;
    uint32_t mat;
};

struct Scene {  // scene.rs:163-178
    std::vector<Object> objects;
    std::vector<Object> planes;
    std::vector<Material> materials;
    std::vector<QuadLight> lights;
    std::vector<SphereLight> sphere_lights;  // [ext]
    Camera camera;
    RenderCfg cfg;
    Bvh bvh;
    bool use_bvh = true;
    V3 lo, hi;

    DistHit dist_mat(V3 p) const;  // scene.rs:191-208
    float dist(V3 p) const { return dist_mat(p).d; }
    V3 normal(V3 p) const;         // scene.rs:218-236
    Material material(uint32_t id) const;
    float diag() const { return length(hi - lo); }
};

// scene.rs:365-571. Returns false and fills `err` on malformed input.
bool parse_scene(const std::string& src, Scene& out, std::string& err);

// ---------------------------------------------------------------- trace.rs --
struct Hit {
    float t;
    V3 p, n;
    uint32_t mat;
};
// trace.rs:27-58; returns hit flag; steps always written.
bool trace(const Scene& sc, V3 ro, V3 rd, float tmin, float tmax, Hit& hit, uint32_t& steps);
// trace.rs:84-124
float soft_shadow(const Scene& sc, V3 ro, V3 rd, float tmin, float tmax, float k, uint32_t& steps);
// trace.rs:128-148
bool intersect_quad(const V3 verts[4], V3 ro, V3 rd, float& t);
// trace.rs:165-186
float hemisphere_closure(const Scene& sc, V3 p, V3 n, float tmax, uint32_t dirs, uint32_t& steps);
float radical_inverse(uint32_t i, uint32_t base);  // trace.rs:189-199

// ------------------------------------------------------------------ ltc.rs --
float quad_form_factor(const V3 l[4]);                                 // ltc.rs:54-83
void frame(V3 n, V3& t, V3& b);                                        // ltc.rs:88-96
void to_local(const V3 verts[4], V3 p, V3 t, V3 b, V3 n, V3 out[4]);   // ltc.rs:108-115
V3 closest_on_quad(const V3 verts[4], V3 q);                           // ltc.rs:119-127
float sphere_form_factor(V3 p, V3 n, V3 c, float r);                   // [ext]

// ---------------------------------------------------------------- shade.rs --
V3 fresnel_schlick(float cos_theta, V3 f0);  // shade.rs:10-14
V3 f0_of(const Material& m);                 // shade.rs:36-38
V3 diffuse_albedo(const Material& m);        // shade.rs:41-43
V3 direct(const Scene& sc, V3 p, V3 n, V3 v, const Material& m, uint32_t& steps);  // shade.rs:50-125
V3 direct_diffuse(const Scene& sc, V3 p, V3 n, V3 albedo, uint32_t& steps);      // shade.rs:133-164
// shade.rs:168-181; quads_only: the quad lights alone, as reference.rs passes
// &sc.lights (the sphere-light extension is not part of the path tracer).
bool emitter_hit(const Scene& sc, V3 ro, V3 rd, float tmax, float& t, V3& emit, bool quads_only = false);
// The same test returning the index of the light it picks (quad lights, then
// sphere lights), -1 when none.
int emitter_index(const Scene& sc, V3 ro, V3 rd, float tmax);

// --------------------------------------------------------------- surfel.rs --
struct Surfels {  // surfel.rs:23-38, stored as structure of arrays
    std::vector<V3> p, n, albedo, direct, irr, rad;
    std::vector<float> area;
    size_t size() const { return p.size(); }
    void resize(size_t k);
};

struct Grid {  // surfel.rs:61-140
    V3 lo;
    float inv_cell = 1.0f;
    int32_t dim[3] = {1, 1, 1};
    std::vector<uint32_t> starts, items;
    void build(const std::vector<V3>& pts, V3 lo, V3 hi, float cell);
    void cell_of(V3 p, int32_t c[3]) const;
};

float halton(uint32_t i, uint32_t base);                            // surfel.rs:44-54
void generate(const Scene& sc, uint64_t target, Surfels& out);     // surfel.rs:147-255
V3 gather(const Surfels& s, const Grid& g, V3 p, V3 n, float radius);  // surfel.rs:262-293

// ----------------------------------------------------------- formfactor.rs --
struct Cluster {  // formfactor.rs:32-39
    V3 p, n;
    float area, radius;
    std::vector<uint32_t> members;
};

struct Transfer {  // formfactor.rs:48-66
    std::vector<Cluster> clusters;
    float mean_row_sum = 0.0f;
    std::vector<uint32_t> starts, idx;
    std::vector<float> w;
    size_t nc = 0, links = 0;
    // Per-row diagnostics kept for parity tests (not in the reference struct).
    std::vector<float> row_sum;    // the row's calibrated sum, min(1)
    std::vector<float> row_sky;    // hemisphere_closure result
    std::vector<uint64_t> row_evals;
    std::vector<uint32_t> cand_count;  // pairs that reached the visibility trace
};

uint32_t normal_bucket(V3 n);                                                 // formfactor.rs:70-89
void build_clusters(const Scene& sc, const Surfels& s, int32_t res, std::vector<Cluster>& out);  // :91-147
// stride > 1 computes only rows i with i % stride == 0 (the others stay
// empty with zero evaluations): a bounded sample of the rows for timing the
// CPU path at sizes where every row would take too long.
uint64_t build_transfer(const Scene& sc, const Surfels& s, std::vector<Cluster> clusters, Transfer& t,
                        int threads, size_t stride = 1);                      // :153-277

// ---------------------------------------------------------------- solve.rs --
struct SolveStats {
    uint32_t iterations;
    float residual;
};
// stride as in build_transfer: only surfels i % stride == 0 are lit.
uint64_t light_surfels(const Scene& sc, Surfels& s, int threads, size_t stride = 1);  // solve.rs:27-39
// no_exit: run all max_bounces bounces (the residual test never stops the
// loop), the fixed-K form the gradient is defined on.
SolveStats solve(Surfels& s, const Transfer& t, uint32_t max_bounces, int threads,
                 bool no_exit = false);  // solve.rs:47-108

// ----------------------------------------------------------------- main.rs --
enum Mode : int32_t {
    M_BEAUTY = 0, M_DIRECT = 1, M_INDIRECT = 2, M_NORMALS = 3, M_DEPTH = 4, M_STEPS = 5, M_REFERENCE = 6
};

struct Cam {  // main.rs:188-218
    V3 origin, fwd, right, up;
    float tan_half, aspect;
    Cam(V3 pos, V3 look, V3 up_hint, float fov, uint32_t w, uint32_t h);
    V3 ray(uint32_t x, uint32_t y, uint32_t w, uint32_t h) const;
};

struct Gi {  // main.rs:222-226
    const Surfels* surfels;
    const Grid* grid;
    float radius;
};

// main.rs:229-367 (the path-traced reference mode is not part of this path).
// `rows` restricts shading to a subset [y0, y1) of rows when y1 > y0; the
// evaluation count of only those rows is returned.
// M_REFERENCE is the brute-force path tracer of reference.rs with `spp`
// samples per pixel (main.rs:249-259).
uint64_t render_frame(const Scene& sc, const Cam& cam, int32_t mode, const Gi* gi, float tmax,
                      uint32_t w, uint32_t h, std::vector<V3>& film, int threads,
                      uint32_t y0 = 0, uint32_t y1 = 0, uint32_t spp = 512);

// reference.rs:24-46 (PCG32) and :61-137 (one path).
struct Pcg {
    uint64_t s;
    explicit Pcg(uint64_t seed);
    float next_f32();
};
V3 path(const Scene& sc, V3 ro, V3 rd, float tmax, uint32_t max_depth, Pcg& rng);

// film.rs:8-61
V3 aces(V3 x);
uint8_t srgb(float c);
void encode(const std::vector<V3>& film, float exposure, bool tonemap, std::vector<uint8_t>& out);

// Instrumented work counters (integer, summed over threads) used to derive the
// algorithmic FLOP count of the tracing kernels. Disabled unless enabled.
struct WorkCounters {
    uint64_t node_visits;      // aabb_dist evaluations inside the BVH
    uint64_t prim_evals[8];    // per PrimType (index 7 = smooth subtractions)
    uint64_t sdf_evals;        // scene-level distance queries
};
void counters_enable(bool on);
void counters_reset();
WorkCounters counters_read();

// ------------------------------------------------------ differentiation --
// FP64 reference of the image as a function of per-surfel albedo rho (N x 3)
// and per-light emission e (nl x 3) with geometry and visibility held fixed,
// and its exact gradient (diff.cpp). Built from the current surfels
// (positions, normals, areas), transfer and grid, for the given camera.
struct DiffModel;
DiffModel* diff_build(const Scene& sc, const Surfels& s, const Transfer& t, const Grid& g, float radius,
                      const Cam& cam, float tmax, uint32_t w, uint32_t h, int threads);
void diff_free(DiffModel* m);
void diff_dims(const DiffModel& m, int64_t* n_surfels, int64_t* n_lights, int64_t* n_pixels);
// Image (P x 3, may be null) and L = sum (image - target)^2 (target may be
// null: zero) after exactly K bounces.
double diff_loss(const DiffModel& m, const double* rho, const double* e, int K, const double* target,
                 double* image);
// dL/drho (N x 3) and dL/de (nl x 3); returns L.
double diff_grad(const DiffModel& m, const double* rho, const double* e, int K, const double* target,
                 double* g_rho, double* g_e);

}  // namespace orc
