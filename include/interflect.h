/*
 * interflect-b200 C ABI: the stage API of Interflect's surfel-radiosity path
 * (scene -> surfels -> transfer -> solve -> shade), executed on one NVIDIA
 * B200 (sm_100a) by hand-written CUDA kernels.
 *
 * The reference crate (`interflect` 0.1.3, Rust) has no FFI: its stages are
 * crate-internal functions called from src/main.rs. Each entry point below
 * replaces one of those functions; the citation names the reference function
 * (file:line, relative to the crate root) whose behaviour it reproduces. A
 * Rust host binds these with an `extern "C"` block that mirrors this header.
 *
 * Conventions
 *  - Every function returns an int status: IFX_OK (0) or an IFX_ERR_* code.
 *    On error the context's message is available from ifx_last_error().
 *    No C++ exception crosses this boundary.
 *  - Vectors are packed f32 triples (x, y, z) in caller-owned host memory.
 *    Output pointers documented as nullable may be NULL to skip that copy.
 *  - Device state (scene, surfels, transfer matrix, grid, film) is owned by
 *    the context. A context drives one GPU from its own CUDA streams, idle
 *    when a call returns (ifx_surfels_upload has read the caller's arrays
 *    when it returns; its copies to the device stay queued ahead of every
 *    later call); it is not thread-safe, but separate contexts are
 *    independent.
 *  - There is no CPU fallback: without a usable CUDA device every
 *    device-side call fails with IFX_ERR_CUDA.
 *  - Results are deterministic: bit-identical across runs and launch
 *    configurations (no floating-point atomics; every float reduction runs
 *    in a fixed order).
 */
#ifndef INTERFLECT_H
#define INTERFLECT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IFX_OK 0
#define IFX_ERR_INVALID 1  /* bad argument or call order */
#define IFX_ERR_PARSE 2    /* malformed .rad scene (scene.rs:365-571 errors) */
#define IFX_ERR_CUDA 3     /* CUDA runtime failure or no device */
#define IFX_ERR_NOMEM 4    /* device or host allocation failed */
#define IFX_ERR_LIMIT 5    /* a size limit was exceeded */
#define IFX_ERR_TIMEOUT 6  /* a bounded device-side wait expired */

/* Render modes: main.rs:25-39 (the path-traced `reference` mode has its own
 * entry point, ifx_render_reference). */
#define IFX_MODE_BEAUTY 0
#define IFX_MODE_DIRECT 1
#define IFX_MODE_INDIRECT 2
#define IFX_MODE_NORMALS 3
#define IFX_MODE_DEPTH 4
#define IFX_MODE_STEPS 5

typedef struct ifx_scene ifx_scene; /* host-side parsed scene */
typedef struct ifx_ctx ifx_ctx;     /* one GPU, one stream */

/* scene.rs:78-84 RenderCfg */
typedef struct ifx_render_cfg {
    uint32_t width, height;
    uint64_t surfels;
    uint32_t bounces;
    float exposure;
} ifx_render_cfg;

/* scene.rs:59-64 Camera */
typedef struct ifx_camera {
    float pos[3], look[3], up[3];
    float fov; /* degrees */
} ifx_camera;

typedef struct ifx_scene_info {
    uint32_t objects;     /* bounded objects (BVH) */
    uint32_t planes;      /* unbounded objects */
    uint32_t lights;      /* quad lights */
    uint32_t sphere_lights;
    uint32_t materials;   /* excluding the implicit default material */
    uint32_t bvh_nodes;
    float bounds_lo[3], bounds_hi[3]; /* scene.rs:573-601 world_bounds */
    ifx_render_cfg cfg;
    ifx_camera camera;
} ifx_scene_info;

/* formfactor.rs:48-66 Transfer (scalars) plus the evaluation count that
 * formfactor::build returns. */
typedef struct ifx_transfer_info {
    uint64_t clusters;
    uint64_t links;
    uint64_t candidates;  /* pairs that reached the visibility trace */
    uint64_t evals;       /* SDF evaluations, reference counting rule */
    uint64_t interior_rows;
    float mean_row_sum;
} ifx_transfer_info;

/* solve.rs:102-105 SolveStats */
typedef struct ifx_solve_stats {
    uint32_t iterations;
    float residual;
} ifx_solve_stats;

/* Device timing and launch accounting of the most recent calls. */
typedef struct ifx_stats {
    uint64_t kernel_launches;  /* kernels this context has launched so far */
    float ms_transfer, ms_light, ms_solve, ms_grid, ms_shade; /* CUDA-event times of the last call of each stage */
    float ms_visibility, ms_closure; /* CUDA-event times of the last visibility and closure kernels */
    /* CUDA-event times of the last frame's shading kernels: camera rays,
     * shadow cones of the camera hits, mirror rays, shadow cones of the
     * mirror hits, and the rest (setup, mirror setup, compose + encode). */
    float ms_primary, ms_shadow, ms_reflect, ms_shadow2, ms_shade_other;
    /* CUDA-event times of the last differentiable forward and backward. */
    float ms_diff_forward, ms_diff_backward;
} ifx_stats;

/* Kernels, for work accounting (ifx_get_work). */
#define IFX_KERNEL_VISIBILITY 0
#define IFX_KERNEL_CLOSURE 1
#define IFX_KERNEL_LIGHT 2
#define IFX_KERNEL_PRIMARY 3
#define IFX_KERNEL_SHADOW 4
#define IFX_KERNEL_REFLECT 5
#define IFX_KERNEL_SHADOW2 6
#define IFX_KERNEL_SHADE_OTHER 7
#define IFX_KERNEL_PATH 8 /* the path tracer of ifx_render_reference */
#define IFX_NUM_KERNELS 9
#define IFX_WORK_COUNTERS 21

/* ------------------------------------------------------------- scene --- */

/* Parses a .rad scene and builds its BVH on the host.
 * Replaces scene::parse (src/scene.rs:365-571) and Bvh::build
 * (src/bvh.rs:53-91). On IFX_ERR_PARSE, `err` receives the diagnostic the
 * reference would print after "error: " (truncated to errlen). */
int ifx_scene_parse(const char* src, size_t len, ifx_scene** out, char* err, size_t errlen);
void ifx_scene_free(ifx_scene* scene);
int ifx_scene_get_info(const ifx_scene* scene, ifx_scene_info* out);
/* Applies CLI overrides and re-validates them, as main.rs:394-413 does with
 * RenderCfg::validate (src/scene.rs:106-148). The message goes to `err`. */
int ifx_scene_set_cfg(ifx_scene* scene, const ifx_render_cfg* cfg, char* err, size_t errlen);
/* --no-bvh: linear object scan instead of the BVH (scene.rs:202-206). */
int ifx_scene_set_use_bvh(ifx_scene* scene, int use_bvh);
/* The host-built BVH (bvh.rs:27-36 node fields): per node lo(3) hi(3) as
 * f32 then start, count, right as u32 (9 words), and the leaf object order
 * (one u32 per bounded object). Both pointers nullable. */
int ifx_scene_get_bvh(const ifx_scene* scene, uint32_t* nodes9, uint32_t* order);

/* ----------------------------------------------------------- context --- */

int ifx_ctx_create(int device, ifx_ctx** out);
void ifx_ctx_destroy(ifx_ctx* ctx);
const char* ifx_last_error(const ifx_ctx* ctx);
int ifx_get_stats(const ifx_ctx* ctx, ifx_stats* out);

/* Measurement support (no reference counterpart). While counting is on, the
 * tracing kernels run an instrumented instantiation (slower; never use it for
 * timing) that tallies their work per kernel: node tests, primitive
 * evaluations by kind, march steps, form factors, gather items.
 * ifx_get_work returns the tallies (IFX_WORK_COUNTERS u64) of one kernel and
 * their algorithmic FLOPs under the library's FLOP model; ifx_reset_work
 * clears them. */
int ifx_set_work_counting(ifx_ctx* ctx, int on);
int ifx_reset_work(ifx_ctx* ctx);
int ifx_get_work(ifx_ctx* ctx, int kernel, uint64_t* counts, double* flops);

/* CUDA events on the context's stream around caller-chosen work. */
int ifx_timer_start(ifx_ctx* ctx);
int ifx_timer_stop(ifx_ctx* ctx, float* ms);
/* Tuning: the largest geometry program (header, objects, primitives, BVH
 * nodes) the ray-marching kernels copy into shared memory per CTA; larger
 * scenes are read from global memory through L1. Never changes results.
 * Default 24 KiB, at most 128 KiB. No counterpart in the reference. */
int ifx_set_stage_limit(ifx_ctx* ctx, uint32_t max_bytes);
/* Failure detection: the poll budget of this context's bounded device-side
 * waits (the scene-staging wait of every ray-marching kernel). A wait that
 * runs out of polls sets a status bit, leaves its kernel without tracing
 * (after its own copy in flight has landed), and the call returns
 * IFX_ERR_TIMEOUT; the context stays usable. 0 polls makes every such wait give up at once; the default
 * is IFX_WAIT_LIMIT_DEFAULT. Lowering it is for tests of that error path.
 * No counterpart in the reference, whose stages cannot fail (it only
 * validates input, src/scene.rs:106-148). */
#define IFX_WAIT_LIMIT_DEFAULT (1u << 22)
/* Tuning: whether the next ifx_scene_upload builds the per-cell candidate
 * leaf lists that the cone-shadow marches of large BVHs (more than three
 * nodes, no cones) use in place of a full traversal, falling back to the
 * traversal of src/bvh.rs:100-150 whenever the two could differ. Never
 * changes results. Default on. No counterpart in the reference. */
int ifx_set_leaf_grid(ifx_ctx* ctx, int on);
int ifx_set_wait_limit(ifx_ctx* ctx, uint32_t polls);

/* Flattens the scene (SDF object program, BVH nodes, planes, lights,
 * materials) into device memory. Must precede every stage below. */
int ifx_scene_upload(ifx_ctx* ctx, const ifx_scene* scene);

/* ----------------------------------------------------------- surfels --- */

/* Replaces surfel::generate (src/surfel.rs:147-255): Halton seeds projected
 * onto the SDF and Poisson-thinned on the GPU, with the reference's
 * seed-order acceptance (the same surfels in the same order).
 * `placed` receives the surfel count. */
int ifx_surfels_generate(ifx_ctx* ctx, uint64_t target, uint64_t* placed);

/* Installs caller-provided surfels (src/surfel.rs:23-38 fields p, n, albedo,
 * area); direct/irr/rad start at zero. */
int ifx_surfels_upload(ifx_ctx* ctx, uint64_t n, const float* p, const float* nrm, const float* albedo,
                       const float* area);
int ifx_surfels_count(const ifx_ctx* ctx, uint64_t* n);
/* Copies surfel state out. Every pointer is nullable. */
int ifx_surfels_download(ifx_ctx* ctx, float* p, float* nrm, float* albedo, float* area, float* direct,
                         float* irr, float* rad);

/* ---------------------------------------------------------- transfer --- */

/* Replaces formfactor::build_clusters (src/formfactor.rs:91-147) followed by
 * formfactor::build (src/formfactor.rs:153-277): clusters, candidate pairs,
 * cone-traced visibility, hemisphere-closure calibration and the CSR matrix,
 * all on the GPU. */
int ifx_transfer_build(ifx_ctx* ctx, int cluster_res, ifx_transfer_info* out);
/* Replaces formfactor::build_clusters (src/formfactor.rs:91-147) alone:
 * clusters of the current surfels, without a transfer (for example before
 * ifx_transfer_upload installs one). `nc` receives the cluster count. */
int ifx_clusters_build(ifx_ctx* ctx, int cluster_res, uint64_t* nc);
/* CSR arrays: starts (n+1), idx (links), w (links). Nullable. */
int ifx_transfer_download(ifx_ctx* ctx, uint32_t* starts, uint32_t* idx, float* w);
/* Clusters: per cluster p(3) n(3) area radius; member offsets (nc+1) and the
 * member list (n). Nullable. */
int ifx_clusters_download(ifx_ctx* ctx, float* pnar8, uint32_t* offsets, uint32_t* members);
/* Per-row diagnostics: calibrated row sum (min 1), sky fraction, SDF
 * evaluations, candidate pairs. Nullable. */
int ifx_transfer_row_diag(ifx_ctx* ctx, float* row_sum, float* row_sky, uint64_t* row_evals,
                          uint32_t* cand_count);
/* Installs a caller-provided CSR matrix over the current clusters. */
int ifx_transfer_upload(ifx_ctx* ctx, const uint32_t* starts, uint64_t links, const uint32_t* idx,
                        const float* w);

/* ------------------------------------------------------------- solve --- */

/* Replaces solve::light_surfels (src/solve.rs:27-39): direct diffuse light
 * (E) on every surfel; sets direct = rad = E and irr = 0. */
int ifx_light_surfels(ifx_ctx* ctx, uint64_t* evals);

/* Replaces solve::solve (src/solve.rs:47-108): Jacobi bounces with
 * area-weighted cluster aggregation, until the residual drops below 1e-4 or
 * max_bounces is reached. */
int ifx_solve(ifx_ctx* ctx, uint32_t max_bounces, ifx_solve_stats* out);

/* Relighting: installs an emission vector E (host, n x 3) as the solve's
 * source, i.e. direct = rad = E and irr = 0, the state solve::light_surfels
 * leaves (solve.rs:30-36) with E given instead of computed. */
int ifx_surfels_set_emission(ifx_ctx* ctx, const float* E);

/* Batched relighting: R right-hand sides E (host, R x n x 3, one emission
 * vector per rhs) solved on the current transfer matrix as a CSR SpMM. Each
 * rhs runs solve::solve (solve.rs:47-108) with its own stop rule and is
 * bit-identical to ifx_surfels_set_emission(E_r) + ifx_solve. E may be
 * NULL to reuse the right-hand sides of the previous call (resident on the
 * device; same R and n). Outputs (all nullable): rad and irr as R x n x 3,
 * iterations and residual per rhs. */
int ifx_solve_batched(ifx_ctx* ctx, uint32_t R, const float* E, uint32_t max_bounces, float* rad_out,
                      float* irr_out, uint32_t* iterations, float* residual);
/* Times ifx_solve_batched's SpMM block shapes (2, 4, 8, 16 warps of rows
 * per block) on the current matrix with R right-hand sides of E and keeps
 * the fastest for later calls; the choice never changes results. `best`
 * receives the chosen warps per block (nullable). */
int ifx_autotune_batched(ifx_ctx* ctx, uint32_t R, const float* E, int* best);

/* Largest cluster count ifx_solve_noalloc accepts. */
#define IFX_NOALLOC_MAX_CLUSTERS 16384

/* The Jacobi solve without any allocation; it has no counterpart in the
 * reference. For callers that cannot let a library allocate GPU memory: a
 * host engine that reserves the device up front and serves memory only from
 * its own arena, a frame loop that must not stall on cudaMalloc's implicit
 * synchronisation, or a binding whose buffers belong to another runtime.
 * It runs the same bounce kernels as ifx_solve on device buffers the caller
 * owns and calls no cudaMalloc, cudaFree or allocating library routine. Its
 * scratch (a radiosity value per cluster and a control block) is one static
 * device array of IFX_NOALLOC_MAX_CLUSTERS * 16 + 256 bytes that every GPU
 * loading this library holds until the process exits; nc above
 * IFX_NOALLOC_MAX_CLUSTERS is rejected with IFX_ERR_LIMIT.
 *
 * All array arguments are DEVICE pointers on `device`, as float4 / uint2
 * records (16 / 8 bytes per element):
 *   p_area4          n   surfel position, w = area (read)
 *   direct4, albedo4 n   E and diffuse albedo (read)
 *   irr4, rad4       n   irradiance and radiosity; rad4 holds the initial B
 *                        (E after ifx_light_surfels) and both are written
 *   cluster_p_area4  nc  cluster position, w = area (read)
 *   cluster_ranges   nc  [begin, end) of each cluster in `members` (uint2)
 *   members, starts, idx, w   cluster members and the CSR matrix (read)
 * The float4 arrays must be 16-byte aligned, cluster_ranges 8-byte aligned
 * and members, starts, idx and w 4-byte aligned; a misaligned pointer is
 * refused with IFX_ERR_INVALID before anything is launched.
 * `stream` is a cudaStream_t (NULL: the default stream). The call returns
 * after the solve has finished on that stream. It makes `device` current
 * for its own work and makes the caller's previous current device current
 * again before it returns, on every path.
 *
 * The first call on a device looks up the scratch array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture. Every call shares the one array and it keeps
 * the last call's contents (the control block is cleared at the start of
 * each call): calls whose work overlaps on the GPU race, so serialise them.
 * Errors are reported as in the rest of this API, with the message written
 * to `err` (nullable). Follows solve.rs:47-108. */
int ifx_solve_noalloc(int device, void* stream, uint32_t n, uint32_t nc, const float* p_area4, const float* direct4,
                      const float* albedo4, float* irr4, float* rad4, const float* cluster_p_area4,
                      const uint32_t* cluster_ranges, const uint32_t* members, const uint32_t* starts,
                      const uint32_t* idx, const float* w, uint32_t max_bounces, ifx_solve_stats* out, char* err,
                      size_t errlen);

/* ------------------------------------------------------------- shade --- */

/* Replaces surfel::Grid::build (src/surfel.rs:71-114) with the gather radius
 * main.rs:473-475 uses. radius <= 0 selects diag/sqrt(cfg.surfels)*2.6. */
int ifx_grid_build(ifx_ctx* ctx, float radius);

/* Replaces render_frame (src/main.rs:229-367) followed by Film::encode
 * (src/film.rs:51-61). `cam` NULL uses the scene camera. out_linear
 * (w*h*3 f32, row-major) and out_srgb (w*h*3 u8) are nullable host buffers.
 * `evals` receives the SDF evaluation count (nullable). */
int ifx_render_frame(ifx_ctx* ctx, const ifx_camera* cam, int mode, uint32_t w, uint32_t h, float exposure,
                     float* out_linear, uint8_t* out_srgb, uint64_t* evals);

/* One whole frame on the current surfels (src/main.rs:433-534 after surfel
 * generation): for the beauty and indirect modes ifx_transfer_build
 * (cluster_res), ifx_light_surfels, ifx_solve(max_bounces) and
 * ifx_grid_build(0), then ifx_render_frame(cam, mode, ...), with results
 * identical to those calls made in that order. The shading passes that read
 * no GI data (primary hits, their shadow rays, mirror rays and theirs) run
 * on a second CUDA stream while the GI stages run, and the light stage, the
 * grid's sort and the transfer's hemisphere closure on a third beside the
 * transfer build; only the composition waits for the grid, and a large
 * film is copied out in row chunks while the rest is composed. Other modes
 * skip the GI stages, as main.rs does. */
typedef struct ifx_frame_info {
    ifx_transfer_info transfer; /* as ifx_transfer_build reports it */
    uint64_t light_evals;       /* ifx_light_surfels */
    ifx_solve_stats solve;      /* ifx_solve */
    uint64_t shade_evals;       /* ifx_render_frame's `evals` */
    float ms_frame;             /* device time of the whole call */
} ifx_frame_info;
int ifx_frame(ifx_ctx* ctx, int cluster_res, uint32_t max_bounces, const ifx_camera* cam, int mode, uint32_t w,
              uint32_t h, float exposure, float* out_linear, uint8_t* out_srgb, ifx_frame_info* out);

/* --------------------------------------------------- differentiation --- */
/* Gradients of an image loss with respect to per-surfel albedo and per-light
 * emission, geometry and visibility held fixed. None of this has a
 * counterpart in the reference, whose surfel albedo is always the material's
 * diffuse albedo (surfel.rs:244) and whose solve stops on its residual. */

/* Per-surfel albedo override: rho (host, n x 3) replaces every surfel's
 * albedo, the value solve::light_surfels and solve::solve read
 * (solve.rs:33, :80). The transfer and grid stay valid. */
int ifx_surfels_set_albedo(ifx_ctx* ctx, const float* rho);
/* Per-light emission (host, nl x 3; quad lights in scene order, then sphere
 * lights) of the uploaded scene. The transfer, surfels and grid stay valid. */
int ifx_lights_set_emission(ifx_ctx* ctx, uint32_t nl, const float* emit);
int ifx_lights_get_emission(ifx_ctx* ctx, uint32_t nl, float* emit);

typedef struct ifx_diff_info {
    uint64_t surfels, lights, pixels;
    uint64_t gather_entries; /* (pixel, surfel) pairs of the frame's gathers */
    uint64_t links;          /* entries of the transposed transfer */
    uint32_t bounces;        /* the fixed bounce count K */
    float ms_setup;
} ifx_diff_info;

/* Prepares the differentiable frame of camera `cam` (NULL: the scene's) at
 * w x h, beauty mode, with exactly `bounces` Jacobi bounces (no residual
 * exit). Needs an uploaded scene, surfels and a transfer. Traces the frame
 * once (light factors of every surfel, the frame's hits, form factors and
 * visibilities), builds the gather grid, the per-pixel emission
 * coefficients, and the transposed gather and transfer operators. Any later
 * call that rebuilds the transfer or grid, uploads a scene or surfels, or
 * renders a frame ends the prepared state. */
int ifx_diff_setup(ifx_ctx* ctx, const ifx_camera* cam, uint32_t w, uint32_t h, uint32_t bounces,
                   ifx_diff_info* out);
/* The prepared frame for albedo rho (n x 3) and emission emit (nl x 3), both
 * nullable (keep the current values): solve::light_surfels' result from the
 * stored light factors, `bounces` Jacobi bounces with their irradiance kept
 * for the adjoint, and the frame re-composed from the stored hits. The image
 * (w*h*3 linear f32, nullable) is bit-identical to ifx_render_frame's after
 * ifx_light_surfels, a fixed-bounce solve and ifx_grid_build with the same
 * albedo and emission. */
int ifx_diff_forward(ifx_ctx* ctx, const float* rho, const float* emit, float* image);
/* Reverse mode of the last ifx_diff_forward for dL/dimage (w*h*3):
 * dL/drho (n x 3) and dL/demit (nl x 3), both nullable. The adjoint runs the
 * bounces backwards on the GPU-built transposes, (I - diag(rho) F A)^T
 * truncated to the same K bounces, in a fixed summation order (bit-identical
 * across runs). */
int ifx_diff_backward(ifx_ctx* ctx, const float* grad_image, float* grad_rho, float* grad_emit);

/* ------------------------------------------------- packed multi-scene --- */
/* Many independent scenes solved and shaded in ONE persistent cooperative
 * kernel launch, replayed from a captured CUDA graph. No counterpart in the
 * reference (one scene per process). Each scene keeps its own context; the
 * packed frame re-lights its surfels from the stored light factors (the
 * result of solve::light_surfels for the context's current albedo and
 * emission), runs solve::solve with the scene's own stop rule and bounce
 * cap, refreshes the gather grid and re-composes every pixel from the hits,
 * form factors and visibilities of the prepared frame. Every scene is
 * bit-identical to ifx_light_surfels + ifx_solve + ifx_grid_build +
 * ifx_render_frame on its own context, whatever the packing or launch shape.
 * A context must stay alive and unused for other rendering while it belongs
 * to a packed frame: rebuilding its transfer or grid, rendering with it or
 * destroying it makes ifx_multiscene_run fail with IFX_ERR_INVALID.
 * ifx_surfels_set_albedo and ifx_lights_set_emission on a member context
 * are picked up by the next run. */
typedef struct ifx_multiscene ifx_multiscene;

int ifx_multiscene_create(int device, ifx_multiscene** out);
void ifx_multiscene_destroy(ifx_multiscene* ms);
const char* ifx_multiscene_last_error(const ifx_multiscene* ms);
/* Adds ctx (scene, surfels and transfer in place, same device) with its
 * frame: camera (NULL: the scene's), w x h, beauty mode, the scene's
 * exposure, at most max_bounces bounces. Traces the frame once on ctx.
 * `index` receives the scene's position. */
int ifx_multiscene_add(ifx_multiscene* ms, ifx_ctx* ctx, const ifx_camera* cam, uint32_t w, uint32_t h,
                       uint32_t max_bounces, int* index);
/* Packs the scenes, picks the launch shape (autotune != 0: times block
 * sizes and CTAs per SM on the packed scenes and keeps the fastest; the
 * choice never changes a bit) and captures the CUDA graph. grid and block
 * (nullable) receive the chosen shape. */
int ifx_multiscene_build(ifx_multiscene* ms, int autotune, int* grid, int* block);
/* Failure detection: the poll budget of each grid barrier of the packed
 * launch (default IFX_MULTISCENE_WAIT_DEFAULT), taking effect at the next
 * ifx_multiscene_build. A barrier that runs out makes ifx_multiscene_run
 * return IFX_ERR_TIMEOUT and leaves the packed frame usable; 0 makes every
 * barrier give up at once, for tests of that path. No counterpart in the
 * reference. */
#define IFX_MULTISCENE_WAIT_DEFAULT (1u << 24)
int ifx_multiscene_set_wait_limit(ifx_multiscene* ms, uint32_t polls);

/* One graph launch: every scene's frame. ms_out (nullable): CUDA-event time. */
int ifx_multiscene_run(ifx_multiscene* ms, float* ms_out);
/* Scene `index` of the last run: linear film (w*h*3 f32), encoded frame
 * (w*h*3 u8) and solve statistics; each nullable. */
int ifx_multiscene_download(ifx_multiscene* ms, int index, float* out_linear, uint8_t* out_srgb,
                            ifx_solve_stats* stats);

/* ----------------------------------------------------- reference mode --- */

/* Replaces render_frame in --mode reference (src/main.rs:249-259 with
 * src/reference.rs:24-137): the brute-force path tracer the reference ships
 * as ground truth, spp paths per pixel from a PCG32 stream seeded with
 * (y << 32) | x, next-event estimation against the quad lights, cosine
 * bounces, Russian roulette, at most 12 vertices. Tone-mapped film and
 * encode as render_frame; out_linear and out_srgb are nullable. The first
 * call on a context also tabulates the libm sine and cosine of the sampler's
 * 2^24 azimuths on the host (128 MiB on the device), so that every pixel
 * equals the CPU path's. Sphere lights (an extension) are not sampled, as in
 * the reference, whose path tracer only knows quad lights. */
int ifx_render_reference(ifx_ctx* ctx, const ifx_camera* cam, uint32_t w, uint32_t h, uint32_t spp, float exposure,
                         float* out_linear, uint8_t* out_srgb);

#ifdef __cplusplus
}
#endif

#endif /* INTERFLECT_H */
