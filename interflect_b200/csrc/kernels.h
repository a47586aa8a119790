// Kernel entry points and their parameter blocks (host <-> device).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "layout.h"

namespace ifx {

struct GatherView;

// Program blob as handed to every tracing kernel. When `staged` is set the
// kernel copies its geometry prefix (header, objects, primitives, BVH nodes:
// the first stage_bytes bytes, all the ray marches read) into dynamic shared
// memory; lights, materials and the linear order are always read from global
// memory. Unstaged (large) scenes are read from global memory through L1.
struct BlobRef {
    const uint8_t* ptr;
    uint32_t bytes;
    uint32_t stage_bytes;
    int staged;
    int stack_depth;  // BVH traversal stack entries per thread (tree depth + 2)
    uint32_t wait_polls;  // poll budget of the staging wait (kDefaultWaitPolls unless the host lowers it)
    int tree3;            // BVH in use and made of a root and two leaves: the NoCount3 kernels apply
    LeafGrid lg;          // enabled only for the scenes dist_fast serves (large BVHs)
};

// Default poll budget of every bounded device-side wait (the scene-staging
// mbarrier and the fused solve's grid barrier); the host may lower it per
// context (ifx_set_wait_limit) so that a test can make a wait run out.
static constexpr uint32_t kDefaultWaitPolls = 1u << 22;  // IFX_WAIT_LIMIT_DEFAULT

struct CamParams {
    float origin[3], fwd[3], right[3], up[3];
    float tan_half, aspect;
};

struct GridParams {
    const float4* gp;
    const float4* gn;
    const float4* girr;
    const uint32_t* starts;
    int dim[3];
    float lo[3];
    float inv_cell;
    float radius;
};

// Surfel state, structure of arrays, 16 bytes per field per surfel.
struct SurfelArrays {
    float4* p;       // xyz, w = area
    float4* n;       // xyz
    float4* albedo;  // xyz
    float4* direct;
    float4* irr;
    float4* rad;
};

// ---- generation (surfel.rs:147-255) ----
void launch_gen_project(cudaStream_t st, BlobRef blob, SceneConsts sc, uint32_t seed0, uint32_t count, float eps,
                        float4* out, uint32_t* status);
void launch_gen_finalize(cudaStream_t st, BlobRef blob, const float4* pts, uint32_t n, float area, SurfelArrays s,
                         uint32_t* status);

// Poisson-disc thinning of the projected seeds (surfel.rs:206-227) on the
// GPU, in batches of consecutive seeds; see k_surfels.cu.
struct GenGrid {
    float lo[3];
    float inv_cell;
    int dim[3];
    float d_min_sq;
    uint32_t* head;       // per occupancy cell: 1 + last point of the current batch inserted, 0 = empty
    uint32_t* next;       // per point: 1 + previous point of its cell, 0 = end
    uint32_t* head_acc;   // the same lists over the accepted points of all earlier batches
    uint32_t* next_acc;
    float4* pts;          // points kept after the batch filter, in seed order
    uint32_t* state;      // per point: 0 undecided, 1 accepted, 2 rejected
    uint32_t cap;         // capacity of pts / next / state
    uint32_t* err;        // device status word (bounded list walks)
};
static constexpr uint32_t kStatusGenWalk = 1u << 5;
// keep[j] = seed j of the batch projected onto the surface and no accepted
// point of an earlier batch lies within d_min of it.
int launch_gen_filter(cudaStream_t st, const GenGrid& g, const float4* cand, uint32_t cnt, uint32_t* keep);
// Appends the kept seeds at base + off[j] (undecided) and links them into
// their cells.
int launch_gen_append(cudaStream_t st, const GenGrid& g, const float4* cand, const uint32_t* keep,
                      const uint32_t* off, uint32_t cnt, uint32_t base);
// One round of deciding the batch's points [base, base + count) in seed
// order; *undecided counts those still open.
int launch_gen_resolve(cudaStream_t st, const GenGrid& g, uint32_t base, uint32_t count, uint32_t* undecided);
int launch_gen_accept_flags(cudaStream_t st, const GenGrid& g, uint32_t base, uint32_t count, uint32_t* flags);
// out[before + rank] = accepted point, for ranks below quota.
// After a batch: its accepted points join the accepted lists, and its cells
// of the batch lists are emptied for the next batch.
int launch_gen_retire(cudaStream_t st, const GenGrid& g, uint32_t base, uint32_t count);
int launch_gen_emit(cudaStream_t st, const GenGrid& g, uint32_t base, uint32_t count, const uint32_t* rank,
                    uint32_t quota, float4* out);

// ---- clusters (formfactor.rs:91-147) ----
void launch_cluster_keys(cudaStream_t st, const float4* p, const float4* n, uint32_t count, SceneConsts sc,
                         int res, unsigned long long* keys);
void launch_seg_heads(cudaStream_t st, const unsigned long long* sorted, uint32_t count, uint32_t* heads);
void launch_seg_starts(cudaStream_t st, const unsigned long long* sorted, const uint32_t* head_scan,
                       uint32_t count, uint32_t* seg_start, uint32_t* members);
void launch_cluster_reduce(cudaStream_t st, const uint32_t* seg_start, const uint32_t* members, uint32_t nseg,
                           const float4* sp, const float4* sn, float4* cp, float4* cn, uint32_t* valid);
void launch_cluster_compact(cudaStream_t st, const uint32_t* valid, const uint32_t* valid_scan, uint32_t nseg,
                            const uint32_t* seg_start, const float4* cp_in, const float4* cn_in, float4* cp,
                            float4* cn, uint2* crange);

// ---- transfer (formfactor.rs:153-277) ----
void launch_pair_count(cudaStream_t st, const float4* sp, const float4* sn, uint32_t n, const float4* cp,
                       const float4* cn, uint32_t nc, unsigned long long* cand_count);
void launch_pair_fill(cudaStream_t st, const float4* sp, const float4* sn, uint32_t n, const float4* cp,
                      const float4* cn, uint32_t nc, const unsigned long long* cand_off, uint32_t* cand_c,
                      float* cand_ff, uint32_t* cand_row);
// `order` (nullable): the permutation of candidates the queue walks.
void launch_visibility(cudaStream_t st, BlobRef blob, SceneConsts sc, const float4* sp, const float4* sn,
                       const float4* cp, const float4* cn, const uint32_t* cand_c, const uint32_t* cand_row,
                       const uint32_t* order, unsigned long long ncand, float* cand_vis, uint8_t* cand_steps,
                       uint32_t* status, unsigned long long* counts, unsigned long long* cursor);
// Keys (target cluster * (nc + 1) + source cluster) and candidate indices
// for the stable sort that gives launch_visibility its order.
int launch_vis_keys(cudaStream_t st, unsigned long long ncand, const uint32_t* cand_c, const uint32_t* cand_row,
                    const uint32_t* cid, uint32_t nc, unsigned long long* keys, uint32_t* vals);
// clo: per (row, ray) slot (open << 8) | steps, n * 16 entries.
void launch_closure(cudaStream_t st, BlobRef blob, SceneConsts sc, const float4* sp, const float4* sn,
                    uint32_t n, const uint32_t* order, uint16_t* clo, uint32_t* status, unsigned long long* counts,
                    unsigned long long* cursor);
// Keys ((row's cluster) * 16 + direction) and item indices for the stable
// sort that gives launch_closure its order.
int launch_clo_keys(cudaStream_t st, uint32_t n, const uint32_t* cid, uint32_t nc, uint32_t* keys, uint32_t* vals);
void launch_row_finalize(cudaStream_t st, uint32_t n, const unsigned long long* cand_off, const float* cand_ff,
                         const float* cand_vis, const uint8_t* cand_steps, const uint16_t* clo, uint32_t* row_links,
                         float* row_scale, float* row_sum, float* row_sky, unsigned long long* row_evals);
void launch_row_fill(cudaStream_t st, uint32_t n, const unsigned long long* cand_off, const uint32_t* cand_c,
                     const float* cand_ff, const float* cand_vis, const float* row_scale, const uint32_t* starts,
                     uint32_t* idx, float* w);
// One thread: the f32 mean of the calibrated row sums over rows with links,
// summed in row order (formfactor.rs:242-253).
void launch_mean_row_sum(cudaStream_t st, uint32_t n, const uint32_t* starts, const float* row_sum,
                         float* out_mean, unsigned long long* out_interior);
void launch_sum_u64(cudaStream_t st, const unsigned long long* v, uint32_t n, unsigned long long* out);

// ---- solve (solve.rs:27-108) ----
struct SolveCtl {
    uint32_t done;
    uint32_t iterations;
    uint32_t residual_bits;  // max |delta| of the bounce in progress (non-negative f32 bits)
    uint32_t last_residual;  // residual of the last completed bounce
};
// solve.rs:27-39 with one thread per surfel walking its lights (k_solve.cu);
// terms (nullable): n x nl, each surfel's per-light factor ff * vis (-1 where
// the light is skipped), for the differentiable relight. The light stage uses
// it below kLightSlotsQueued (surfel, light) slots and launch_light_slots
// from there on; both compute the same values in the same order.
static constexpr uint64_t kLightSlotsQueued = 32768;
void launch_light_surfels(cudaStream_t st, BlobRef blob, SurfelArrays s, uint32_t n, unsigned long long* evals,
                          uint32_t* status, unsigned long long* counts = nullptr, float* terms = nullptr);
// The transfer in sliced-ELL form (k_solve.cu): rows sorted by link count
// (descending, stable), slices of 32 consecutive sorted rows, each slice's
// links stored as [link / 4][lane][link % 4] so that a warp's 32 rows read
// one contiguous 512-byte block per 4 links. Every row keeps its links in
// CSR order. perm == nullptr means "use the CSR arrays".
#ifdef IFX_CHECKED
// Bounds-checked build: validates the transfer's CSR and cluster structures.
void launch_check_transfer(cudaStream_t st, uint32_t n, uint32_t nc, unsigned long long links,
                           const uint32_t* starts, const uint32_t* idx, const uint2* crange,
                           const uint32_t* members, uint32_t* status);
#endif

// Bounded grid barrier state of a cooperative launch (kcommon.cuh).
// The arrival count and the generation word sit on separate 128-byte lines,
// so that the CTAs polling `gen` do not contend with the arrivals' atomics.
struct alignas(128) MsBarrier {
    uint32_t count;
    uint32_t pad0[31];
    uint32_t gen;
    uint32_t pad1[31];
};
struct SellMatrix {
    const uint32_t* perm;       // sorted position -> row
    const uint32_t* len;        // sorted position -> link count
    const uint32_t* slice_off;  // per slice: first entry (multiple of 128)
    const uint32_t* idx;
    const float* w;
};
void launch_solve_bounce(cudaStream_t st, SurfelArrays s, uint32_t n, const float4* cp, const uint2* crange,
                         const uint32_t* members, uint32_t nc, const uint32_t* starts, const uint32_t* idx,
                         const float* w, float4* cluster_rad, SolveCtl* ctl, uint32_t it, int* launches,
                         int no_exit = 0, const SellMatrix* sell = nullptr);
// Sliced-ELL construction: row link counts (keys) with the identity (vals);
// after a stable descending sort of (keys, vals), the slice sizes, then the
// interleaved copy of idx and w.
int launch_sell_lens(cudaStream_t st, const uint32_t* starts, uint32_t n, uint32_t* lens, uint32_t* rows);
int launch_sell_sizes(cudaStream_t st, const uint32_t* sorted_len, uint32_t n, uint32_t* sizes);
int launch_sell_fill(cudaStream_t st, const uint32_t* starts, const uint32_t* idx, const float* w, uint32_t n,
                     const uint32_t* perm, const uint32_t* sorted_len, const uint32_t* slice_off, uint32_t* sidx,
                     float* sw);

// ---- batched relighting (solve.rs:47-108 over R right-hand sides) ----
int launch_batch_init(cudaStream_t st, const float* E, uint32_t n, uint32_t R, float4* direct, float4* rad,
                      float4* irr);
int launch_batch_unpack(cudaStream_t st, const float4* x, uint32_t n, uint32_t R, float* out);
int launch_batched_bounce(cudaStream_t st, uint32_t n, uint32_t R, const float4* sp, const float4* albedo,
                          const float4* direct, float4* irr, float4* rad, const float4* cp, const uint2* crange,
                          const uint32_t* members, uint32_t nc, const uint32_t* starts, const uint32_t* idx,
                          const float* w, float4* crad, uint32_t* done, uint32_t* iterations, uint32_t* res_bits,
                          uint32_t* last_res, uint32_t it, int rows_per_block_warps);

// ---- grid + shade (surfel.rs:71-114, main.rs:229-367, film.rs:51-61) ----
void launch_grid_keys(cudaStream_t st, const float4* p, uint32_t n, GridParams g, unsigned long long* keys);
void launch_grid_starts(cudaStream_t st, const unsigned long long* sorted, uint32_t n, uint32_t ncells,
                        uint32_t* starts);
void launch_grid_scatter(cudaStream_t st, const unsigned long long* sorted, uint32_t n, SurfelArrays s,
                         float4* gp, float4* gn, float4* girr, uint32_t* items);

struct ShadeParams {
    BlobRef blob;
    GridParams grid;
    int has_gi;
    CamParams cam;
    uint32_t w, h;
    float tmax;
    int mode;
    float exposure;
    int tonemap;
    const float* srgb_t;  // 256 thresholds
    float* film;          // w*h*3, nullable
    uint8_t* out8;        // w*h*3
    unsigned long long* evals;
    uint32_t* status;
    unsigned long long* counts;  // non-null: the counting instantiation (work counters, kNumCounters u64)
    // Wavefront state, per pixel: hp = (hit point, t), hn = (normal, flags | material);
    // per pixel and light: form factor and visibility; queues of shadow-ray
    // slots (pixel * nl + light) and of mirror-ray pixels with their lengths
    // qlen[0] (primary shadows), qlen[1] (mirror rays), qlen[2] (mirror-hit
    // shadows); persistent-kernel cursors[4]. qlen and cursors start at zero.
    float4 *hp1, *hn1, *hp2, *hn2;
    float *ff1, *vis1, *ff2, *vis2;
    uint32_t *q1, *q2, *qr, *qlen;
    unsigned long long* cursors;
    int nl;  // quad lights + sphere lights
    // Re-composition over stored hits (differentiable forward): emitter
    // pixels are rewritten from the current emissions as well.
    int recompose;
    // k_compose's pixels: [pix0, pix1), or the whole film when pix1 == 0.
    uint32_t pix0, pix1;
};
// Returns the number of kernels launched. `ev` (nullable) holds
// kShadeEvents events recorded around the kernels (see k_shade.cu);
// p.counts (nullable) points at 5 consecutive counter slots.
// `part` selects the passes before the composition (primary hits, their
// shadow rays, mirror rays and theirs: nothing there reads the gather grid),
// the composition, or both.
static constexpr int kShadeEvents = 14;
enum : int { kShadeFront = 1, kShadeCompose = 2, kShadeAll = 3 };
int launch_shade(cudaStream_t st, const ShadeParams& p, cudaEvent_t* ev, int part = kShadeAll);
// k_compose alone over the hits, form factors and visibilities a previous
// launch_shade with the same parameters left in the wavefront buffers.
int launch_compose(cudaStream_t st, const ShadeParams& p);
// solve.rs:27-39 over (surfel, light) slots (k_shade.cu): form factors into
// ff, the queued slots' cone visibilities into vis (k_shadow, with p.q1 /
// p.qlen[0] as the queue and `cursor` its position, both zeroed by the
// caller), then direct = rad = E and irr = 0 per surfel, and terms (nullable,
// n x nl) = ff * vis or -1. Uses p.blob, p.status, p.nl, p.evals (SDF
// evaluations added), p.counts. Returns the kernels launched.
int launch_light_slots(cudaStream_t st, const ShadeParams& p, const SurfelArrays& s, uint32_t n, float* ff,
                       float* vis, float* terms, unsigned long long* cursor);

// ---- differentiation (k_diff.cu) ----
// Pixel flags shared with k_shade.cu (hn1.w / hn2.w): hit, done, emitter.
static constexpr uint32_t kPixHit = 1u << 24;
static constexpr uint32_t kPixDone = 1u << 25;
static constexpr uint32_t kPixEmit = 1u << 26;
static constexpr uint32_t kPixMatMask = (1u << 24) - 1u;

int launch_relight(cudaStream_t st, const float4* albedo, const float* terms, const float4* emit, int nl,
                   uint32_t n, float4* direct, float4* rad, float4* irr);
int launch_grid_refresh(cudaStream_t st, const uint32_t* items, const float4* irr, uint32_t n, float4* girr);
// Pass 0: per pixel, the emission coefficients dpix[l * npix + pix] and the
// number of gather entries cnt[pix]. Pass 1: the entries, at off[pix], as
// (surfel, coefficient xyz + pixel in w).
int launch_diff_pixels(cudaStream_t st, const ShadeParams& p, int pass, float4* dpix, uint32_t* cnt,
                       const uint32_t* off, const uint32_t* gitems, uint32_t* ekey, float4* eval);
int launch_iota(cudaStream_t st, uint32_t* v, uint32_t n);
int launch_link_rows(cudaStream_t st, const uint32_t* starts, uint32_t n, uint32_t* rows);
// CSR row starts (nrows + 1) from sorted row keys.
int launch_csr_starts(cudaStream_t st, const uint32_t* sorted_keys, uint32_t count, uint32_t nrows,
                      uint32_t* starts);
int launch_permute_entries(cudaStream_t st, const uint32_t* perm, const float4* in, uint32_t count, float4* out);
int launch_transpose_fill(cudaStream_t st, const uint32_t* perm, const uint32_t* link_rows, const float* w,
                          uint32_t links, uint2* out);
int launch_cluster_ids(cudaStream_t st, const uint2* crange, const uint32_t* members, uint32_t nc, uint32_t* cid);
// h_i = sum over the pixels that gather surfel i of coef * dL/dimage.
int launch_gather_t(cudaStream_t st, const uint32_t* gstarts, const float4* gent, const float* gimg, uint32_t n,
                    float4* h);
// y_c = sum over links (i, c) of w * t_i (the transposed transfer).
int launch_ft_spmv(cudaStream_t st, const uint32_t* ftstarts, const uint2* ft, const float4* t, uint32_t nc,
                   float4* y);
// Adjoint of bounce k (K..1): b = A^T y; Ebar += b; for k >= 2
// rhobar += b * irr_{k-1} and t = rho * b.
int launch_adj_surfel(cudaStream_t st, const uint32_t* cid, const float4* sp, const float4* cp, const float4* y,
                      const float4* albedo, const float4* irr_prev, uint32_t n, int first, float4* ebar,
                      float4* rhobar, float4* t);
// rhobar += Ebar * S (S = sum_l e_l a_il); the emission gradient from the
// pixels (partials over fixed pixel chunks) and from the surfels, reduced in
// a fixed order into out (nl x 3).
int launch_adj_final(cudaStream_t st, const float4* ebar, const float4* albedo, const float* terms,
                     const float4* emit, int nl, uint32_t n, float4* rhobar);
static constexpr uint32_t kEmitChunk = 4096;
int launch_emit_grad(cudaStream_t st, const float4* dpix, const float* gimg, uint32_t npix, const float4* ebar,
                     const float4* albedo, const float* terms, uint32_t n, int nl, float* partials, float* out);
int launch_unpack3(cudaStream_t st, const float4* in, uint32_t n, float* out);

// ---- packed multi-scene frame (k_multi.cu) ----
// One scene's device state, as its own context prepared it.
struct MsScene {
    const float4* sp;       // surfel position, w = area
    const float4* albedo;
    float4 *direct, *irr, *rad;
    const float* terms;     // n x nl light factors (-1: skipped)
    const float4* lemit;    // nl emissions
    int nl;
    uint32_t n, nc;
    const float4* cp;       // cluster position, w = area
    const uint2* crange;
    const uint32_t* members;
    const uint32_t *starts, *idx;
    const float* w;
    float4* crad;
    const uint32_t* gitems;  // grid slot -> surfel
    float4* girr;
    uint32_t max_bounces;
    uint32_t surf_base, clus_base, pix_base;  // first packed item of this scene
    ShadeParams P;           // the prepared frame (recompose set)
};
struct MsParams {
    const MsScene* scenes;
    int S;
    const uint32_t *surf_base, *clus_base, *pix_base;  // S entries each
    uint32_t total_surf, total_clus, total_pix;
    uint32_t max_bounces;  // largest per-scene cap
    SolveCtl* ctl;         // S
    uint32_t* live;        // scenes still bouncing
    MsBarrier* bar;
    uint32_t* status;
    const float* srgb_t;
    uint32_t polls;        // poll budget of each grid barrier
};
// Cooperative launch (every CTA resident); capturable in a CUDA graph.
// Returns 1, or -1 if the launch was refused.
int launch_multi_frame(cudaStream_t st, const MsParams& p, int grid, int block);
// Largest cooperative grid for this block size on the current device.
int multi_frame_max_blocks(int block);

// Raises the dynamic shared-memory limit of every scene-staging kernel.
void configure_surfel_kernels(int max_dyn_smem);
void configure_transfer_kernels(int max_dyn_smem);
void configure_solve_kernels(int max_dyn_smem);
void configure_shade_kernels(int max_dyn_smem);
void configure_diff_kernels(int max_dyn_smem);
void configure_path_kernels(int max_dyn_smem);
void configure_leafgrid_kernels(int max_dyn_smem);
// The leaf grid (k_leafgrid.cu): per-cell bounds U, then the lists (count
// pass with start == nullptr, fill pass with the scanned starts).
void launch_lg_bound(cudaStream_t st, const BlobRef& blob, const LeafGrid& g, float cell, float half_diag,
                     uint32_t ncells, float* U, uint32_t* status);
void launch_lg_lists(cudaStream_t st, const uint8_t* blob, const LeafGrid& g, double cell, double pad, uint32_t ncells,
                     const float* U, const uint32_t* leaves, uint32_t nleaf, uint32_t* count, const uint32_t* start,
                     uint32_t* out, float* key);
// The path-traced reference mode (k_path.cu): p.film / p.out8 receive the
// frame; sincos holds (sinf, cosf) of the 2^24 sampler angles.
int launch_path(cudaStream_t st, const ShadeParams& p, uint32_t spp, const float2* sincos,
                unsigned long long* cursor);
inline void configure_kernels(int max_dyn_smem) {
    configure_surfel_kernels(max_dyn_smem);
    configure_transfer_kernels(max_dyn_smem);
    configure_solve_kernels(max_dyn_smem);
    configure_shade_kernels(max_dyn_smem);
    configure_diff_kernels(max_dyn_smem);
    configure_path_kernels(max_dyn_smem);
    configure_leafgrid_kernels(max_dyn_smem);
}

}  // namespace ifx
