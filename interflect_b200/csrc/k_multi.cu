// Packed multi-scene frame: the solve and the shade of many independent
// scenes in ONE persistent cooperative launch (no counterpart in the
// reference, which renders one scene per process).
//
// Each scene was prepared through its own context: transfer, gather grid,
// per-surfel light factors (the emission-free terms of solve.rs:27-39) and
// one beauty frame whose hits, form factors and visibilities stay in that
// context's wavefront buffers. Per launch, for every scene at once:
//
//   relight   E_i = sum_l (rho_i * e_l) * a_il        (solve.rs:30-36)
//   bounce k  cluster means, Jacobi rows, per-scene stop rule
//                                                     (solve.rs:47-108)
//   refresh   the grid's copy of irr                  (surfel.rs:262-293)
//   compose   every pixel from its stored hits        (main.rs:289-358)
//
// Work items of all scenes are packed end to end (scene-major) and handed
// out grid-stride; phases are separated by a bounded grid barrier (the
// launch is cooperative, so every CTA is resident). Every item performs
// exactly the operations of the single-scene kernels in the same order,
// so each scene is bit-identical to its own unbatched frame, whatever the
// packing, block size or grid.
#include "shade.cuh"

namespace ifx {

// Scene owning packed item `item`: the last scene whose base is <= item.
__device__ __forceinline__ int scene_of(const uint32_t* base, int S, uint32_t item) {
    int lo = 0, hi = S - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (base[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(256) k_multi_frame(MsParams M) {
    __shared__ float t8[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) t8[i] = M.srgb_t[i];
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    const MsScene* sc = M.scenes;

    // Relight, and reset the per-scene solve controls.
    for (uint32_t s = tid; s < (uint32_t)M.S; s += stride) M.ctl[s] = SolveCtl{0u, 0u, 0u, 0u};
    if (tid == 0) M.live[0] = (uint32_t)M.S;
    for (uint32_t item = tid; item < M.total_surf; item += stride) {
        const MsScene& S = sc[scene_of(M.surf_base, M.S, item)];
        const uint32_t i = item - S.surf_base;
        const V rho = mk4(S.albedo[i]);
        V out{0.0f, 0.0f, 0.0f};
        for (int l = 0; l < S.nl; ++l) {
            const float a = S.terms[(size_t)i * S.nl + l];
            if (a < 0.0f) continue;
            out = out + rho * mk4(S.lemit[l]) * a;
        }
        S.direct[i] = f4(out, 0.0f);
        S.rad[i] = f4(out, 0.0f);
        S.irr[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    if (!grid_barrier(M.bar, M.status, M.polls)) return;

    for (uint32_t it = 0; it < M.max_bounces; ++it) {
        // solve.rs:61-73: cluster means, members summed in member order.
        for (uint32_t item = tid; item < M.total_clus; item += stride) {
            const int s = scene_of(M.clus_base, M.S, item);
            if (M.ctl[s].done) continue;
            const MsScene& S = sc[s];
            const uint32_t c = item - S.clus_base;
            const uint2 r = S.crange[c];
            V acc{0.0f, 0.0f, 0.0f};
            for (uint32_t k = r.x; k < r.y; ++k) {
                const uint32_t m = S.members[k];
                const float4 v = S.rad[m];
                const float a = S.sp[m].w;
                acc = acc + V{v.x * a, v.y * a, v.z * a};
            }
            S.crad[c] = f4(acc / fmaxf(S.cp[c].w, 1e-12f), 0.0f);
        }
        if (!grid_barrier(M.bar, M.status, M.polls)) return;
        // solve.rs:76-102: Jacobi rows; the residual is the per-scene max.
        for (uint32_t item = tid; item < M.total_surf; item += stride) {
            const int s = scene_of(M.surf_base, M.S, item);
            uint32_t bits = 0;  // this row's change as non-negative f32 bits (NaN ignored)
            if (!M.ctl[s].done) {
                const MsScene& S = sc[s];
                const uint32_t i = item - S.surf_base;
                V irr{0.0f, 0.0f, 0.0f};
                const uint32_t e = S.starts[i + 1];
                for (uint32_t k = S.starts[i]; k < e; ++k) irr = irr + mk4(S.crad[S.idx[k]]) * S.w[k];
                V nr = mk4(S.direct[i]) + mk4(S.albedo[i]) * irr;
                V diff = vabs(nr - mk4(S.rad[i]));
                float d = fmaxf(diff.x, fmaxf(diff.y, diff.z));
                S.irr[i] = f4(irr, 0.0f);
                S.rad[i] = f4(nr, 0.0f);
                if (!isnan(d) && d > 0.0f) bits = __float_as_uint(d);
            }
            // One atomic per (warp, scene): the lanes of a scene reduce first.
            const unsigned grp = __match_any_sync(__activemask(), s);
            bits = __reduce_max_sync(grp, bits);
            if ((int)(threadIdx.x & 31) == __ffs(grp) - 1 && bits) atomicMax(&M.ctl[s].residual_bits, bits);
        }
        if (!grid_barrier(M.bar, M.status, M.polls)) return;
        // solve.rs:93-101 per scene, with each scene's own bounce cap.
        if (blockIdx.x == 0) {
            __shared__ uint32_t live;
            if (threadIdx.x == 0) live = 0;
            __syncthreads();
            for (int s = threadIdx.x; s < M.S; s += blockDim.x) {
                SolveCtl& c = M.ctl[s];
                if (c.done) continue;
                const float res = __uint_as_float(c.residual_bits);
                c.iterations = it + 1;
                c.last_residual = c.residual_bits;
                c.residual_bits = 0;
                if (res < 1e-4f || it + 1 >= sc[s].max_bounces) c.done = 1;
                else atomicAdd(&live, 1u);
            }
            __syncthreads();
            if (threadIdx.x == 0) M.live[0] = live;
        }
        if (!grid_barrier(M.bar, M.status, M.polls)) return;
        if (*(volatile uint32_t*)&M.live[0] == 0) break;
    }

    // The grid's irradiance copy.
    for (uint32_t item = tid; item < M.total_surf; item += stride) {
        const MsScene& S = sc[scene_of(M.surf_base, M.S, item)];
        const uint32_t k = item - S.surf_base;
        S.girr[k] = S.irr[S.gitems[k]];
    }
    if (!grid_barrier(M.bar, M.status, M.polls)) return;

    // main.rs:289-358 for every pixel of every scene.
    NoCount cnt;
    for (uint32_t item = tid; item < M.total_pix; item += stride) {
        const MsScene& S = sc[scene_of(M.pix_base, M.S, item)];
        const SceneView sv = make_view(S.P.blob.ptr);
        const GatherView g = gview(S.P.grid);
        compose_pixel(sv, S.P, t8, g, item - S.pix_base, cnt);
    }
}

int launch_multi_frame(cudaStream_t st, const MsParams& p, int grid, int block) {
    void* args[] = {const_cast<MsParams*>(&p)};
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, (const void*)k_multi_frame, args) == cudaSuccess ? 1 : -1;
}

int multi_frame_max_blocks(int block) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_multi_frame, block, 0) != cudaSuccess) return 0;
    return per_sm * sm_count();
}

}  // namespace ifx
