// Per-pixel shading (main.rs:229-367) with the film encode (film.rs:8-61)
// fused as its epilogue.
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

// main.rs:247-361 for one pixel.
template <class C>
__device__ V shade_pixel(const SceneView& sv, const ShadeParams& P, uint32_t x, uint32_t y, uint32_t& evals,
                         C& cnt) {
    const CamParams& c = P.cam;
    const V org{c.origin[0], c.origin[1], c.origin[2]};
    // main.rs:213-217
    float px = (2.0f * ((float)x + 0.5f) / (float)P.w - 1.0f) * c.aspect * c.tan_half;
    float py = (1.0f - 2.0f * ((float)y + 0.5f) / (float)P.h) * c.tan_half;
    V rd = nrm(V{c.fwd[0], c.fwd[1], c.fwd[2]} + V{c.right[0], c.right[1], c.right[2]} * px +
               V{c.up[0], c.up[1], c.up[2]} * py);
    TraceHit th = trace(sv, org, rd, 1e-3f, P.tmax, cnt);
    evals += th.steps;
    const bool tonemapped = P.mode <= 2;
    V e;
    if (emitter_hit(sv, org, rd, fminf(th.hit ? th.t : kMaxF, P.tmax), e)) return tonemapped ? e : V{0.9f, 0.9f, 0.9f};
    if (!th.hit) return sky();
    if (P.mode == 4) {  // depth
        float d = 1.0f - clampr(th.t / P.tmax, 0.0f, 1.0f);
        return V{d * d, d * d, d * d};
    }
    if (P.mode == 5) {  // steps
        float f = (float)th.steps / 128.0f;
        return V{f, 1.0f - f, 0.2f};
    }
    const V n = scene_normal(sv, th.p, cnt);
    if (P.mode == 3) return n * 0.5f + V{0.5f, 0.5f, 0.5f};  // normals
    const DMaterial& m = sv.mats[th.mat];
    V col{0.0f, 0.0f, 0.0f};
    if (P.mode != 2) {
        uint32_t s = 0;
        V d = direct(sv, th.p, n, -rd, m, s, cnt);
        evals += s;
        col = col + (d + V{m.emissive[0], m.emissive[1], m.emissive[2]});
    }
    if (P.has_gi) {
        GatherView g = gview(P.grid);
        V irr = gather(g, th.p, n, cnt);
        col = col + V{m.kd[0], m.kd[1], m.kd[2]} * irr;
        if (m.f0[3] != 0.0f) {  // roughness < 0.45 || metallic > 0.05
            V refl = rd - n * (2.0f * dot(n, rd));
            TraceHit rh = trace(sv, th.p + n * 1e-3f, refl, 1e-3f, P.tmax, cnt);
            evals += rh.steps;
            V rc;
            V e2;
            if (emitter_hit(sv, th.p, refl, fminf(rh.hit ? rh.t : kMaxF, P.tmax), e2)) {
                rc = e2;
            } else if (rh.hit) {
                const V n2 = scene_normal(sv, rh.p, cnt);
                const DMaterial& m2 = sv.mats[rh.mat];
                uint32_t s2 = 0;
                V d2 = direct(sv, rh.p, n2, -refl, m2, s2, cnt);
                evals += s2;
                V i2 = gather(g, rh.p, n2, cnt);
                rc = d2 + V{m2.kd[0], m2.kd[1], m2.kd[2]} * i2 + V{m2.emissive[0], m2.emissive[1], m2.emissive[2]};
            } else {
                rc = sky();
            }
            V f = fresnel_schlick(fmaxf(dot(n, -rd), 0.0f), V{m.f0[0], m.f0[1], m.f0[2]});
            float gloss = clampr(1.0f - m.albedo[3] / 0.45f, 0.0f, 1.0f);
            gloss = gloss * gloss;
            col = col + f * rc * gloss;
        }
    }
    return col;
}

template <class C>
__global__ void __launch_bounds__(128) k_shade(ShadeParams P) {
    IFX_SCENE_PROLOGUE(P.blob, P.status, sv);
    C cnt;
    __shared__ float t8[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) t8[i] = P.srgb_t[i];
    __syncthreads();
    // 16x8 pixel tiles, grid-stride over tiles; a warp covers 16x2 pixels.
    const uint32_t tiles_x = (P.w + 15) / 16, tiles_y = (P.h + 7) / 8;
    const uint32_t ntiles = tiles_x * tiles_y;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        uint32_t x = (tile % tiles_x) * 16 + (threadIdx.x & 15);
        uint32_t y = (tile / tiles_x) * 8 + (threadIdx.x >> 4);
        unsigned long long ev = 0;
        if (x < P.w && y < P.h) {
            uint32_t e = 0;
            V c = shade_pixel(sv, P, x, y, e, cnt);
            ev = e;
            size_t o = ((size_t)y * P.w + x) * 3;
            if (P.film) {
                P.film[o] = c.x;
                P.film[o + 1] = c.y;
                P.film[o + 2] = c.z;
            }
            if (P.out8) {
                V s = c * P.exposure;
                V m = P.tonemap ? aces(s) : s;
                P.out8[o] = srgb8(t8, m.x);
                P.out8[o + 1] = srgb8(t8, m.y);
                P.out8[o + 2] = srgb8(t8, m.z);
            }
        }
        for (int o = 16; o >= 1; o >>= 1) ev += __shfl_xor_sync(kFull, ev, o);
        if ((threadIdx.x & 31) == 0 && ev) atomicAdd(P.evals, ev);
    }
    if constexpr (sizeof(C) > 1) cnt.flush(P.counts);
}

void launch_shade(cudaStream_t st, const ShadeParams& p) {
    unsigned long long tiles = (unsigned long long)((p.w + 15) / 16) * ((p.h + 7) / 8);
    const unsigned g = grid_for(tiles * 128ull, 128, 16);
    if (p.counts) k_shade<Counts><<<g, 128, blob_smem(p.blob), st>>>(p);
    else k_shade<NoCount><<<g, 128, blob_smem(p.blob), st>>>(p);
}

void configure_shade_kernels(int max_dyn_smem) {
    cudaFuncSetAttribute(k_shade<NoCount>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_shade<Counts>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
}

}  // namespace ifx
