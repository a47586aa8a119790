// The brute-force path tracer of `--mode reference` (reference.rs:24-137,
// main.rs:249-259): per pixel a PCG32 stream seeded with (y << 32) | x, spp
// paths of at most 12 vertices, next-event estimation against every quad
// light, cosine-weighted bounces, Russian roulette after depth 3. Each lane
// takes whole pixels from a global cursor (a pixel's samples are sequential
// in its random stream). The sine and cosine of the sampled azimuth come from
// a host table of the platform libm's sinf/cosf over the 2^24 angles the
// sampler can produce, so every pixel matches the CPU path bit for bit.
#include "shade.cuh"

namespace ifx {

// reference.rs:31-46: returns the 24-bit draw k; the sample is k * 2^-24.
struct Pcg32 {
    unsigned long long s;
    __device__ __forceinline__ explicit Pcg32(unsigned long long seed) : s(seed * 6364136223846793005ull + 1ull) {}
    __device__ __forceinline__ uint32_t next24() {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        const unsigned long long x = ((s >> 18) ^ s) >> 27;
        const uint32_t rot = (uint32_t)(s >> 59);
        const uint32_t v0 = (uint32_t)x;
        const uint32_t v = (v0 >> rot) | (v0 << ((32u - rot) & 31u));
        return v >> 8;
    }
    __device__ __forceinline__ float next_f32() { return (float)next24() * (1.0f / 16777216.0f); }
};

// reference.rs:48-57; sincos[k] = (sinf(TAU * u), cosf(TAU * u)), u = k * 2^-24.
__device__ __forceinline__ V cosine_hemisphere(V n, Pcg32& rng, const float2* sincos) {
    V t, b;
    frame(n, t, b);
    const float u1 = rng.next_f32();
    const uint32_t k2 = rng.next24();
    const float r = sqrtf(u1);
    const float2 sc = __ldg(&sincos[k2]);
    return nrm(t * (r * sc.y) + b * (r * sc.x) + n * sqrtf(fmaxf(1.0f - u1, 0.0f)));
}

// reference.rs:61-137. `cnt` tallies the tracing work (counting launches
// only; the timed kernel uses NoCount).
template <class C>
__device__ V path(const SceneView& sv, V ro, V rd, float tmax, uint32_t max_depth, Pcg32& rng,
                  const float2* sincos, C& cnt) {
    V radiance{0.0f, 0.0f, 0.0f}, throughput{1.0f, 1.0f, 1.0f};
    V origin = ro, dir = rd;
    for (uint32_t depth = 0; depth < max_depth; ++depth) {
        const TraceHit h = trace(sv, origin, dir, 1e-3f, tmax, cnt);
        const float surf_t = h.hit ? h.t : kMaxF;
        V e;
        if (emitter_hit(sv, origin, dir, fminf(surf_t, tmax), e, nullptr, true)) {
            if (depth == 0) radiance = radiance + throughput * e;
            break;
        }
        if (!h.hit) break;
        const V n = scene_normal(sv, h.p, cnt);
        const DMaterial& m = sv.mats[h.mat];
        const V albedo{m.kd[0], m.kd[1], m.kd[2]};
        radiance = radiance + throughput * V{m.emissive[0], m.emissive[1], m.emissive[2]};
        for (int li = 0; li < sv.n_lights; ++li) {
            const DQuadLight& L = sv.lights[li];
            const V v0{L.v[0][0], L.v[0][1], L.v[0][2]};
            const V e1 = V{L.v[1][0], L.v[1][1], L.v[1][2]} - v0;
            const V e2 = V{L.v[3][0], L.v[3][1], L.v[3][2]} - v0;
            const float r1 = rng.next_f32();
            const float r2 = rng.next_f32();
            const V lp = v0 + e1 * r1 + e2 * r2;
            const V to = lp - h.p;
            const float dist2 = dot(to, to);
            if (dist2 < 1e-9f) continue;
            const float dist = sqrtf(dist2);
            const V l = to / dist;
            const float cos_s = dot(n, l);
            const float cos_l = dot(V{L.normal[0], L.normal[1], L.normal[2]}, -l);
            if (cos_s <= 0.0f || cos_l <= 0.0f) continue;
            if (trace(sv, h.p + n * 1e-3f, l, 1e-3f, dist - 1e-2f, cnt).hit) continue;
            const float pdf = dist2 / (cos_l * L.normal[3]);
            radiance = radiance + throughput * albedo * V{L.emit[0], L.emit[1], L.emit[2]} * (cos_s / (kPiF * pdf));
        }
        throughput = throughput * albedo;
        dir = cosine_hemisphere(n, rng, sincos);
        origin = h.p + n * 1e-3f;
        if (depth >= 3) {
            const float q = clampr(fmaxf(throughput.x, fmaxf(throughput.y, throughput.z)), 0.05f, 0.95f);
            if (rng.next_f32() > q) break;
            throughput = throughput / q;
        }
    }
    return radiance;
}

template <class C>
__global__ void __launch_bounds__(128) k_path(ShadeParams P, uint32_t spp, const float2* sincos,
                                               unsigned long long* cursor) {
    C cnt;
    IFX_SCENE_PROLOGUE(P.blob, P.status, sv);
    __shared__ float t8[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) t8[i] = P.srgb_t[i];
    __syncthreads();
    const V org{P.cam.origin[0], P.cam.origin[1], P.cam.origin[2]};
    const unsigned long long total = (unsigned long long)P.w * P.h;
    while (true) {
        const unsigned long long pix = atomicAdd(cursor, 1ull);
        if (pix >= total) break;
        const uint32_t x = (uint32_t)(pix % P.w), y = (uint32_t)(pix / P.w);
        const V rd = camera_ray(P, (uint32_t)pix);
        Pcg32 rng(((unsigned long long)y << 32) | (unsigned long long)x);
        V acc{0.0f, 0.0f, 0.0f};
        for (uint32_t i = 0; i < spp; ++i) acc = acc + path(sv, org, rd, P.tmax, 12u, rng, sincos, cnt);
        write_pixel(P, t8, (uint32_t)pix, acc / (float)spp);
    }
    if constexpr (sizeof(C) > 1) cnt.flush(P.counts);
}

int launch_path(cudaStream_t st, const ShadeParams& p, uint32_t spp, const float2* sincos,
                unsigned long long* cursor) {
    const size_t sm = blob_smem(p.blob, 128);
    const unsigned long long px = (unsigned long long)p.w * p.h;
    if (p.counts)
        k_path<Counts><<<persistent_grid(k_path<Counts>, 128, sm, px), 128, sm, st>>>(p, spp, sincos, cursor);
    else
        k_path<NoCount><<<persistent_grid(k_path<NoCount>, 128, sm, px), 128, sm, st>>>(p, spp, sincos, cursor);
    return 1;
}

void configure_path_kernels(int max_dyn_smem) {
    cudaFuncSetAttribute(k_path<NoCount>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_path<Counts>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
}

}  // namespace ifx
