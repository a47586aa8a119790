// The brute-force path tracer of `--mode reference` (reference.rs:24-137,
// main.rs:249-259): per pixel a PCG32 stream seeded with (y << 32) | x, spp
// paths of at most 12 vertices, next-event estimation against every quad
// light, cosine-weighted bounces, Russian roulette after depth 3. Each lane
// takes whole pixels from a global cursor (a pixel's samples are sequential
// in its random stream, so they cannot be spread over lanes). The sine and cosine of the sampled azimuth come from
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

// reference.rs:61-137 as a per-lane state machine, so that every loop
// iteration is one warp-synchronous SDF query (dist_mat_warp) for whatever
// each lane marches at that moment: its camera or bounce ray, one of the four
// normal taps at a hit, or the hard shadow ray toward a light. A lane that
// finishes a march moves on at once (next light, next bounce, next sample,
// next pixel from the global cursor) instead of idling while the rest of its
// warp finishes a longer loop. Each lane's sequence of operations (and of
// random draws) is exactly the reference's for its pixel, so films are
// bit-identical to the CPU path tracer.
enum : int { kPhIdle = 0, kPhMain = 1, kPhTap = 2, kPhShadow = 3 };

template <class C>
__global__ void __launch_bounds__(128) k_path(ShadeParams P, uint32_t spp, const float2* sincos,
                                               unsigned long long* cursor) {
    IFX_SCENE_PROLOGUE(P.blob, P.status, sv);
    C cnt;
    __shared__ float t8[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) t8[i] = P.srgb_t[i];
    __syncthreads();
    const V org{P.cam.origin[0], P.cam.origin[1], P.cam.origin[2]};
    const unsigned long long total = (unsigned long long)P.w * P.h;
    const float tmax = P.tmax;
    constexpr uint32_t kMaxDepth = 12u;  // main.rs:255
    WarpQueue q(total);

    int phase = kPhIdle, tap = 0, li = 0;
    uint32_t pix = 0, sample = 0, depth = 0, hmat = 0;
    Pcg32 rng(0ull);
    V cam_rd{}, acc{}, radiance{}, throughput{}, hp{}, n{}, contrib{};
    TraceRay ray{};
    while (true) {
        const uint32_t got = q.refill(phase == kPhIdle, total, cursor);
        if (got != ~0u) {
            pix = got;
            const uint32_t x = pix % P.w, y = pix / P.w;
            cam_rd = camera_ray(P, pix);
            rng = Pcg32(((unsigned long long)y << 32) | (unsigned long long)x);
            acc = V{0.0f, 0.0f, 0.0f};
            sample = 0;
            radiance = V{0.0f, 0.0f, 0.0f};
            throughput = V{1.0f, 1.0f, 1.0f};
            depth = 0;
            ray = TraceRay{org, cam_rd, 1e-3f, tmax, 0u};
            phase = kPhMain;
        }
        if (!__any_sync(kFull, phase != kPhIdle)) {
            if (q.empty()) break;
            continue;
        }
        const bool active = phase != kPhIdle;
        // scene.rs:218-236 tap offsets, in the order scene_normal() sums them.
        const float kx = (tap == 0 || tap == 3) ? 1.0f : -1.0f, ky = tap >= 2 ? 1.0f : -1.0f,
                    kz = (tap == 1 || tap == 3) ? 1.0f : -1.0f;
        const V qp = phase == kPhTap ? hp + V{kx, ky, kz} * 5e-4f : ray.ro + ray.rd * ray.t;
        const DistHit h = dist_mat_warp(sv, qp, active, cnt);
        if (!active) continue;

        // Where the lane goes after this query.
        enum : int { kQuery, kSurface, kNee, kBounce, kEndPath } act = kQuery;
        if (phase == kPhMain || phase == kPhShadow) {
            // trace.rs:27-58, one step
            cnt.add(CN_TSTEP);
            ray.steps += 1;
            const float eps = 1e-4f * fmaxf(ray.t, 1.0f);
            const bool hit = h.d < eps;
            bool done = hit;
            if (!hit) {
                ray.t += h.d;
                done = ray.t > ray.tmax || ray.steps >= kMaxSteps;
            }
            if (done && phase == kPhMain) {
                // reference.rs:71-86
                const float surf_t = hit ? ray.t : kMaxF;
                V e;
                if (emitter_hit(sv, ray.ro, ray.rd, fminf(surf_t, tmax), e, nullptr, true)) {
                    if (depth == 0) radiance = radiance + throughput * e;
                    act = kEndPath;
                } else if (!hit) {
                    act = kEndPath;
                } else {
                    hp = qp;
                    hmat = h.mat;
                    n = V{0.0f, 0.0f, 0.0f};
                    tap = 0;
                    phase = kPhTap;
                }
            } else if (done) {
                // reference.rs:107-116: the hard shadow ray ended
                if (!hit) radiance = radiance + contrib;
                ++li;
                act = kNee;
            }
        } else {
            n = n + V{kx, ky, kz} * h.d;
            if (++tap == 4) {
                const float l = len(n);
                n = l > 1e-12f ? n / l : V{0.0f, 1.0f, 0.0f};
                act = kSurface;
            }
        }
        if (act == kSurface) {
            const DMaterial& m = sv.mat(hmat);
            radiance = radiance + throughput * V{m.emissive[0], m.emissive[1], m.emissive[2]};
            li = 0;
            act = kNee;
        }
        if (act == kNee) {
            // reference.rs:89-118: the next light whose sample needs a shadow ray
            const DMaterial& m = sv.mat(hmat);
            const V albedo{m.kd[0], m.kd[1], m.kd[2]};
            act = kBounce;
            for (; li < sv.n_lights; ++li) {
                const DQuadLight& L = sv.light(li);
                const V v0{L.v[0][0], L.v[0][1], L.v[0][2]};
                const V e1 = V{L.v[1][0], L.v[1][1], L.v[1][2]} - v0;
                const V e2 = V{L.v[3][0], L.v[3][1], L.v[3][2]} - v0;
                const float r1 = rng.next_f32();
                const float r2 = rng.next_f32();
                const V lp = v0 + e1 * r1 + e2 * r2;
                const V to = lp - hp;
                const float dist2 = dot(to, to);
                if (dist2 < 1e-9f) continue;
                const float dist = sqrtf(dist2);
                const V l = to / dist;
                const float cos_s = dot(n, l);
                const float cos_l = dot(V{L.normal[0], L.normal[1], L.normal[2]}, -l);
                if (cos_s <= 0.0f || cos_l <= 0.0f) continue;
                const float pdf = dist2 / (cos_l * L.normal[3]);
                contrib = throughput * albedo * V{L.emit[0], L.emit[1], L.emit[2]} * (cos_s / (kPiF * pdf));
                ray = TraceRay{hp + n * 1e-3f, l, 1e-3f, dist - 1e-2f, 0u};
                phase = kPhShadow;
                act = kQuery;
                break;
            }
        }
        if (act == kBounce) {
            // reference.rs:120-133
            const DMaterial& m = sv.mat(hmat);
            throughput = throughput * V{m.kd[0], m.kd[1], m.kd[2]};
            const V dir = cosine_hemisphere(n, rng, sincos);
            const V origin = hp + n * 1e-3f;
            act = kQuery;
            if (depth >= 3) {
                const float qq = clampr(fmaxf(throughput.x, fmaxf(throughput.y, throughput.z)), 0.05f, 0.95f);
                if (rng.next_f32() > qq) act = kEndPath;
                else throughput = throughput / qq;
            }
            if (act == kQuery) {
                if (++depth >= kMaxDepth) {
                    act = kEndPath;
                } else {
                    ray = TraceRay{origin, dir, 1e-3f, tmax, 0u};
                    phase = kPhMain;
                }
            }
        }
        if (act == kEndPath) {
            // main.rs:254-257
            acc = acc + radiance;
            if (++sample == spp) {
                write_pixel(P, t8, pix, acc / (float)spp);
                phase = kPhIdle;
            } else {
                radiance = V{0.0f, 0.0f, 0.0f};
                throughput = V{1.0f, 1.0f, 1.0f};
                depth = 0;
                ray = TraceRay{org, cam_rd, 1e-3f, tmax, 0u};
                phase = kPhMain;
            }
        }
    }
    if constexpr (sizeof(C) > 1) cnt.flush(P.counts);
}

int launch_path(cudaStream_t st, const ShadeParams& p, uint32_t spp, const float2* sincos,
                unsigned long long* cursor) {
    const size_t sm = blob_smem(p.blob, 128);
    const unsigned long long px = (unsigned long long)p.w * p.h;
    if (p.counts)
        k_path<Counts><<<persistent_grid(k_path<Counts>, 128, sm, px), 128, sm, st>>>(p, spp, sincos, cursor);
    else if (p.blob.tree3)
        k_path<NoCount3><<<persistent_grid(k_path<NoCount3>, 128, sm, px), 128, sm, st>>>(p, spp, sincos, cursor);
    else
        k_path<NoCount><<<persistent_grid(k_path<NoCount>, 128, sm, px), 128, sm, st>>>(p, spp, sincos, cursor);
    return 1;
}

void configure_path_kernels(int max_dyn_smem) {
    cudaFuncSetAttribute(k_path<NoCount>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_path<NoCount3>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
    cudaFuncSetAttribute(k_path<Counts>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
}

}  // namespace ifx
