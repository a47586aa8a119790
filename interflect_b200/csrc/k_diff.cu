// Differentiation: gradients of an image loss with respect to per-surfel
// albedo and per-light emission, geometry and visibility held fixed (no
// counterpart in the reference).
//
// With the hits, form factors and visibilities of one beauty frame kept in
// the wavefront buffers, the frame is an affine function of the emissions
// and of the irradiance after K bounces:
//   image = sum_l Dpix_l * e_l + G irr_K + const          (main.rs:289-356)
//   E = rho * sum_l e_l * a_l;  B_0 = E;  B_k = E + rho * F A B_{k-1}
//   irr_k = F A B_{k-1}                                    (solve.rs:47-108)
// where a_l = ff * vis of each surfel (shade.rs:133-164), A the area-weighted
// cluster mean, F the transfer and G the normalised gathers
// (surfel.rs:262-293). The adjoint runs the bounces backwards on the
// transposed operators: G^T and F^T are built once on the GPU by a stable
// radix sort of (column, position) pairs, so every output is a sum over a
// fixed, sorted list and the gradient is bit-identical across runs and launch
// shapes (no floating-point atomics anywhere).
#include "kcommon.cuh"

namespace ifx {

// ----------------------------------------------------------- forward ----
// E_i = sum_l (rho_i * e_l) * a_il over the lights the light stage does not
// skip, in light order: the operations of the light stage's light loop with
// the stored factors, so the result is bit-identical to it.
__global__ void k_relight(const float4* albedo, const float* terms, const float4* emit, int nl, uint32_t n,
                          float4* direct, float4* rad, float4* irr) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V rho = mk4(albedo[i]);
        V out{0.0f, 0.0f, 0.0f};
        for (int l = 0; l < nl; ++l) {
            const float a = terms[(size_t)i * nl + l];
            if (a < 0.0f) continue;
            out = out + rho * mk4(emit[l]) * a;
        }
        direct[i] = f4(out, 0.0f);
        rad[i] = f4(out, 0.0f);
        irr[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

// The grid's irradiance copy (surfel.rs:262-293 reads irr in grid order).
__global__ void k_grid_refresh(const uint32_t* items, const float4* irr, uint32_t n, float4* girr) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        girr[k] = irr[items[k]];
}

// ---------------------------------------------------- linearisation ----
__device__ __forceinline__ GatherView gview_d(const GridParams& g) {
    GatherView v;
    v.gp = g.gp;
    v.gn = g.gn;
    v.girr = g.girr;
    v.starts = g.starts;
    for (int a = 0; a < 3; ++a) {
        v.dim[a] = g.dim[a];
        v.lo[a] = g.lo[a];
    }
    v.inv_cell = g.inv_cell;
    v.radius = g.radius;
    return v;
}

// surfel.rs:262-293's walk: f(k, w) for every accepted grid slot k, in the
// gather's order; returns the weight sum as the gather forms it.
template <class F>
__device__ __forceinline__ float gather_walk(const GatherView& g, V p, V n, F&& f) {
    float wsum = 0.0f;
    float r2 = g.radius * g.radius;
    int cx = clampi(as_i32((p.x - g.lo[0]) * g.inv_cell), 0, g.dim[0] - 1);
    int cy = clampi(as_i32((p.y - g.lo[1]) * g.inv_cell), 0, g.dim[1] - 1);
    int cz = clampi(as_i32((p.z - g.lo[2]) * g.inv_cell), 0, g.dim[2] - 1);
    for (int z = max(cz - 1, 0); z <= min(cz + 1, g.dim[2] - 1); ++z)
        for (int y = max(cy - 1, 0); y <= min(cy + 1, g.dim[1] - 1); ++y) {
            size_t row = (size_t)g.dim[0] * ((size_t)y + (size_t)g.dim[1] * (size_t)z);
            int x0 = max(cx - 1, 0), x1 = min(cx + 1, g.dim[0] - 1);
            uint32_t s = __ldg(&g.starts[row + x0]);
            uint32_t e = __ldg(&g.starts[row + x1 + 1]);
            for (uint32_t k = s; k < e; ++k) {
                float4 sp = __ldg(&g.gp[k]);
                float d2 = dot(mk4(sp) - p, mk4(sp) - p);
                if (d2 > r2) continue;
                float align = dot(mk4(__ldg(&g.gn[k])), n);
                if (align <= 0.15f) continue;
                float t = 1.0f - d2 / r2;
                float w = t * t * align;
                f(k, w);
                wsum += w;
            }
        }
    return wsum;
}

// shade.rs:104-121 without the radiance factor: f * d * vis * energy * n.l.
__device__ __forceinline__ V spec_factor(V p, V n, V v, V rep, float radius, float alpha, float n_dot_v, V f0) {
    V l = nrm(rep - p);
    float n_dot_l = dot(n, l);
    if (n_dot_l <= 0.0f) return V{0.0f, 0.0f, 0.0f};
    float rep_dist = fmaxf(len(rep - p), 1e-4f);
    float wide = clampr(alpha + radius / (2.0f * rep_dist), alpha, 1.0f);
    float energy = (alpha / wide) * (alpha / wide);
    V h = nrm(l + v);
    float d = d_ggx(fmaxf(dot(n, h), 0.0f), wide);
    float vis_s = v_smith(n_dot_v, n_dot_l, wide);
    V f = fresnel_schlick(fmaxf(dot(l, h), 0.0f), f0);
    return f * (d * vis_s * energy * n_dot_l);
}

// shade.rs:50-125 from the stored form factors and visibilities, emission
// factored out: acc(l, coefficient of e_l), scaled by `scale`.
template <class F>
__device__ __forceinline__ void direct_coeffs(const SceneView& sv, V p, V n, V v, const DMaterial& m,
                                              const float* ffs, const float* viss, V scale, F&& acc) {
    float n_dot_v = fmaxf(dot(n, v), 1e-4f);
    float alpha = m.kd[3];
    V f0{m.f0[0], m.f0[1], m.f0[2]};
    V kd{m.kd[0], m.kd[1], m.kd[2]};
    for (int li = 0; li < sv.n_lights; ++li) {
        const DQuadLight& L = sv.light(li);
        V lc{L.center[0], L.center[1], L.center[2]};
        V ln{L.normal[0], L.normal[1], L.normal[2]};
        if (dot(ln, -nrm(lc - p)) <= 0.0f) continue;
        float ff = ffs[li];
        if (ff <= 1e-6f) continue;
        float vis = viss[li];
        if (vis <= 1e-4f) continue;
        V r = (-v) - n * (2.0f * dot(n, -v));
        float denom = dot(r, ln);
        V rep = lc;
        if (fabsf(denom) > 1e-6f) {
            float t = dot(V{L.v[0][0], L.v[0][1], L.v[0][2]} - p, ln) / denom;
            if (t > 0.0f) rep = closest_on_quad(L, p + r * t);
        }
        V c = kd * (vis * ff) + spec_factor(p, n, v, rep, L.center[3], alpha, n_dot_v, f0) * vis;
        acc(li, c * scale);
    }
    for (int si = 0; si < sv.n_slights; ++si) {
        const int li = sv.n_lights + si;
        const DSphereLight& S = sv.slight(si);
        V to_light = V{S.c[0], S.c[1], S.c[2]} - p;
        float ff = ffs[li];
        if (ff <= 1e-6f) continue;
        float radius = fmaxf(S.c[3], 1e-4f);
        float vis = viss[li];
        if (vis <= 1e-4f) continue;
        V r = (-v) - n * (2.0f * dot(n, -v));
        V ctr = r * dot(to_light, r) - to_light;
        float cl = len(ctr);
        V rep = p + to_light + ctr * clampr(radius / fmaxf(cl, 1e-9f), 0.0f, 1.0f);
        V c = kd * (vis * ff) + spec_factor(p, n, v, rep, radius, alpha, n_dot_v, f0) * vis;
        acc(li, c * scale);
    }
}

// Gather entries of one surface point: coefficient scale * w / wsum per
// accepted surfel, nothing when the weight sum is below the 1e-6 cut.
template <class F>
__device__ __forceinline__ uint32_t gather_entries(const GatherView& g, V p, V n, V scale, F&& emit) {
    uint32_t count = 0;
    const float wsum = gather_walk(g, p, n, [&](uint32_t, float) { ++count; });
    if (!(wsum > 1e-6f)) return 0;
    gather_walk(g, p, n, [&](uint32_t k, float w) { emit(k, scale * (w / wsum)); });
    return count;
}

// main.rs:289-356 linearised per pixel (beauty mode with the GI solve).
__global__ void __launch_bounds__(128) k_diff_pixels(ShadeParams P, int pass, float4* dpix, uint32_t* cnt,
                                                      const uint32_t* off, const uint32_t* gitems, uint32_t* ekey,
                                                      float4* eval) {
    IFX_SCENE_PROLOGUE(P.blob, P.status, sv);
    const uint32_t total = P.w * P.h;
    const GatherView g = gview_d(P.grid);
    const int nl = P.nl;
    const V one{1.0f, 1.0f, 1.0f};
    for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < total; pix += gridDim.x * blockDim.x) {
        const float4 b = P.hn1[pix];
        const uint32_t flags = __float_as_uint(b.w);
        uint32_t wpos = pass ? off[pix] : 0u;
        auto put = [&](uint32_t k, V c) {
            ekey[wpos] = gitems[k];
            eval[wpos] = make_float4(c.x, c.y, c.z, __uint_as_float(pix));
            ++wpos;
        };
        auto nop = [&](uint32_t, V) {};
        auto acc = [&](int l, V c) {
            float4& d = dpix[(size_t)l * total + pix];
            d = make_float4(d.x + c.x, d.y + c.y, d.z + c.z, 0.0f);
        };
        if (pass == 0)
            for (int l = 0; l < nl; ++l) dpix[(size_t)l * total + pix] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (flags & kPixDone) {
            if (pass == 0) {
                if (flags & kPixEmit) acc((int)__float_as_uint(b.y), one);
                cnt[pix] = 0;
            }
            continue;
        }
        // main.rs:213-217, as k_shade.cu's camera_ray forms it.
        const uint32_t x = pix % P.w, y = pix / P.w;
        float px = (2.0f * ((float)x + 0.5f) / (float)P.w - 1.0f) * P.cam.aspect * P.cam.tan_half;
        float py = (1.0f - 2.0f * ((float)y + 0.5f) / (float)P.h) * P.cam.tan_half;
        const V rd = nrm(V{P.cam.fwd[0], P.cam.fwd[1], P.cam.fwd[2]} +
                         V{P.cam.right[0], P.cam.right[1], P.cam.right[2]} * px +
                         V{P.cam.up[0], P.cam.up[1], P.cam.up[2]} * py);
        const V p = mk4(P.hp1[pix]), n = mk4(b);
        const DMaterial& m = sv.mat(flags & kPixMatMask);
        const V kd{m.kd[0], m.kd[1], m.kd[2]};
        if (pass == 0) direct_coeffs(sv, p, n, -rd, m, P.ff1 + (size_t)pix * nl, P.vis1 + (size_t)pix * nl, one, acc);
        uint32_t count = pass ? gather_entries(g, p, n, kd, put) : gather_entries(g, p, n, kd, nop);
        if (m.f0[3] != 0.0f) {
            const V refl = rd - n * (2.0f * dot(n, rd));
            const float4 a2 = P.hp2[pix];
            const float4 b2 = P.hn2[pix];
            const uint32_t f2 = __float_as_uint(b2.w);
            V f = fresnel_schlick(fmaxf(dot(n, -rd), 0.0f), V{m.f0[0], m.f0[1], m.f0[2]});
            float gloss = clampr(1.0f - m.albedo[3] / 0.45f, 0.0f, 1.0f);
            gloss = gloss * gloss;
            const V fg = f * gloss;
            if (f2 & kPixEmit) {
                if (pass == 0) acc((int)__float_as_uint(b2.x), fg);
            } else if (f2 & kPixHit) {
                const V p2 = mk4(a2), n2 = mk4(b2);
                const DMaterial& m2 = sv.mat(f2 & kPixMatMask);
                if (pass == 0)
                    direct_coeffs(sv, p2, n2, -refl, m2, P.ff2 + (size_t)pix * nl, P.vis2 + (size_t)pix * nl, fg,
                                  acc);
                const V kd2 = V{m2.kd[0], m2.kd[1], m2.kd[2]} * fg;
                count += pass ? gather_entries(g, p2, n2, kd2, put) : gather_entries(g, p2, n2, kd2, nop);
            }
        }
        if (pass == 0) cnt[pix] = count;
    }
}

// -------------------------------------------------------- transposes ----
__global__ void k_iota(uint32_t* v, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

// Row index of every CSR entry.
__global__ void k_link_rows(const uint32_t* starts, uint32_t n, uint32_t* rows) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (uint32_t q = starts[i]; q < starts[i + 1]; ++q) rows[q] = i;
}

// starts[r] = first position whose key is >= r; starts[nrows] = count.
__global__ void k_csr_starts(const uint32_t* keys, uint32_t count, uint32_t nrows, uint32_t* starts) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j <= count; j += gridDim.x * blockDim.x) {
        const uint32_t lo = j == 0 ? 0u : keys[j - 1] + 1u;
        const uint32_t hi = j == count ? nrows : keys[j];
        for (uint32_t r = lo; r <= hi && r <= nrows; ++r) starts[r] = j;
    }
}

__global__ void k_permute_entries(const uint32_t* perm, const float4* in, uint32_t count, float4* out) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x)
        out[j] = in[perm[j]];
}

// F^T entries in cluster order: (row i, weight bits).
__global__ void k_transpose_fill(const uint32_t* perm, const uint32_t* rows, const float* w, uint32_t links,
                                 uint2* out) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < links; j += gridDim.x * blockDim.x) {
        const uint32_t q = perm[j];
        out[j] = make_uint2(rows[q], __float_as_uint(w[q]));
    }
}

__global__ void k_cluster_ids(const uint2* crange, const uint32_t* members, uint32_t nc, uint32_t* cid) {
    for (uint32_t c = blockIdx.x; c < nc; c += gridDim.x)
        for (uint32_t k = crange[c].x + threadIdx.x; k < crange[c].y; k += blockDim.x) cid[members[k]] = c;
}

// ---------------------------------------------------------- adjoint ----
__device__ __forceinline__ V warp_sum(V a) {
    for (int o = 16; o >= 1; o >>= 1) {
        a.x += __shfl_xor_sync(kFull, a.x, o);
        a.y += __shfl_xor_sync(kFull, a.y, o);
        a.z += __shfl_xor_sync(kFull, a.z, o);
    }
    return a;
}

// G^T: warp per surfel, lane-strided over its sorted entries, butterfly sum.
__global__ void __launch_bounds__(256) k_gather_t(const uint32_t* gstarts, const float4* gent, const float* gimg,
                                                  uint32_t n, float4* h) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        V a{0.0f, 0.0f, 0.0f};
        for (uint32_t j = gstarts[i] + lane; j < gstarts[i + 1]; j += 32) {
            const float4 e = gent[j];
            const float* gp = gimg + (size_t)__float_as_uint(e.w) * 3;
            a = a + V{e.x * gp[0], e.y * gp[1], e.z * gp[2]};
        }
        a = warp_sum(a);
        if (lane == 0) h[i] = f4(a, 0.0f);
    }
}

// F^T: CTA per cluster, thread-strided over its links, fixed tree in shared
// memory.
static constexpr int kFtBlock = 256;
__global__ void __launch_bounds__(kFtBlock) k_ft_spmv(const uint32_t* ftstarts, const uint2* ft, const float4* t,
                                                      uint32_t nc, float4* y) {
    __shared__ V red[kFtBlock];
    for (uint32_t c = blockIdx.x; c < nc; c += gridDim.x) {
        V a{0.0f, 0.0f, 0.0f};
        for (uint32_t j = ftstarts[c] + threadIdx.x; j < ftstarts[c + 1]; j += kFtBlock) {
            const uint2 e = ft[j];
            a = a + mk4(t[e.x]) * __uint_as_float(e.y);
        }
        red[threadIdx.x] = a;
        __syncthreads();
        for (int s = kFtBlock / 2; s >= 1; s >>= 1) {
            if ((int)threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) y[c] = f4(red[0], 0.0f);
        __syncthreads();
    }
}

__global__ void k_adj_surfel(const uint32_t* cid, const float4* sp, const float4* cp, const float4* y,
                             const float4* albedo, const float4* irr_prev, uint32_t n, int first, float4* ebar,
                             float4* rhobar, float4* t) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = cid[i];
        V b{0.0f, 0.0f, 0.0f};
        if (c != ~0u) b = mk4(y[c]) * (sp[i].w / fmaxf(cp[c].w, 1e-12f));
        const V eb = first ? b : mk4(ebar[i]) + b;
        ebar[i] = f4(eb, 0.0f);
        if (irr_prev) {
            const V rho = mk4(albedo[i]);
            const V rb = first ? b * mk4(irr_prev[i]) : mk4(rhobar[i]) + b * mk4(irr_prev[i]);
            rhobar[i] = f4(rb, 0.0f);
            t[i] = f4(rho * b, 0.0f);
        } else if (first) {
            rhobar[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
}

// E = rho * S with S = sum_l e_l a_il: rhobar += Ebar * S.
__global__ void k_adj_final(const float4* ebar, const float4* albedo, const float* terms, const float4* emit, int nl,
                            uint32_t n, float4* rhobar) {
    (void)albedo;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        V S{0.0f, 0.0f, 0.0f};
        for (int l = 0; l < nl; ++l) {
            const float a = terms[(size_t)i * nl + l];
            if (a < 0.0f) continue;
            S = S + mk4(emit[l]) * a;
        }
        rhobar[i] = f4(mk4(rhobar[i]) + mk4(ebar[i]) * S, 0.0f);
    }
}

// Emission gradient, stage 1: one CTA per (light, chunk of kEmitChunk
// pixels or surfels), a fixed tree per chunk. Chunks 0..npc-1 are pixels
// (sum_p dpix * g), the rest surfels (sum_i Ebar * rho * a_il).
static constexpr int kRedBlock = 256;
__global__ void __launch_bounds__(kRedBlock) k_emit_partials(const float4* dpix, const float* gimg, uint32_t npix,
                                                             const float4* ebar, const float4* albedo,
                                                             const float* terms, uint32_t n, int nl,
                                                             uint32_t chunks, float* partials) {
    __shared__ V red[kRedBlock];
    const uint32_t npc = (npix + kEmitChunk - 1) / kEmitChunk;
    const int l = (int)blockIdx.y;
    for (uint32_t ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
        V a{0.0f, 0.0f, 0.0f};
        if (ch < npc) {
            const uint32_t e = min(npix, (ch + 1) * kEmitChunk);
            for (uint32_t p = ch * kEmitChunk + threadIdx.x; p < e; p += kRedBlock) {
                const float4 d = dpix[(size_t)l * npix + p];
                const float* gp = gimg + (size_t)p * 3;
                a = a + V{d.x * gp[0], d.y * gp[1], d.z * gp[2]};
            }
        } else {
            const uint32_t c0 = (ch - npc) * kEmitChunk, e = min(n, c0 + kEmitChunk);
            for (uint32_t i = c0 + threadIdx.x; i < e; i += kRedBlock) {
                const float t = terms[(size_t)i * nl + l];
                if (t < 0.0f) continue;
                a = a + mk4(ebar[i]) * mk4(albedo[i]) * t;
            }
        }
        red[threadIdx.x] = a;
        __syncthreads();
        for (int s = kRedBlock / 2; s >= 1; s >>= 1) {
            if ((int)threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            float* o = partials + ((size_t)l * chunks + ch) * 3;
            o[0] = red[0].x;
            o[1] = red[0].y;
            o[2] = red[0].z;
        }
        __syncthreads();
    }
}

// Stage 2: per light, the chunk partials in chunk order.
__global__ void k_emit_finish(const float* partials, uint32_t chunks, int nl, float* out) {
    for (int l = (int)threadIdx.x; l < nl; l += (int)blockDim.x) {
        float a[3] = {0.0f, 0.0f, 0.0f};
        for (uint32_t ch = 0; ch < chunks; ++ch)
            for (int c = 0; c < 3; ++c) a[c] += partials[((size_t)l * chunks + ch) * 3 + c];
        for (int c = 0; c < 3; ++c) out[l * 3 + c] = a[c];
    }
}

__global__ void k_unpack3(const float4* in, uint32_t n, float* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 v = in[i];
        out[3 * (size_t)i] = v.x;
        out[3 * (size_t)i + 1] = v.y;
        out[3 * (size_t)i + 2] = v.z;
    }
}

// ---------------------------------------------------------- launchers ----
int launch_relight(cudaStream_t st, const float4* albedo, const float* terms, const float4* emit, int nl,
                   uint32_t n, float4* direct, float4* rad, float4* irr) {
    k_relight<<<grid_for(n, 256), 256, 0, st>>>(albedo, terms, emit, nl, n, direct, rad, irr);
    return 1;
}

int launch_grid_refresh(cudaStream_t st, const uint32_t* items, const float4* irr, uint32_t n, float4* girr) {
    k_grid_refresh<<<grid_for(n, 256), 256, 0, st>>>(items, irr, n, girr);
    return 1;
}

int launch_diff_pixels(cudaStream_t st, const ShadeParams& p, int pass, float4* dpix, uint32_t* cnt,
                       const uint32_t* off, const uint32_t* gitems, uint32_t* ekey, float4* eval) {
    const size_t sm = blob_smem(p.blob, 128);
    k_diff_pixels<<<grid_for((unsigned long long)p.w * p.h, 128, 16), 128, sm, st>>>(p, pass, dpix, cnt, off, gitems,
                                                                                    ekey, eval);
    return 1;
}

int launch_iota(cudaStream_t st, uint32_t* v, uint32_t n) {
    k_iota<<<grid_for(n, 256), 256, 0, st>>>(v, n);
    return 1;
}

int launch_link_rows(cudaStream_t st, const uint32_t* starts, uint32_t n, uint32_t* rows) {
    k_link_rows<<<grid_for(n, 256), 256, 0, st>>>(starts, n, rows);
    return 1;
}

int launch_csr_starts(cudaStream_t st, const uint32_t* sorted_keys, uint32_t count, uint32_t nrows,
                      uint32_t* starts) {
    k_csr_starts<<<grid_for((unsigned long long)count + 1, 256), 256, 0, st>>>(sorted_keys, count, nrows, starts);
    return 1;
}

int launch_permute_entries(cudaStream_t st, const uint32_t* perm, const float4* in, uint32_t count, float4* out) {
    k_permute_entries<<<grid_for(count, 256), 256, 0, st>>>(perm, in, count, out);
    return 1;
}

int launch_transpose_fill(cudaStream_t st, const uint32_t* perm, const uint32_t* link_rows, const float* w,
                          uint32_t links, uint2* out) {
    k_transpose_fill<<<grid_for(links, 256), 256, 0, st>>>(perm, link_rows, w, links, out);
    return 1;
}

int launch_cluster_ids(cudaStream_t st, const uint2* crange, const uint32_t* members, uint32_t nc, uint32_t* cid) {
    k_cluster_ids<<<nc < 4096u ? nc : 4096u, 128, 0, st>>>(crange, members, nc, cid);
    return 1;
}

int launch_gather_t(cudaStream_t st, const uint32_t* gstarts, const float4* gent, const float* gimg, uint32_t n,
                    float4* h) {
    k_gather_t<<<grid_for((unsigned long long)n * 32, 256), 256, 0, st>>>(gstarts, gent, gimg, n, h);
    return 1;
}

int launch_ft_spmv(cudaStream_t st, const uint32_t* ftstarts, const uint2* ft, const float4* t, uint32_t nc,
                   float4* y) {
    k_ft_spmv<<<nc < 8192u ? nc : 8192u, kFtBlock, 0, st>>>(ftstarts, ft, t, nc, y);
    return 1;
}

int launch_adj_surfel(cudaStream_t st, const uint32_t* cid, const float4* sp, const float4* cp, const float4* y,
                      const float4* albedo, const float4* irr_prev, uint32_t n, int first, float4* ebar,
                      float4* rhobar, float4* t) {
    k_adj_surfel<<<grid_for(n, 256), 256, 0, st>>>(cid, sp, cp, y, albedo, irr_prev, n, first, ebar, rhobar, t);
    return 1;
}

int launch_adj_final(cudaStream_t st, const float4* ebar, const float4* albedo, const float* terms,
                     const float4* emit, int nl, uint32_t n, float4* rhobar) {
    k_adj_final<<<grid_for(n, 256), 256, 0, st>>>(ebar, albedo, terms, emit, nl, n, rhobar);
    return 1;
}

int launch_emit_grad(cudaStream_t st, const float4* dpix, const float* gimg, uint32_t npix, const float4* ebar,
                     const float4* albedo, const float* terms, uint32_t n, int nl, float* partials, float* out) {
    const uint32_t chunks = (npix + kEmitChunk - 1) / kEmitChunk + (n + kEmitChunk - 1) / kEmitChunk;
    dim3 grid(chunks < 1024u ? chunks : 1024u, (unsigned)nl);
    k_emit_partials<<<grid, kRedBlock, 0, st>>>(dpix, gimg, npix, ebar, albedo, terms, n, nl, chunks, partials);
    k_emit_finish<<<1, 32, 0, st>>>(partials, chunks, nl, out);
    return 2;
}

int launch_unpack3(cudaStream_t st, const float4* in, uint32_t n, float* out) {
    k_unpack3<<<grid_for(n, 256), 256, 0, st>>>(in, n, out);
    return 1;
}

void configure_diff_kernels(int max_dyn_smem) {
    cudaFuncSetAttribute(k_diff_pixels, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
}

}  // namespace ifx
