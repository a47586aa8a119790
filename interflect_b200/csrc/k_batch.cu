// Batched relighting: R right-hand sides (emission vectors E^(r)) solved
// on one transfer matrix, the Jacobi bounce of solve.rs:47-108 as a CSR
// SpMM. Vectors are stored surfel-major with the R right-hand sides
// innermost (x[i * R + r], one float4 each), so a warp's lanes are 32
// right-hand sides of the same row: every load of a link's cluster value is
// one coalesced 512-byte access, and the link index and weight are
// warp-uniform. Each (row, rhs) accumulates its links in CSR order and each
// (cluster, rhs) its members in member order, exactly as the single-RHS
// kernels do, so every right-hand side is bit-identical to its own solve.
// Per-RHS done flags freeze a right-hand side at the bounce where its own
// residual fell below 1e-4 (solve.rs:99).
#include "kcommon.cuh"

namespace ifx {

// solve.rs:61-73 for every rhs: warp per (cluster, 32 rhs).
__global__ void __launch_bounds__(256) k_agg_batched(const float4* rad, const float4* sp, const float4* cp,
                                                      const uint2* crange, const uint32_t* members, uint32_t nc,
                                                      uint32_t R, float4* crad, const uint32_t* done) {
    const int lane = threadIdx.x & 31;
    const uint32_t chunks = (R + 31) / 32;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nc * chunks; t += warps) {
        const uint32_t c = t / chunks, r = (t % chunks) * 32 + lane;
        if (r >= R || done[r]) continue;
        const uint2 rg = crange[c];
        V acc{0.0f, 0.0f, 0.0f};
        for (uint32_t k = rg.x; k < rg.y; ++k) {
            const uint32_t m = __ldg(&members[k]);
            const float a = __ldg(&sp[m].w);
            acc = acc + mk4(rad[(size_t)m * R + r]) * a;
        }
        crad[(size_t)c * R + r] = f4(acc / fmaxf(cp[c].w, 1e-12f), 0.0f);
    }
}

// solve.rs:76-102 for every rhs: blockIdx.y picks 32 rhs, warps stride over
// rows; a lane keeps its rhs for the whole kernel and reduces its residual
// to one integer atomicMax at the end.
__global__ void __launch_bounds__(512) k_spmm(const float4* direct, const float4* albedo, float4* irr, float4* rad,
                                               uint32_t n, uint32_t R, const uint32_t* starts, const uint32_t* idx,
                                               const float* w, const float4* crad, const uint32_t* done,
                                               uint32_t* res_bits) {
    const int lane = threadIdx.x & 31;
    const uint32_t r = blockIdx.y * 32 + lane;
    const bool live = r < R && !done[r];
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    float dmax = 0.0f;
    if (live) {
        for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
            V acc{0.0f, 0.0f, 0.0f};
            const uint32_t e = starts[i + 1];
            for (uint32_t k = starts[i]; k < e; ++k)
                acc = acc + mk4(crad[(size_t)__ldg(&idx[k]) * R + r]) * __ldg(&w[k]);
            const size_t o = (size_t)i * R + r;
            const V nr = mk4(direct[o]) + mk4(__ldg(&albedo[i])) * acc;
            const V diff = vabs(nr - mk4(rad[o]));
            const float d = fmaxf(diff.x, fmaxf(diff.y, diff.z));
            irr[o] = f4(acc, 0.0f);
            rad[o] = f4(nr, 0.0f);
            if (!isnan(d)) dmax = fmaxf(dmax, d);
        }
        if (dmax > 0.0f) atomicMax(&res_bits[r], __float_as_uint(dmax));
    }
}

// solve.rs:93-101 per rhs.
__global__ void k_bounce_end_batched(uint32_t R, uint32_t it, uint32_t* done, uint32_t* iterations,
                                     uint32_t* res_bits, uint32_t* last_res) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < R; r += gridDim.x * blockDim.x) {
        if (done[r]) continue;
        const float res = __uint_as_float(res_bits[r]);
        iterations[r] = it + 1;
        last_res[r] = res_bits[r];
        res_bits[r] = 0;
        if (res < 1e-4f) done[r] = 1;
    }
}

// E (R x n x 3 f32, rhs-major on the host side) -> direct = rad = E, irr = 0
// in the interleaved layout.
__global__ void k_batch_init(const float* E, uint32_t n, uint32_t R, float4* direct, float4* rad, float4* irr) {
    const size_t total = (size_t)n * R;
    for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < total; o += (size_t)gridDim.x * blockDim.x) {
        const size_t i = o / R, r = o % R;
        const float* e = E + (r * n + i) * 3;
        const float4 v = make_float4(e[0], e[1], e[2], 0.0f);
        direct[o] = v;
        rad[o] = v;
        irr[o] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

// Interleaved float4 -> rhs-major packed xyz.
__global__ void k_batch_unpack(const float4* x, uint32_t n, uint32_t R, float* out) {
    const size_t total = (size_t)n * R;
    for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < total; o += (size_t)gridDim.x * blockDim.x) {
        const size_t i = o / R, r = o % R;
        const float4 v = x[o];
        float* d = out + (r * n + i) * 3;
        d[0] = v.x;
        d[1] = v.y;
        d[2] = v.z;
    }
}

int launch_batch_init(cudaStream_t st, const float* E, uint32_t n, uint32_t R, float4* direct, float4* rad,
                      float4* irr) {
    k_batch_init<<<grid_for((unsigned long long)n * R, 256), 256, 0, st>>>(E, n, R, direct, rad, irr);
    return 1;
}

int launch_batch_unpack(cudaStream_t st, const float4* x, uint32_t n, uint32_t R, float* out) {
    k_batch_unpack<<<grid_for((unsigned long long)n * R, 256), 256, 0, st>>>(x, n, R, out);
    return 1;
}

int launch_batched_bounce(cudaStream_t st, uint32_t n, uint32_t R, const float4* sp, const float4* albedo,
                          const float4* direct, float4* irr, float4* rad, const float4* cp, const uint2* crange,
                          const uint32_t* members, uint32_t nc, const uint32_t* starts, const uint32_t* idx,
                          const float* w, float4* crad, uint32_t* done, uint32_t* iterations, uint32_t* res_bits,
                          uint32_t* last_res, uint32_t it, int rows_per_block_warps) {
    const uint32_t chunks = (R + 31) / 32;
    k_agg_batched<<<grid_for((unsigned long long)nc * chunks * 32ull, 256), 256, 0, st>>>(rad, sp, cp, crange,
                                                                                          members, nc, R, crad, done);
    const int block = 32 * rows_per_block_warps;
    unsigned gx = grid_for((unsigned long long)n * 32ull, block, 4);
    if (gx * chunks > 65535u * 64u) gx = (65535u * 64u) / chunks;
    dim3 grid(gx, chunks);
    k_spmm<<<grid, block, 0, st>>>(direct, albedo, irr, rad, n, R, starts, idx, w, crad, done, res_bits);
    k_bounce_end_batched<<<grid_for(R, 256), 256, 0, st>>>(R, it, done, iterations, res_bits, last_res);
    return 3;
}

}  // namespace ifx
