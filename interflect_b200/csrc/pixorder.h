// The order in which the shading passes take pixels: 8 x 4 tiles (one warp's
// worth of neighbouring camera rays) over the largest tiled part of the film,
// row by row of tiles, then the pixels of the right strip and of the bottom
// rows in row order. A bijection of [0, w*h); every result is still written
// to its own pixel, so the order changes only which rays share a warp.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define IFX_PX_FN __host__ __device__ __forceinline__
#else
#define IFX_PX_FN inline
#endif

namespace ifx {

IFX_PX_FN uint32_t tile_pixel(uint32_t t, uint32_t w, uint32_t h) {
    const uint32_t w8 = w & ~7u, h4 = h & ~3u;
    const uint32_t main = w8 * h4;
    if (t < main) {
        const uint32_t tile = t >> 5, in = t & 31u, tiles_x = w8 >> 3;
        const uint32_t x = (tile % tiles_x) * 8u + (in & 7u), y = (tile / tiles_x) * 4u + (in >> 3);
        return y * w + x;
    }
    const uint32_t r = t - main, rw = w - w8;
    if (r < h4 * rw) return (r / rw) * w + w8 + r % rw;
    return h4 * w + (r - h4 * rw);
}

}  // namespace ifx
