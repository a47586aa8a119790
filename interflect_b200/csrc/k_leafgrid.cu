// The per-cell candidate leaf lists of a scene (layout.h LeafGrid), built
// once per scene upload for the distance-only queries of cone-shadow marches
// (device.cuh dist_fast). No counterpart in the reference, which traverses
// its BVH for every query; the lists only select which leaves a query looks
// at, and dist_fast falls back to the reference traversal whenever its
// answer could differ.
#include "kcommon.cuh"

namespace ifx {

__device__ __forceinline__ void lg_cell(const LeafGrid& g, uint32_t c, uint32_t& x, uint32_t& y, uint32_t& z) {
    x = c % (uint32_t)g.dim[0];
    y = (c / (uint32_t)g.dim[0]) % (uint32_t)g.dim[1];
    z = c / ((uint32_t)g.dim[0] * (uint32_t)g.dim[1]);
}

// U(cell): the reference's distance at the cell centre (scene.rs:191-208)
// plus the cell's half-diagonal: every point of the cell is nearer than U to
// the object nearest its centre, the distance functions being 1-Lipschitz.
__global__ void __launch_bounds__(128) k_lg_bound(BlobRef blob, LeafGrid g, float cell, float half_diag,
                                                  uint32_t ncells, float* U, uint32_t* status) {
    IFX_SCENE_PROLOGUE(blob, status, sv);
    NoCount nc;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) {
        uint32_t x, y, z;
        lg_cell(g, c, x, y, z);
        const V ctr{g.lo[0] + ((float)x + 0.5f) * cell, g.lo[1] + ((float)y + 0.5f) * cell,
                    g.lo[2] + ((float)z + 0.5f) * cell};
        U[c] = dist_mat(sv, ctr, nc).d + half_diag;
    }
}

// Distance in FP64 from a cell, widened by `pad` on every side, to a box.
__device__ __forceinline__ double lg_box_dist(const LeafGrid& g, double cell, double pad, uint32_t x, uint32_t y,
                                              uint32_t z, const DNode& nd) {
    const uint32_t ix[3] = {x, y, z};
    double s = 0.0;
    for (int a = 0; a < 3; ++a) {
        const double clo = (double)g.lo[a] + (double)ix[a] * cell - pad;
        const double chi = (double)g.lo[a] + (double)(ix[a] + 1) * cell + pad;
        const double gap = fmax(0.0, fmax((double)nd.lo[a] - chi, clo - (double)nd.hi[a]));
        s += gap * gap;
    }
    return sqrt(s);
}

// count: the number of listed leaves per cell; fill (start != nullptr): the
// list itself, then ordered by the distance from the cell centre to the
// leaf's box (insertion sort; lists are short).
__global__ void k_lg_lists(const uint8_t* blob, LeafGrid g, double cell, double pad, uint32_t ncells, const float* U,
                           const uint32_t* leaves, uint32_t nleaf, uint32_t* count, const uint32_t* start,
                           uint32_t* out, float* key) {
    const SceneView sv = make_view(blob);
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) {
        uint32_t x, y, z;
        lg_cell(g, c, x, y, z);
        // Inside an object U can be negative while the box holding the point
        // is at distance 0: the bound is taken against 0 at least.
        const double lim = fmax((double)U[c], 0.0) + 2.0 * (double)g.tol;
        uint32_t n = 0;
        const uint32_t o = start ? start[c] : 0u;
        for (uint32_t i = 0; i < nleaf; ++i) {
            const DNode& nd = sv.nodes[leaves[i]];
            if (lg_box_dist(g, cell, pad, x, y, z, nd) < lim) {
                if (start) {
                    // Centre-to-box distance orders the list nearest-first.
                    const double cx[3] = {(double)g.lo[0] + ((double)x + 0.5) * cell,
                                          (double)g.lo[1] + ((double)y + 0.5) * cell,
                                          (double)g.lo[2] + ((double)z + 0.5) * cell};
                    double s = 0.0;
                    for (int a = 0; a < 3; ++a) {
                        const double gap = fmax(0.0, fmax((double)nd.lo[a] - cx[a], cx[a] - (double)nd.hi[a]));
                        s += gap * gap;
                    }
                    const float kv = (float)s;
                    uint32_t j = n;
                    while (j > 0 && key[o + j - 1] > kv) {
                        key[o + j] = key[o + j - 1];
                        out[o + j] = out[o + j - 1];
                        --j;
                    }
                    key[o + j] = kv;
                    out[o + j] = leaves[i];
                }
                ++n;
            }
        }
        if (!start) count[c] = n;
    }
}

void launch_lg_bound(cudaStream_t st, const BlobRef& blob, const LeafGrid& g, float cell, float half_diag,
                     uint32_t ncells, float* U, uint32_t* status) {
    k_lg_bound<<<grid_for(ncells, 128, 16), 128, blob_smem(blob, 128), st>>>(blob, g, cell, half_diag, ncells, U,
                                                                             status);
}

void launch_lg_lists(cudaStream_t st, const uint8_t* blob, const LeafGrid& g, double cell, double pad, uint32_t ncells,
                     const float* U, const uint32_t* leaves, uint32_t nleaf, uint32_t* count, const uint32_t* start,
                     uint32_t* out, float* key) {
    k_lg_lists<<<grid_for(ncells, 128, 16), 128, 0, st>>>(blob, g, cell, pad, ncells, U, leaves, nleaf, count, start,
                                                          out, key);
}

void configure_leafgrid_kernels(int max_dyn_smem) {
    cudaFuncSetAttribute(k_lg_bound, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn_smem);
}

}  // namespace ifx
