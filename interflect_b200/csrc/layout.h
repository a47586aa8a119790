// Device data layout shared by the host flattener and the CUDA kernels.
//
// A scene becomes one contiguous, 16-byte aligned "program" blob that every
// tracing kernel copies into shared memory once per CTA (one bulk copy):
//
//   BlobHeader                      64 B
//   DObject[n_planes + n_objects]   16 B each: planes first, then the
//                                   bounded objects in BVH leaf order
//   DPrim[n_prims]                  64 B each: an object's base primitive
//                                   followed by its subtracted primitives
//   DNode[n_nodes]                  32 B each: flattened BVH, left child = i+1
//   DQuadLight[n_lights]           160 B each
//   DSphereLight[n_sphere_lights]   32 B each
//   DMaterial[n_materials]          64 B each (index 0 = default material)
//   uint32 linear_order[n_objects]  stored index of each object in parse
//                                   order, for the --no-bvh linear scan
//
// Every p-independent subexpression of a primitive's distance function is
// evaluated once on the host with the same f32 operations the per-point code
// would use (for example b - splat(r) of a rounded box, dot(ba, ba) of a
// capsule), so hoisting it does not change a single bit of the result.
#pragma once

#include <stdint.h>

namespace ifx {

enum PrimKind : int32_t {
    K_SPHERE = 0,    // v: c.xyz, r
    K_BOX = 1,       // v: c.xyz, (b - r).xyz, r, [rot] cos, sin
    K_PLANE = 2,     // v: n.xyz, h
    K_CAPSULE = 3,   // v: a.xyz, ba.xyz, dot(ba,ba), r
    K_TORUS = 4,     // v: c.xyz, major, minor
    K_CYLINDER = 5,  // v: a.xyz, ba.xyz, baba, r, r*baba, baba*0.5
    K_CONE = 6,      // v: a.xyz, ba.xyz, baba, ra, rb, rb-ra, (rb-ra)^2+baba
    K_BOX_ROT = 7,   // K_BOX rotated about +y (extension)
};
static const int N_PRIM_KINDS = 8;

// Device status bit of the bounds-checked build (IFX_CHECKED): a checked
// index was out of range.
static const uint32_t kStatusBounds = 1u << 7;

struct alignas(16) DPrim {
    int32_t kind;
    int32_t pad[3];
    float v[12];
};

struct alignas(16) DObject {
    int32_t prim;    // index of the base primitive in the DPrim array
    int32_t nsub;    // subtracted primitives follow the base primitive
    uint32_t mat;
    float smooth;    // smooth-subtraction radius (extension); 0 = max(d, -s)
};

struct alignas(16) DNode {
    float lo[3];
    int32_t count;   // > 0: leaf with `count` objects starting at `link`
    float hi[3];
    int32_t link;    // leaf: first stored object; interior: right child
};

struct alignas(16) DQuadLight {
    float v[4][4];       // vertices (w unused)
    float center[4];     // (v0+v1+v2+v3)*0.25, w = cone radius max(sqrt(area/pi), 1e-4)
    float normal[4];     // normalize(cross(v1-v0, v3-v0)), w = area
    float emit[4];
    float e1[4];         // v1 - v0, w = dot(e1, e1)
    float e2[4];         // v3 - v0, w = dot(e2, e2)
    float ncross[4];     // cross(e1, e2) (unnormalised)
};

struct alignas(16) DSphereLight {
    float c[4];          // centre, w = radius
    float emit[4];
};

struct alignas(16) DMaterial {
    float albedo[4];     // w = roughness
    float emissive[4];   // w = metallic
    float kd[4];         // albedo * (1 - metallic), w = alpha = max(roughness^2, 1e-3)
    float f0[4];         // lerp(0.04, albedo, metallic), w = 1 if a mirror ray is traced
};

struct alignas(16) BlobHeader {
    int32_t n_planes, n_objects, n_prims, n_nodes;
    int32_t n_lights, n_sphere_lights, n_materials, use_bvh;
    uint32_t off_objects, off_prims, off_nodes, off_lights;
    uint32_t off_sphere_lights, off_materials, off_linear, total_bytes;
};

// Candidate leaves per cell of a uniform grid over the scene, used by the
// distance-only queries of cone-shadow marches in large BVHs (device.cuh,
// dist_fast). A cell lists every BVH leaf whose box comes within
// U(cell) + 2 tol of the cell, U(cell) being the reference's distance at the
// cell centre plus the cell's half-diagonal (an upper bound of the nearest
// distance anywhere in the cell); leaves appear nearest-first.
struct LeafGrid {
    const uint32_t* start;  // per cell: first entry of its list; start[ncells] = total
    const uint32_t* leaf;   // BVH node index of each listed leaf
    float lo[3];
    float inv_cell;
    int dim[3];
    float tol;              // pruning margin, far above any f32 rounding of the distances
    int enabled;
};

// Per-scene scalars passed to kernels by value.
struct SceneConsts {
    float lo[3], hi[3];
    float diag;
    float closure[16][3];  // hemisphere_closure's fixed direction coefficients
};

#ifdef __CUDACC__
__host__ __device__
#endif
static inline uint32_t align16(uint32_t x) { return (x + 15u) & ~15u; }

}  // namespace ifx
