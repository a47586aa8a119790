// Algorithmic FLOP model of the tracing kernels.
//
// Each counted work item (device.cuh CounterId) is charged the f32
// operations its code performs, counting add, sub, mul, div, sqrt, min, max,
// abs and neg as one FLOP each and comparisons as none. The SDF rows (node
// tests, primitive distances, subtractions, march steps) are exact counts of
// the expressions in device.cuh; the shading rows (form factor, light,
// specular, gather) are the counts of their straight-line paths and ignore
// rarely taken branches (horizon clipping), so they are within a few FLOPs.
#pragma once

#include <cstdint>

namespace ifx {

static const double kFlopsPerItem[21] = {
    18,  // CN_NODE: (lo-p), (p-hi), 2 x max, dot, sqrt
    10,  // CN_PRIM + K_SPHERE
    23,  // CN_PRIM + K_BOX
    6,   // CN_PRIM + K_PLANE
    24,  // CN_PRIM + K_CAPSULE
    13,  // CN_PRIM + K_TORUS
    38,  // CN_PRIM + K_CYLINDER
    46,  // CN_PRIM + K_CONE
    29,  // CN_PRIM + K_BOX_ROT
    15,  // CN_SMOOTH
    2,   // CN_HARD
    0,   // CN_SDF (the query's work is in the node and primitive rows)
    9,   // CN_TSTEP: p = ro + rd*t, eps, t += d
    22,  // CN_SSTEP: p, closest-approach correction, penumbra update, clamped step
    86,  // CN_FF: to_local of 4 vertices and the horizon clip
    64,  // CN_FF_EDGE: vertex normalisation, dot, clamp, acos, cross, length, accumulate
    33,  // CN_LIGHT: cone parameters, shadow origin, diffuse accumulation
    173, // CN_SPEC: mirror direction, representative point, GGX D, Smith V, Schlick F
    8,   // CN_GVISIT: distance test
    16,  // CN_GACCEPT: alignment, weight, accumulation
    0,   // reserved
};

static inline double work_flops(const unsigned long long* counts, int n) {
    double f = 0.0;
    for (int i = 0; i < n && i < 21; ++i) f += kFlopsPerItem[i] * (double)counts[i];
    return f;
}

}  // namespace ifx
