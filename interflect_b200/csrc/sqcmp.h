// Comparisons of correctly rounded square roots from the squares.
//
// The BVH query (bvh.rs:100-150) only ever compares box distances:
// sqrtf(s) >= best (prune) and sqrtf(a) < sqrtf(b) (near child first).
// sqrtf is correctly rounded and monotone, so both outcomes follow from the
// squares whenever the squares are more than a relative 2^-20 apart: the
// margin exceeds every rounding step involved (products rounded to within
// 2^-24, square roots to within 2^-24), so e.g. s >= fl(fl(b*b)*(1+2^-20))
// implies sqrt(s) > b*(1+2^-23) and hence sqrtf(s) > b. Inside the band,
// for tiny operands (where b*b is not a normal float) and for NaN, the square
// roots are taken. Results are therefore exactly those of comparing
// sqrtf(.) values; the square roots are skipped in almost every case.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define IFX_SQ_FN __host__ __device__ __forceinline__
#else
#define IFX_SQ_FN inline
#endif

namespace ifx {

// sqrtf(a) < sqrtf(b) for squared distances a, b (>= 0 or NaN).
IFX_SQ_FN bool sq_lt(float a, float b) {
    if (!(a < b)) return false;  // includes NaN; sqrtf is monotone
    if (b >= 0x1p-100f && a <= b * (1.0f - 0x1p-20f)) return true;
    return sqrtf(a) < sqrtf(b);
}

// sqrtf(s) >= b for a squared distance s (>= 0 or NaN) and any b.
IFX_SQ_FN bool sq_ge(float s, float b) {
    if (b <= 0.0f) return s >= 0.0f;  // sqrtf(s) >= 0 >= b unless s is NaN
    if (b >= 0x1p-60f) {
        const float bb = b * b;
        if (s >= bb * (1.0f + 0x1p-20f)) return true;
        if (s <= bb * (1.0f - 0x1p-20f)) return false;
    }
    return sqrtf(s) >= b;
}

}  // namespace ifx
