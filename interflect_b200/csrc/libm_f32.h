// f32 acos and atan that return glibc's acosf/atanf results bit for bit.
//
// The reference calls Rust's f32::acos (ltc.rs) and the sphere-light
// extension calls atan; on Linux both are the platform libm's float
// functions, which in glibc 2.39 are the fdlibm algorithms (Sun
// Microsystems 1993, float versions by Cygnus). They are restated here from
// that published algorithm (argument reduction, rational or polynomial
// kernel, split constants) in plain IEEE f32 operations, so that, built
// without FMA contraction (the device code is built with --fmad=false, the
// host check with -ffp-contract=off), they give the same float as glibc for
// every input; tests/test_libm_f32.py checks that over every float.
#pragma once

#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define IFX_LM_FN __host__ __device__ __forceinline__
#else
#define IFX_LM_FN inline
#endif

namespace ifx {

IFX_LM_FN float lm_bits(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}
IFX_LM_FN uint32_t lm_word(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

// fdlibm e_acosf: |x| < 0.5 through pi/2 - (x + x*r(x^2)), |x| >= 0.5 through
// 2*asin(sqrt((1-|x|)/2)) with the square root split for the positive side.
IFX_LM_FN float acos_f32(float x) {
    const float pi = lm_bits(0x40490fdau), pio2_hi = lm_bits(0x3fc90fdau), pio2_lo = lm_bits(0x33a22168u);
    const float p0 = lm_bits(0x3e2aaaabu), p1 = lm_bits(0xbea6b090u), p2 = lm_bits(0x3e4e0aa8u),
                p3 = lm_bits(0xbd241146u), p4 = lm_bits(0x3a4f7f04u), p5 = lm_bits(0x3811ef08u);
    const float q1 = lm_bits(0xc019d139u), q2 = lm_bits(0x4001572du), q3 = lm_bits(0xbf303361u),
                q4 = lm_bits(0x3d9dc62eu);
    const uint32_t hx = lm_word(x), ix = hx & 0x7fffffffu;
    if (ix == 0x3f800000u) return (hx >> 31) ? pi + 2.0f * pio2_lo : 0.0f;
    if (ix > 0x3f800000u) return (x - x) / (x - x);
    float z;
    if (ix < 0x3f000000u) {
        if (ix <= 0x32800000u) return pio2_hi + pio2_lo;
        z = x * x;
    } else {
        z = ((hx >> 31) ? (1.0f + x) : (1.0f - x)) * 0.5f;
    }
    const float p = z * (p0 + z * (p1 + z * (p2 + z * (p3 + z * (p4 + z * p5)))));
    const float q = 1.0f + z * (q1 + z * (q2 + z * (q3 + z * q4)));
    const float r = p / q;
    if (ix < 0x3f000000u) return pio2_hi - (x - (pio2_lo - x * r));
    const float s = sqrtf(z);
    if (hx >> 31) return pi - 2.0f * (s + (r * s - pio2_lo));
    const float df = lm_bits(lm_word(s) & 0xfffff000u);
    const float c = (z - df * df) / (s + df);
    return 2.0f * (df + (r * s + c));
}

// fdlibm s_atanf: reduce |x| to [0, 7/16) around the breakpoints 0.5, 1,
// 1.5 and infinity (atan(x) = atan(c) + atan((x - c)/(1 + c*x))), then an
// odd polynomial of degree 23 split into odd and even halves in z = x^2, with
// atan(c) carried as a high and a low part.
IFX_LM_FN float atan_f32(float x) {
    const float atanhi[4] = {4.6364760399e-01f, 7.8539812565e-01f, 9.8279368877e-01f, 1.5707962513e+00f};
    const float atanlo[4] = {5.0121582440e-09f, 3.7748947079e-08f, 3.4473217170e-08f, 7.5497894159e-08f};
    const float aT[11] = {3.3333334327e-01f,  -2.0000000298e-01f, 1.4285714924e-01f,  -1.1111110449e-01f,
                          9.0908870101e-02f,  -7.6918758452e-02f, 6.6610731184e-02f,  -5.8335702866e-02f,
                          4.9768779427e-02f,  -3.6531571299e-02f, 1.6285819933e-02f};
    const uint32_t hx = lm_word(x), ix = hx & 0x7fffffffu;
    int id;
    if (ix >= 0x4c000000u) {  // |x| >= 2^25
        if (ix > 0x7f800000u) return x + x;  // NaN
        return (hx >> 31) ? -atanhi[3] - atanlo[3] : atanhi[3] + atanlo[3];
    }
    if (ix < 0x3ee00000u) {  // |x| < 0.4375
        if (ix < 0x31000000u) return x;  // |x| < 2^-29
        id = -1;
    } else {
        x = fabsf(x);
        if (ix < 0x3f980000u) {    // |x| < 1.1875
            if (ix < 0x3f300000u) {  // 7/16 <= |x| < 11/16
                id = 0;
                x = (2.0f * x - 1.0f) / (2.0f + x);
            } else {  // 11/16 <= |x| < 19/16
                id = 1;
                x = (x - 1.0f) / (x + 1.0f);
            }
        } else {
            if (ix < 0x401c0000u) {  // |x| < 2.4375
                id = 2;
                x = (x - 1.5f) / (1.0f + 1.5f * x);
            } else {  // 2.4375 <= |x| < 2^25
                id = 3;
                x = -1.0f / x;
            }
        }
    }
    const float z = x * x;
    const float w = z * z;
    const float s1 = z * (aT[0] + w * (aT[2] + w * (aT[4] + w * (aT[6] + w * (aT[8] + w * aT[10])))));
    const float s2 = w * (aT[1] + w * (aT[3] + w * (aT[5] + w * (aT[7] + w * aT[9]))));
    if (id < 0) return x - x * (s1 + s2);
    const float r = atanhi[id] - ((x * (s1 + s2) - atanlo[id]) - x);
    return (hx >> 31) ? -r : r;
}

}  // namespace ifx
