// Checks sq_lt / sq_ge (interflect_b200/csrc/sqcmp.h) against comparing the
// square roots directly, on random, adversarial and special operands.
// Prints the number of cases and exits 1 on the first disagreement.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>

#include "../../interflect_b200/csrc/sqcmp.h"

static uint64_t st = 0x9E3779B97F4A7C15ull;
static uint64_t next() {
    st ^= st << 13;
    st ^= st >> 7;
    st ^= st << 17;
    return st;
}
static float bits(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
static float any_float() { return bits((uint32_t)next()); }
static float nonneg() { return std::fabs(bits((uint32_t)next() & 0x7fffffffu)); }

static uint64_t n = 0;
static bool check(float a, float b) {
    ++n;
    if (!std::isnan(a) && a < 0.0f) a = -a;  // the squared operands are never negative
    const bool lt = ifx::sq_lt(a, b), lt_ref = std::sqrt(a) < std::sqrt(std::fabs(b));
    bool ok = true;
    if (!(b < 0.0f) && lt != lt_ref) ok = false;
    const bool ge = ifx::sq_ge(a, b), ge_ref = std::sqrt(a) >= b;
    if (ge != ge_ref) ok = false;
    if (!ok) printf("mismatch a=%a b=%a lt=%d/%d ge=%d/%d\n", a, b, lt, lt_ref, ge, ge_ref);
    return ok;
}

int main() {
    const float special[] = {0.0f, -0.0f, 1.0f, -1.0f, 0x1p-149f, 0x1p-126f, 0x1p-100f, 0x1p-60f, 0x1p-61f,
                             std::numeric_limits<float>::max(), std::numeric_limits<float>::infinity(),
                             -std::numeric_limits<float>::infinity(), std::numeric_limits<float>::quiet_NaN(),
                             1e-30f, 1e30f, 3.0f, 4.0f};
    for (float a : special)
        for (float b : special)
            if (!check(a, b)) return 1;
    for (int i = 0; i < 20000000; ++i) {
        // Random operands over the whole range.
        if (!check(nonneg(), any_float())) return 1;
        // The same square and a value near its root, a few ulps either way.
        float s = nonneg();
        float r = std::sqrt(s);
        int k = (int)(next() % 9) - 4;
        float b = r;
        for (int j = 0; j < (k < 0 ? -k : k); ++j) b = std::nextafter(b, k < 0 ? 0.0f : 1e38f);
        if (!check(s, b)) return 1;
        // Nearby squares: a within a few ulps of b.
        float a = s;
        int m = (int)(next() % 9) - 4;
        for (int j = 0; j < (m < 0 ? -m : m); ++j) a = std::nextafter(a, m < 0 ? 0.0f : 1e38f);
        if (!check(a, s)) return 1;
        // Squares straddling the 2^-20 band.
        float c = s * (1.0f - 0x1p-20f);
        for (int j = 0; j < 3; ++j) c = std::nextafter(c, (next() & 1) ? 0.0f : 1e38f);
        if (!check(c, s)) return 1;
        if (!check(c, r)) return 1;
    }
    printf("%llu cases agree\n", (unsigned long long)n);
    return 0;
}
