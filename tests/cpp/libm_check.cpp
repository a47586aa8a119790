// Checks acos_f32 and atan_f32 (interflect_b200/csrc/libm_f32.h) against the
// platform libm's acosf and atanf on every float (acos: every float in
// [-1, 1] plus the special values). Prints the counts and exits 1 on the
// first disagreement (NaN results agree with NaN).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <thread>
#include <vector>
#include <atomic>

#include "../../interflect_b200/csrc/libm_f32.h"

static bool same(float a, float b) {
    if (std::isnan(a) && std::isnan(b)) return true;
    return ifx::lm_word(a) == ifx::lm_word(b);
}

int main() {
    const unsigned nt = std::thread::hardware_concurrency() ? std::thread::hardware_concurrency() : 1;
    std::atomic<uint64_t> bad_atan{0}, bad_acos{0}, n_acos{0};
    std::atomic<uint32_t> first_atan{0}, first_acos{0};
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t)
        pool.emplace_back([&, t]() {
            uint64_t ba = 0, bc = 0, nc = 0;
            for (uint64_t u = t; u <= 0xffffffffull; u += nt) {
                const float x = ifx::lm_bits((uint32_t)u);
                if (!same(ifx::atan_f32(x), atanf(x))) {
                    if (!ba) first_atan = (uint32_t)u;
                    ++ba;
                }
                if (!(std::fabs(x) <= 1.0f) && !std::isnan(x) && !std::isinf(x)) continue;
                ++nc;
                if (!same(ifx::acos_f32(x), acosf(x))) {
                    if (!bc) first_acos = (uint32_t)u;
                    ++bc;
                }
            }
            bad_atan += ba;
            bad_acos += bc;
            n_acos += nc;
        });
    for (auto& th : pool) th.join();
    std::printf("atan: 4294967296 inputs, %llu differ (first 0x%08x)\n", (unsigned long long)bad_atan.load(),
                first_atan.load());
    std::printf("acos: %llu inputs, %llu differ (first 0x%08x)\n", (unsigned long long)n_acos.load(),
                (unsigned long long)bad_acos.load(), first_acos.load());
    if (bad_atan || bad_acos) return 1;
    std::printf("every input agrees\n");
    return 0;
}
