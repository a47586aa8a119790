// tile_pixel (interflect_b200/csrc/pixorder.h) is a permutation of [0, w*h)
// for film sizes with and without partial tiles.
#include <cstdio>
#include <vector>

#include "../../interflect_b200/csrc/pixorder.h"

int main() {
    const unsigned sizes[][2] = {{1, 1}, {7, 3}, {8, 4}, {17, 3}, {3, 17}, {129, 1}, {1, 65}, {640, 360},
                                 {1920, 1080}, {33, 9}, {300, 300}, {8, 5}, {9, 4}};
    unsigned long long checked = 0;
    for (auto& s : sizes) {
        const unsigned w = s[0], h = s[1];
        std::vector<unsigned char> seen((size_t)w * h, 0);
        for (unsigned t = 0; t < w * h; ++t) {
            const unsigned p = ifx::tile_pixel(t, w, h);
            if (p >= w * h || seen[p]) {
                printf("not a permutation at %ux%u, t=%u -> %u\n", w, h, t, p);
                return 1;
            }
            seen[p] = 1;
            ++checked;
        }
    }
    printf("%llu pixels checked, permutation\n", checked);
    return 0;
}
