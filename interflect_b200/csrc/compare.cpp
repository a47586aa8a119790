// `compare a.png b.png [--diff out.png]`: the reference's image comparison
// tool (src/bin/compare.rs) — differing pixels, max and mean absolute error,
// mean Rec.709 luma, and SSIM over 8x8 tiles of the sRGB luma — with the same
// report lines. Host code only.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace ifx_cli {
std::string write_png_rgb8(const std::string& path, const uint8_t* rgb, uint32_t w, uint32_t h);
std::string read_png_rgb8(const std::string& path, uint32_t& w, uint32_t& h, std::vector<uint8_t>& rgb);
}  // namespace ifx_cli

// compare.rs:12-16
static double luma(const uint8_t* p) { return 0.2126 * p[0] + 0.7152 * p[1] + 0.0722 * p[2]; }

// compare.rs:19-66: tiles in row-major order, sums in pixel order.
static double ssim(const std::vector<double>& a, const std::vector<double>& b, size_t w, size_t h) {
    const double C1 = 6.5025, C2 = 58.5225;
    const size_t WIN = 8;
    double total = 0.0;
    size_t n = 0;
    for (size_t y = 0; y + WIN <= h; y += WIN)
        for (size_t x = 0; x + WIN <= w; x += WIN) {
            double ma = 0.0, mb = 0.0;
            for (size_t j = 0; j < WIN; ++j)
                for (size_t i = 0; i < WIN; ++i) {
                    ma += a[(y + j) * w + x + i];
                    mb += b[(y + j) * w + x + i];
                }
            const double cnt = (double)(WIN * WIN);
            ma /= cnt;
            mb /= cnt;
            double va = 0.0, vb = 0.0, cov = 0.0;
            for (size_t j = 0; j < WIN; ++j)
                for (size_t i = 0; i < WIN; ++i) {
                    const double da = a[(y + j) * w + x + i] - ma;
                    const double db = b[(y + j) * w + x + i] - mb;
                    va += da * da;
                    vb += db * db;
                    cov += da * db;
                }
            va /= cnt - 1.0;
            vb /= cnt - 1.0;
            cov /= cnt - 1.0;
            total += ((2.0 * ma * mb + C1) * (2.0 * cov + C2)) / ((ma * ma + mb * mb + C1) * (va + vb + C2));
            ++n;
        }
    return n == 0 ? 1.0 : total / (double)n;
}

int main(int argc, char** argv) {
    std::vector<std::string> a(argv + 1, argv + argc);
    if (a.size() < 2) {
        fprintf(stderr, "usage: compare <a.png> <b.png> [--diff out.png]\n");
        return 2;
    }
    uint32_t w1, h1, w2, h2;
    std::vector<uint8_t> p1, p2;
    std::string e = ifx_cli::read_png_rgb8(a[0], w1, h1, p1);
    if (e.empty()) e = ifx_cli::read_png_rgb8(a[1], w2, h2, p2);
    if (!e.empty()) {
        // The reference panics here ("cannot open ..."); exit status 101 as a Rust panic.
        fprintf(stderr, "cannot open: %s\n", e.c_str());
        return 101;
    }
    if (w1 != w2 || h1 != h2) {
        fprintf(stderr, "size mismatch: %ux%u vs %ux%u\n", w1, h1, w2, h2);
        return 1;
    }
    uint32_t max_err = 0;
    uint64_t sum_err = 0;
    size_t ndiff = 0;
    std::vector<uint8_t> diff(p1.size(), 0);
    for (size_t i = 0; i < p1.size(); i += 3) {
        uint32_t pix_max = 0;
        for (int c = 0; c < 3; ++c) {
            const int d = (int)p1[i + c] - (int)p2[i + c];
            const uint32_t ad = (uint32_t)(d < 0 ? -d : d);
            sum_err += ad;
            pix_max = pix_max > ad ? pix_max : ad;
        }
        if (pix_max > 0) ++ndiff;
        max_err = max_err > pix_max ? max_err : pix_max;
        const uint8_t v = (uint8_t)(pix_max * 8 < 255 ? pix_max * 8 : 255);  // 8x amplified
        diff[i] = diff[i + 1] = diff[i + 2] = v;
    }
    const size_t npx = (size_t)w1 * h1;
    std::vector<double> la(npx), lb(npx);
    for (size_t i = 0; i < npx; ++i) {
        la[i] = luma(&p1[i * 3]);
        lb[i] = luma(&p2[i * 3]);
    }
    const double s = ssim(la, lb, w1, h1);
    double mean_a = 0.0, mean_b = 0.0;
    for (size_t i = 0; i < npx; ++i) mean_a += la[i];
    for (size_t i = 0; i < npx; ++i) mean_b += lb[i];
    mean_a /= (double)npx;
    mean_b /= (double)npx;
    printf("  size          %ux%u  (%zu px)\n", w1, h1, npx);
    printf("  differing px  %zu (%.4f%%)\n", ndiff, 100.0 * (double)ndiff / (double)npx);
    printf("  max abs err   %u / 255\n", max_err);
    printf("  mean abs err  %.5f / 255\n", (double)sum_err / (double)(npx * 3));
    printf("  mean luma     %.2f vs %.2f  (ratio %.3f)\n", mean_a, mean_b, mean_a / mean_b);
    printf("  SSIM          %.6f\n", s);
    for (size_t i = 0; i + 1 < a.size(); ++i)
        if (a[i] == "--diff") {
            if (ifx_cli::write_png_rgb8(a[i + 1], diff.data(), w1, h1).empty())
                printf("  diff map      %s (8x amplified)\n", a[i + 1].c_str());
            break;
        }
    return 0;
}
