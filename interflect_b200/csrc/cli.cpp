// `interflect render <scene.rad> [OPTIONS]` on the GPU: the reference's
// command line (main.rs:68-185) and stage report (main.rs:419-540) over the
// C ABI. `-t` is accepted for compatibility; threads do not apply on the GPU.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/interflect.h"

namespace ifx_cli {
std::string write_png_rgb8(const std::string& path, const uint8_t* rgb, uint32_t w, uint32_t h);
}

namespace {

[[noreturn]] void usage() {
    fprintf(stderr,
            "interflect — noise-free renderer (CUDA, sm_100a)\n\n"
            "USAGE:\n"
            "    interflect render <scene.rad> [OPTIONS]\n\n"
            "OPTIONS:\n"
            "    -o, --output <FILE>    output PNG                  [default: out.png]\n"
            "    -t, --threads <N>      accepted for compatibility (GPU)\n"
            "    -w, --width <N>        override scene width\n"
            "    -h, --height <N>       override scene height\n"
            "        --mode <MODE>      beauty | direct | indirect | normals | depth | steps | reference\n"
            "        --spp <N>          samples/pixel for --mode reference   [default: 512]\n"
            "        --clusters <N>     transfer cluster grid resolution     [default: 8]\n"
            "        --surfels <N>      override surfel count\n"
            "        --bounces <N>      override bounce count\n"
            "        --turntable <N>    render N orbit frames reusing one GI solve\n"
            "        --no-bvh           linear scan; for verifying BVH correctness\n"
            "        --device <N>       CUDA device                   [default: 0]\n");
    exit(2);
}

// Rust's `str::parse::<T>().ok()` for the unsigned overrides: digits only
// (an optional leading '+'), no overflow.
bool parse_u64(const std::string& s, uint64_t& out) {
    size_t i = (!s.empty() && s[0] == '+') ? 1 : 0;
    if (i >= s.size()) return false;
    uint64_t v = 0;
    for (; i < s.size(); ++i) {
        if (s[i] < '0' || s[i] > '9') return false;
        uint64_t d = (uint64_t)(s[i] - '0');
        if (v > (UINT64_MAX - d) / 10) return false;
        v = v * 10 + d;
    }
    out = v;
    return true;
}

bool parse_i32(const std::string& s, int& out) {
    size_t i = (!s.empty() && (s[0] == '+' || s[0] == '-')) ? 1 : 0;
    if (i >= s.size()) return false;
    long long v = 0;
    for (size_t k = i; k < s.size(); ++k) {
        if (s[k] < '0' || s[k] > '9') return false;
        v = v * 10 + (s[k] - '0');
        if (v > 2147483648LL) return false;
    }
    if (s[0] == '-') v = -v;
    if (v > 2147483647LL || v < -2147483648LL) return false;
    out = (int)v;
    return true;
}

double ms_since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

int fail_ctx(ifx_ctx* ctx, const char* what) {
    fprintf(stderr, "error: %s: %s\n", what, ifx_last_error(ctx));
    ifx_ctx_destroy(ctx);
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    std::vector<std::string> a(argv + 1, argv + argc);
    if (a.size() < 2 || a[0] != "render") usage();
    std::string input = a[1], output = "out.png";
    // `--mode reference` is the path tracer (reference.rs), which has its own
    // entry point rather than an ifx_render_frame mode.
    const int kModeReference = -1;
    int mode = IFX_MODE_BEAUTY, cluster_res = 8, device = 0;
    uint32_t spp = 512;
    bool no_bvh = false;
    uint64_t turntable = 0, v = 0;
    bool have_w = false, have_h = false, have_s = false, have_b = false;
    uint64_t ow = 0, oh = 0, os = 0, ob = 0;
    for (size_t i = 2; i < a.size();) {
        auto need = [&]() -> std::string {
            if (i + 1 >= a.size()) usage();
            return a[i + 1];
        };
        const std::string& f = a[i];
        if (f == "-o" || f == "--output") {
            output = need();
            i += 2;
        } else if (f == "-t" || f == "--threads") {
            need();
            i += 2;
        } else if (f == "--spp") {
            uint64_t v2 = 0;
            spp = parse_u64(need(), v2) && v2 >= 1 && v2 <= (1u << 20) ? (uint32_t)v2 : 512u;  // main.rs:150-151; 0 and counts above 2^20 take the default
            i += 2;
        } else if (f == "-w" || f == "--width") {
            have_w = parse_u64(need(), ow) && ow <= 0xffffffffull;
            i += 2;
        } else if (f == "-h" || f == "--height") {
            have_h = parse_u64(need(), oh) && oh <= 0xffffffffull;
            i += 2;
        } else if (f == "--surfels") {
            have_s = parse_u64(need(), os);
            i += 2;
        } else if (f == "--bounces") {
            have_b = parse_u64(need(), ob) && ob <= 0xffffffffull;
            i += 2;
        } else if (f == "--clusters") {
            if (!parse_i32(need(), cluster_res)) cluster_res = 12;  // main.rs:147
            i += 2;
        } else if (f == "--turntable") {
            turntable = parse_u64(need(), v) && v <= 0xffffffffull ? v : 0;
            i += 2;
        } else if (f == "--device") {
            if (!parse_i32(need(), device)) usage();
            i += 2;
        } else if (f == "--mode") {
            std::string m = need();
            if (m == "beauty") mode = IFX_MODE_BEAUTY;
            else if (m == "direct") mode = IFX_MODE_DIRECT;
            else if (m == "indirect") mode = IFX_MODE_INDIRECT;
            else if (m == "normals") mode = IFX_MODE_NORMALS;
            else if (m == "depth") mode = IFX_MODE_DEPTH;
            else if (m == "steps") mode = IFX_MODE_STEPS;
            else if (m == "reference") mode = kModeReference;
            else {
                fprintf(stderr, "unknown mode `%s`\n", m.c_str());
                usage();
            }
            i += 2;
        } else if (f == "--no-bvh") {
            no_bvh = true;
            i += 1;
        } else {
            fprintf(stderr, "unknown flag `%s`\n", f.c_str());
            usage();
        }
    }

    std::ifstream in(input, std::ios::binary);
    if (!in) {
        fprintf(stderr, "error: cannot read %s: %s\n", input.c_str(), strerror(errno));
        return 1;
    }
    std::stringstream ss;
    ss << in.rdbuf();
    std::string src = ss.str();
    char err[512];
    ifx_scene* scene = nullptr;
    if (ifx_scene_parse(src.data(), src.size(), &scene, err, sizeof err) != IFX_OK) {
        fprintf(stderr, "error: %s: %s\n", input.c_str(), err);
        return 1;
    }
    ifx_scene_set_use_bvh(scene, no_bvh ? 0 : 1);
    ifx_scene_info info;
    ifx_scene_get_info(scene, &info);
    ifx_render_cfg cfg = info.cfg;
    if (have_w) cfg.width = (uint32_t)ow;
    if (have_h) cfg.height = (uint32_t)oh;
    if (have_s) cfg.surfels = os;
    if (have_b) cfg.bounces = (uint32_t)ob;
    if (ifx_scene_set_cfg(scene, &cfg, err, sizeof err) != IFX_OK) {
        fprintf(stderr, "error: %s\n", err);
        ifx_scene_free(scene);
        return 1;
    }
    if (cluster_res < 1 || cluster_res > 512) {
        fprintf(stderr, "error: --clusters must be in 1..512, got %d\n", cluster_res);
        ifx_scene_free(scene);
        return 1;
    }
    const uint32_t w = cfg.width, h = cfg.height;
    ifx_ctx* ctx = nullptr;
    if (ifx_ctx_create(device, &ctx) != IFX_OK) {
        fprintf(stderr, "error: no usable CUDA device %d\n", device);
        ifx_scene_free(scene);
        return 1;
    }
    printf("interflect 0.1.3 (interflect-b200, CUDA sm_100a)\n");
    printf("  scene      %u objects, %u lights, %u materials, %u bvh nodes\n", info.objects + info.planes,
           info.lights + info.sphere_lights, info.materials, info.bvh_nodes);
    printf("  film       %ux%u\n", w, h);
    if (ifx_scene_upload(ctx, scene) != IFX_OK) return fail_ctx(ctx, "scene upload");

    auto t_gi = std::chrono::steady_clock::now();
    const bool needs_gi = mode == IFX_MODE_BEAUTY || mode == IFX_MODE_INDIRECT;
    if (needs_gi) {
        auto t = std::chrono::steady_clock::now();
        uint64_t placed = 0;
        if (ifx_surfels_generate(ctx, cfg.surfels, &placed) != IFX_OK) return fail_ctx(ctx, "surfels");
        if (placed == 0) {
            fprintf(stderr, "error: no surfels generated — scene may have no surface inside its bounds\n");
            ifx_ctx_destroy(ctx);
            return 1;
        }
        printf("  surfels    %llu placed of %llu requested   (%.0f ms)\n", (unsigned long long)placed,
               (unsigned long long)cfg.surfels, ms_since(t));
        t = std::chrono::steady_clock::now();
        ifx_transfer_info ti;
        if (ifx_transfer_build(ctx, cluster_res, &ti) != IFX_OK) return fail_ctx(ctx, "transfer");
        printf("  transfer   %llu clusters, %llu links, row-sum %.3f, %.1fM sdf evals   (%.0f ms)\n",
               (unsigned long long)ti.clusters, (unsigned long long)ti.links, (double)ti.mean_row_sum,
               (double)ti.evals / 1e6, ms_since(t));
        t = std::chrono::steady_clock::now();
        uint64_t de = 0;
        ifx_solve_stats st;
        if (ifx_light_surfels(ctx, &de) != IFX_OK) return fail_ctx(ctx, "light_surfels");
        if (ifx_solve(ctx, cfg.bounces, &st) != IFX_OK) return fail_ctx(ctx, "solve");
        printf("  solve      %u bounces, residual %.2e, %.1fM sdf evals   (%.0f ms)\n", st.iterations,
               (double)st.residual, (double)de / 1e6, ms_since(t));
        if (ifx_grid_build(ctx, 0.0f) != IFX_OK) return fail_ctx(ctx, "grid");
    }
    const double gi_ms = ms_since(t_gi);

    std::vector<uint8_t> rgb((size_t)w * h * 3);
    if (turntable > 0) {
        // main.rs:492-520: orbit the camera about its look point.
        const float tau = 6.28318530717958647692f;
        float base[3] = {info.camera.pos[0] - info.camera.look[0], info.camera.pos[1] - info.camera.look[1],
                         info.camera.pos[2] - info.camera.look[2]};
        auto t0 = std::chrono::steady_clock::now();
        for (uint64_t i = 0; i < turntable; ++i) {
            float ang = tau * (float)i / (float)turntable;
            float s = std::sin(ang), co = std::cos(ang);
            ifx_camera cam = info.camera;
            cam.pos[0] = info.camera.look[0] + (base[0] * co - base[2] * s);
            cam.pos[1] = info.camera.look[1] + base[1];
            cam.pos[2] = info.camera.look[2] + (base[0] * s + base[2] * co);
            const int rc = mode == kModeReference
                               ? ifx_render_reference(ctx, &cam, w, h, spp, cfg.exposure, nullptr, rgb.data())
                               : ifx_render_frame(ctx, &cam, mode, w, h, cfg.exposure, nullptr, rgb.data(), nullptr);
            if (rc != IFX_OK) return fail_ctx(ctx, "render");
            std::string stem = output;
            if (stem.size() >= 4 && stem.compare(stem.size() - 4, 4, ".png") == 0) stem.resize(stem.size() - 4);
            char name[64];
            snprintf(name, sizeof name, "_%03llu.png", (unsigned long long)i);
            std::string e = ifx_cli::write_png_rgb8(stem + name, rgb.data(), w, h);
            if (!e.empty()) {
                fprintf(stderr, "error: %s\n", e.c_str());
                ifx_ctx_destroy(ctx);
                return 1;
            }
        }
        double ms = ms_since(t0);
        printf("  turntable  %llu frames in %.0f ms  (%.0f ms/frame, GI solved once in %.0f ms)\n",
               (unsigned long long)turntable, ms, ms / (double)turntable, gi_ms);
        ifx_ctx_destroy(ctx);
        ifx_scene_free(scene);
        return 0;
    }
    auto t0 = std::chrono::steady_clock::now();
    uint64_t evals = 0;  // the path tracer counts no evaluations (main.rs:249-258)
    const int rc = mode == kModeReference
                       ? ifx_render_reference(ctx, nullptr, w, h, spp, cfg.exposure, nullptr, rgb.data())
                       : ifx_render_frame(ctx, nullptr, mode, w, h, cfg.exposure, nullptr, rgb.data(), &evals);
    if (rc != IFX_OK) return fail_ctx(ctx, "render");
    double ms = ms_since(t0);
    double px = (double)w * (double)h;
    printf("  shade      %.0f ms   %.1fM sdf evals   %.0f evals/px\n", ms, (double)evals / 1e6, (double)evals / px);
    printf("  total      %.0f ms\n", gi_ms + ms);
    std::string e = ifx_cli::write_png_rgb8(output, rgb.data(), w, h);
    if (!e.empty()) {
        fprintf(stderr, "error: %s\n", e.c_str());
        ifx_ctx_destroy(ctx);
        return 1;
    }
    printf("  wrote      %s\n", output.c_str());
    ifx_ctx_destroy(ctx);
    ifx_scene_free(scene);
    return 0;
}
