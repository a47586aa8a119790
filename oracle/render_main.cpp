// Oracle (test infrastructure only): a command-line driver over the oracle
// that prints the reference's stage report lines (main.rs:419-471,528-534),
// used to pin the restatement against the reference's published counts.
//
//   oracle_render <scene.rad> [-t threads] [-w W] [-h H] [--surfels N]
//                 [--bounces N] [--clusters N] [--mode M] [--no-bvh] [-o out.ppm]
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "oracle.h"

using namespace orc;

static double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

int main(int argc, char** argv) {
    if (argc < 2) {
        fprintf(stderr, "usage: oracle_render <scene.rad> [options]\n");
        return 2;
    }
    std::string input = argv[1], output;
    int threads = 1, cluster_res = 8;
    long width = -1, height = -1, surfels = -1, bounces = -1;
    int32_t mode = M_BEAUTY;
    bool no_bvh = false;
    for (int i = 2; i < argc; ++i) {
        std::string a = argv[i];
        auto need = [&]() -> const char* {
            if (i + 1 >= argc) {
                fprintf(stderr, "missing value for %s\n", a.c_str());
                exit(2);
            }
            return argv[++i];
        };
        if (a == "-t") threads = atoi(need());
        else if (a == "-w") width = atol(need());
        else if (a == "-h") height = atol(need());
        else if (a == "--surfels") surfels = atol(need());
        else if (a == "--bounces") bounces = atol(need());
        else if (a == "--clusters") cluster_res = atoi(need());
        else if (a == "-o") output = need();
        else if (a == "--no-bvh") no_bvh = true;
        else if (a == "--mode") {
            std::string m = need();
            if (m == "beauty") mode = M_BEAUTY;
            else if (m == "direct") mode = M_DIRECT;
            else if (m == "indirect") mode = M_INDIRECT;
            else if (m == "normals") mode = M_NORMALS;
            else if (m == "depth") mode = M_DEPTH;
            else if (m == "steps") mode = M_STEPS;
            else {
                fprintf(stderr, "unknown mode `%s`\n", m.c_str());
                return 2;
            }
        } else {
            fprintf(stderr, "unknown flag `%s`\n", a.c_str());
            return 2;
        }
    }
    std::ifstream f(input);
    if (!f) {
        fprintf(stderr, "error: cannot read %s\n", input.c_str());
        return 1;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    Scene sc;
    std::string err;
    if (!parse_scene(ss.str(), sc, err)) {
        fprintf(stderr, "error: %s: %s\n", input.c_str(), err.c_str());
        return 1;
    }
    sc.use_bvh = !no_bvh;
    if (width >= 0) sc.cfg.width = (uint32_t)width;
    if (height >= 0) sc.cfg.height = (uint32_t)height;
    if (surfels >= 0) sc.cfg.surfels = (uint64_t)surfels;
    if (bounces >= 0) sc.cfg.bounces = (uint32_t)bounces;
    if (!sc.cfg.validate(err)) {
        fprintf(stderr, "error: %s\n", err.c_str());
        return 1;
    }
    uint32_t w = sc.cfg.width, h = sc.cfg.height;
    float diag = sc.diag();
    float tmax = diag * 4.0f;
    printf("oracle (interflect 0.1.3 restatement)\n");
    printf("  scene      %zu objects, %zu lights, %zu materials, %zu bvh nodes\n",
           sc.objects.size() + sc.planes.size(), sc.lights.size() + sc.sphere_lights.size(),
           sc.materials.size() - 1, sc.bvh.nodes.size());
    printf("  film       %ux%u\n", w, h);
    auto t_gi = std::chrono::steady_clock::now();
    Surfels s;
    Transfer tr;
    Grid grid;
    float radius = 0.0f;
    bool needs_gi = (mode == M_BEAUTY || mode == M_INDIRECT);
    if (needs_gi) {
        auto t = std::chrono::steady_clock::now();
        generate(sc, sc.cfg.surfels, s);
        double gen_ms = ms_since(t);
        if (s.size() == 0) {
            fprintf(stderr, "error: no surfels generated\n");
            return 1;
        }
        printf("  surfels    %zu placed of %llu requested   (%.0f ms)\n", s.size(),
               (unsigned long long)sc.cfg.surfels, gen_ms);
        t = std::chrono::steady_clock::now();
        std::vector<Cluster> cl;
        build_clusters(sc, s, cluster_res, cl);
        uint64_t ff_evals = build_transfer(sc, s, cl, tr, threads);
        double ff_ms = ms_since(t);
        printf("  transfer   %zu clusters, %zu links, row-sum %.3f, %.1fM sdf evals   (%.0f ms)\n", tr.nc, tr.links,
               (double)tr.mean_row_sum, (double)ff_evals / 1e6, ff_ms);
        t = std::chrono::steady_clock::now();
        uint64_t de = light_surfels(sc, s, threads);
        SolveStats st = solve(s, tr, sc.cfg.bounces, threads);
        double solve_ms = ms_since(t);
        printf("  solve      %u bounces, residual %.2e, %.1fM sdf evals   (%.0f ms)\n", st.iterations,
               (double)st.residual, (double)de / 1e6, solve_ms);
        radius = (diag / std::sqrt((float)sc.cfg.surfels)) * 2.6f;
        grid.build(s.p, sc.lo, sc.hi, radius);
    }
    double gi_ms = ms_since(t_gi);
    Cam cam(sc.camera.pos, sc.camera.look, sc.camera.up, sc.camera.fov, w, h);
    std::vector<V3> film;
    Gi gi{&s, &grid, radius};
    auto t0 = std::chrono::steady_clock::now();
    uint64_t ev = render_frame(sc, cam, mode, needs_gi ? &gi : nullptr, tmax, w, h, film, threads);
    double ms = ms_since(t0);
    double px = (double)w * (double)h;
    printf("  shade      %.0f ms   %.1fM sdf evals   %.0f evals/px\n", ms, (double)ev / 1e6, (double)ev / px);
    printf("  total      %.0f ms\n", gi_ms + ms);
    if (!output.empty()) {
        std::vector<uint8_t> buf;
        bool tonemap = (mode == M_BEAUTY || mode == M_DIRECT || mode == M_INDIRECT);
        encode(film, sc.cfg.exposure, tonemap, buf);
        FILE* o = fopen(output.c_str(), "wb");
        if (!o) {
            fprintf(stderr, "error: cannot write %s\n", output.c_str());
            return 1;
        }
        fprintf(o, "P6\n%u %u\n255\n", w, h);
        fwrite(buf.data(), 1, buf.size(), o);
        fclose(o);
        printf("  wrote      %s\n", output.c_str());
    }
    return 0;
}
