// CPU check of the per-cell candidate-leaf query used by cone-shadow marches
// in large BVHs (interflect_b200/csrc/device.cuh dist_fast,
// k_leafgrid.cu): the grid and the exactness test are restated here over the
// oracle's scene (oracle/), and at points along shadow-style marches every
// answer the test accepts must give the march what the oracle's
// Scene::dist_mat (the reference's pruned near-first traversal,
// bvh.rs:100-150) gives it: both below the 1e-4 stop, or bit for bit equal.
// Prints the query and fallback counts; exits 1 on a disagreement.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>

#include "../../oracle/oracle.h"

using namespace orc;

static float box_d2(V3 p, const BvhNode& n) {
    V3 q = vmax(vmax(n.lo - p, p - n.hi), V3(0.0f, 0.0f, 0.0f));
    return dot(q, q);
}

int main(int argc, char** argv) {
    std::ifstream f(argv[1]);
    std::stringstream ss;
    ss << f.rdbuf();
    Scene sc;
    std::string err;
    if (!parse_scene(ss.str(), sc, err)) {
        std::printf("parse: %s\n", err.c_str());
        return 1;
    }
    std::vector<int> leaves;
    for (size_t i = 0; i < sc.bvh.nodes.size(); ++i)
        if (sc.bvh.nodes[i].count > 0) leaves.push_back((int)i);
    // The grid, as the library builds it.
    double ext = 0.0, mag = 0.0;
    const float lo[3] = {sc.lo.x, sc.lo.y, sc.lo.z}, hi[3] = {sc.hi.x, sc.hi.y, sc.hi.z};
    for (int a = 0; a < 3; ++a) {
        ext = std::max(ext, (double)hi[a] - (double)lo[a]);
        mag = std::max(mag, std::max(std::fabs((double)lo[a]), std::fabs((double)hi[a])));
    }
    const int kCells = 64;
    const double cs = ext / kCells;
    int dim[3];
    for (int a = 0; a < 3; ++a) dim[a] = std::min(kCells, std::max(1, (int)std::ceil(((double)hi[a] - lo[a]) / cs)));
    const float inv_cell = (float)(1.0 / cs);
    const float tol = (float)((mag + (double)sc.diag()) / 4096.0);
    const double pad = tol;
    const float half_diag = (float)((cs * 0.5 + pad) * std::sqrt(3.0) * (1.0 + 1e-6) + pad);
    const size_t ncells = (size_t)dim[0] * dim[1] * dim[2];
    std::vector<std::vector<int>> lists(ncells);
    for (size_t c = 0; c < ncells; ++c) {
        const int x = (int)(c % dim[0]), y = (int)((c / dim[0]) % dim[1]), z = (int)(c / ((size_t)dim[0] * dim[1]));
        const int ix[3] = {x, y, z};
        const float fcell = (float)cs;
        V3 ctr(lo[0] + ((float)x + 0.5f) * fcell, lo[1] + ((float)y + 0.5f) * fcell, lo[2] + ((float)z + 0.5f) * fcell);
        const double lim = std::max((double)(sc.dist(ctr) + half_diag), 0.0) + 2.0 * tol;
        std::vector<std::pair<float, int>> cand;
        for (int L : leaves) {
            const BvhNode& nd = sc.bvh.nodes[L];
            const float nlo[3] = {nd.lo.x, nd.lo.y, nd.lo.z}, nhi[3] = {nd.hi.x, nd.hi.y, nd.hi.z};
            double s = 0.0, k = 0.0;
            for (int a = 0; a < 3; ++a) {
                const double clo = (double)lo[a] + ix[a] * cs - pad, chi = (double)lo[a] + (ix[a] + 1) * cs + pad;
                const double g = std::fmax(0.0, std::fmax((double)nlo[a] - chi, clo - (double)nhi[a]));
                s += g * g;
                const double cc = (double)lo[a] + (ix[a] + 0.5) * cs;
                const double g2 = std::fmax(0.0, std::fmax((double)nlo[a] - cc, cc - (double)nhi[a]));
                k += g2 * g2;
            }
            if (std::sqrt(s) < lim) cand.push_back({(float)k, L});
        }
        std::stable_sort(cand.begin(), cand.end(),
                         [](const std::pair<float, int>& a, const std::pair<float, int>& b) { return a.first < b.first; });
        for (auto& e : cand) lists[c].push_back(e.second);
    }
    // Queries along marches.
    std::mt19937 rng(11);
    std::uniform_real_distribution<float> U(-1.0f, 1.0f);
    long q = 0, fall = 0, bad = 0, listed = 0, outside = 0;
    const float diag = sc.diag();
    for (int ray = 0; ray < 4000; ++ray) {
        V3 ro(U(rng) * 0.95f * hi[0], U(rng) * 0.95f * hi[1], U(rng) * 0.95f * hi[2]);
        V3 rd = normalize(V3(U(rng), U(rng), U(rng)));
        float t = diag * 1e-3f;
        for (int st = 0; st < 96 && t < diag; ++st) {
            const V3 p = ro + rd * t;
            const float href = sc.dist_mat(p).d;
            float P = 3.4028235e38f;
            for (auto& pl : sc.planes) {
                const float d = pl.dist(p);
                if (d < P) P = d;
            }
            const float fx = (p.x - lo[0]) * inv_cell, fy = (p.y - lo[1]) * inv_cell, fz = (p.z - lo[2]) * inv_cell;
            bool ok = false, inside = false;
            float G = P;
            if (fx >= 0.0f && fy >= 0.0f && fz >= 0.0f && fx < (float)dim[0] && fy < (float)dim[1] && fz < (float)dim[2]) {
                const size_t cell = (size_t)fx + (size_t)dim[0] * ((size_t)fy + (size_t)dim[1] * (size_t)fz);
                float best = P, m1 = 3.4028235e38f, m2 = 3.4028235e38f, d2_1 = 0.0f;
                listed += (long)lists[cell].size();
                inside = true;
                for (int L : lists[cell]) {
                    const BvhNode& nd = sc.bvh.nodes[L];
                    const float d2 = box_d2(p, nd);
                    const float lim = best + tol;
                    if (!(lim > 0.0f) || d2 >= lim * lim) continue;
                    float m = 3.4028235e38f;
                    for (uint32_t k = nd.start; k < nd.start + nd.count; ++k) {
                        const float d = sc.objects[sc.bvh.order[k]].dist(p);
                        if (d < m) m = d;
                    }
                    if (m < m1) {
                        m2 = m1;
                        m1 = m;
                        d2_1 = d2;
                    } else if (m < m2) {
                        m2 = m;
                    }
                    if (m < best) best = m;
                }
                G = P <= m1 ? P : m1;
                if (G <= 0.0f) {
                    ok = true;
                } else if (P <= m1) {
                    ok = true;
                } else {
                    const float v1 = std::sqrt(d2_1);
                    ok = v1 <= m1 || (m2 > v1 && P > v1);
                    G = m1;
                }
            }
            ++q;
            if (!ok) {
                ++fall;
                if (!inside) ++outside;
            } else if ((G < 1e-4f) != (href < 1e-4f) || (href >= 1e-4f && std::memcmp(&G, &href, 4) != 0)) {
                if (bad < 5) std::printf("disagree at (%g %g %g): %.9g vs %.9g\n", p.x, p.y, p.z, G, href);
                ++bad;
            }
            if (href < 1e-4f) break;
            t += std::fmin(std::fmax(href, 0.006f), 0.12f);
        }
    }
    std::printf("cells %zu, queries %ld, mean listed %.2f, fallbacks %ld (outside the grid %ld), disagreements %ld\n",
                ncells, q, (double)listed / q, fall, outside, bad);
    if (bad) return 1;
    std::printf("every accepted answer equals the reference traversal\n");
    return 0;
}
