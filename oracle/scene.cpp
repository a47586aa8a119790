// Oracle (test infrastructure only): SDF primitives, BVH, scene queries and
// the `.rad` parser, restated from the reference's sdf.rs, bvh.rs and
// scene.rs. Compiled with -ffp-contract=off; see ovec.h.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

#include "oracle.h"

namespace orc {

// ------------------------------------------------------------ counters ----
static std::atomic<bool> g_count_on{false};
static std::mutex g_count_mu;
static WorkCounters g_count = {};
thread_local WorkCounters t_count = {};

void counters_enable(bool on) { g_count_on = on; }
void counters_reset() {
    std::lock_guard<std::mutex> lk(g_count_mu);
    memset(&g_count, 0, sizeof(g_count));
    memset(&t_count, 0, sizeof(t_count));
}
void counters_flush() {
    std::lock_guard<std::mutex> lk(g_count_mu);
    g_count.node_visits += t_count.node_visits;
    g_count.sdf_evals += t_count.sdf_evals;
    for (int i = 0; i < 8; ++i) g_count.prim_evals[i] += t_count.prim_evals[i];
    memset(&t_count, 0, sizeof(t_count));
}
WorkCounters counters_read() {
    counters_flush();
    std::lock_guard<std::mutex> lk(g_count_mu);
    return g_count;
}
#define COUNT(expr)                 \
    do {                            \
        if (g_count_on) { expr; }   \
    } while (0)

// -------------------------------------------------------------- sdf.rs ----
// sdf.rs:52-125
float Prim::dist(V3 p) const {
    COUNT(t_count.prim_evals[type]++);
    switch (type) {
        case P_SPHERE:
            return length(p - c) - r;
        case P_ROUNDBOX: {
            V3 d = p - c;
            if (rotated) {  // [ext] into the box frame: R_y(theta)^T * d
                d = V3(rot_c * d.x - rot_s * d.z, d.y, rot_s * d.x + rot_c * d.z);
            }
            V3 q = vabs(d) - (b - V3::splat(r));
            return length(vmax(q, V3::splat(0.0f))) + fminr(fmaxr(q.x, fmaxr(q.y, q.z)), 0.0f) - r;
        }
        case P_PLANE:
            return dot(p, n) - h;
        case P_CAPSULE: {
            V3 pa = p - a;
            V3 ba = b - a;
            float hh = clampf(dot(pa, ba) / dot(ba, ba), 0.0f, 1.0f);
            return length(pa - ba * hh) - r;
        }
        case P_TORUS: {
            V3 q = p - c;
            float xz = std::sqrt(q.x * q.x + q.z * q.z) - h;
            return std::sqrt(xz * xz + q.y * q.y) - r2;
        }
        case P_CYLINDER: {
            V3 ba = b - a;
            V3 pa = p - a;
            float baba = dot(ba, ba);
            if (baba < 1e-12f) return length(p - a) - r;
            float paba = dot(pa, ba);
            float x = length(pa * baba - ba * paba) - r * baba;
            float y = std::fabs(paba - baba * 0.5f) - baba * 0.5f;
            float x2 = x * x;
            float y2 = y * y * baba;
            float d;
            if (fmaxr(x, y) < 0.0f) {
                d = -fminr(x2, y2);
            } else {
                d = (x > 0.0f ? x2 : 0.0f) + (y > 0.0f ? y2 : 0.0f);
            }
            return signumr(d) * std::sqrt(std::fabs(d)) / baba;
        }
        case P_CONE: {
            V3 ba = b - a;
            float baba = dot(ba, ba);
            if (baba < 1e-12f) return length(p - a) - fmaxr(r, r2);
            float rba = r2 - r;
            V3 pa = p - a;
            float papa = dot(pa, pa);
            float paba = dot(pa, ba) / baba;
            float x = std::sqrt(fmaxr(papa - paba * paba * baba, 0.0f));
            float cax = fmaxr(0.0f, x - (paba < 0.5f ? r : r2));
            float cay = std::fabs(paba - 0.5f) - 0.5f;
            float k = rba * rba + baba;
            float f = clampf((rba * (x - r) + paba * baba) / k, 0.0f, 1.0f);
            float cbx = x - r - f * rba;
            float cby = paba - f;
            float s = (cbx < 0.0f && cay < 0.0f) ? -1.0f : 1.0f;
            return s * std::sqrt(fminr(cax * cax + cay * cay * baba, cbx * cbx + cby * cby * baba));
        }
    }
    return 3.0e38f;
}

// sdf.rs:128-148
bool Prim::bounds(V3& lo, V3& hi) const {
    switch (type) {
        case P_SPHERE:
            lo = c - V3::splat(r);
            hi = c + V3::splat(r);
            return true;
        case P_ROUNDBOX:
            if (rotated) {  // [ext] AABB of the rotated box, padded by 1e-6 relative
                float ex = (std::fabs(rot_c) * b.x + std::fabs(rot_s) * b.z) * 1.000001f;
                float ez = (std::fabs(rot_s) * b.x + std::fabs(rot_c) * b.z) * 1.000001f;
                V3 e(ex, b.y, ez);
                lo = c - e;
                hi = c + e;
                return true;
            }
            lo = c - b;
            hi = c + b;
            return true;
        case P_PLANE:
            return false;
        case P_CAPSULE:
        case P_CYLINDER:
            lo = vmin(a, b) - V3::splat(r);
            hi = vmax(a, b) + V3::splat(r);
            return true;
        case P_TORUS: {
            V3 e(h + r2, r2, h + r2);
            lo = c - e;
            hi = c + e;
            return true;
        }
        case P_CONE: {
            float rr = fmaxr(r, r2);
            lo = vmin(a, b) - V3::splat(rr);
            hi = vmax(a, b) + V3::splat(rr);
            return true;
        }
    }
    return false;
}

// sdf.rs:166-172, plus the [ext] smooth subtraction (Quilez's polynomial
// smooth maximum of d and -s with radius k; k = 0 is the reference's max).
float Object::dist(V3 p) const {
    float d = prim.dist(p);
    for (const Prim& s : subtract) {
        float sd = s.dist(p);
        if (smooth > 0.0f) {
            COUNT(t_count.prim_evals[7]++);
            float hk = clampf(0.5f - 0.5f * (d + sd) / smooth, 0.0f, 1.0f);
            d = d * (1.0f - hk) + (-sd) * hk + smooth * hk * (1.0f - hk);
        } else {
            d = fmaxr(d, -sd);
        }
    }
    return d;
}

// -------------------------------------------------------------- bvh.rs ----
static const int N_BINS = 12;     // bvh.rs:23
static const uint32_t LEAF_SIZE = 4;  // bvh.rs:24

// bvh.rs:46-50
static inline float aabb_dist(V3 p, V3 lo, V3 hi) {
    COUNT(t_count.node_visits++);
    V3 d = vmax(vmax(lo - p, p - hi), V3::splat(0.0f));
    return length(d);
}

struct BoxC {
    V3 lo, hi, c;
};

static float sa_of(V3 lo, V3 hi) {  // bvh.rs:226-232
    if (lo.x > hi.x) return 0.0f;
    V3 d = hi - lo;
    return 2.0f * (d.x * d.y + d.y * d.z + d.z * d.x);
}

static inline size_t bin_of(float cv, float clo, float scale) {
    uint64_t bi = as_usize((cv - clo) * scale);
    return bi < (uint64_t)(N_BINS - 1) ? (size_t)bi : (size_t)(N_BINS - 1);
}

// bvh.rs:166-309
static void build_recursive(std::vector<BvhNode>& nodes, std::vector<uint32_t>& order,
                            const std::vector<BoxC>& boxes, size_t node_idx, size_t start, size_t count) {
    V3 lo = V3::splat(3.40282347e38f), hi = V3::splat(-3.40282347e38f);
    V3 clo = V3::splat(3.40282347e38f), chi = V3::splat(-3.40282347e38f);
    for (size_t i = start; i < start + count; ++i) {
        const BoxC& bx = boxes[order[i]];
        lo = vmin(lo, bx.lo);
        hi = vmax(hi, bx.hi);
        clo = vmin(clo, bx.c);
        chi = vmax(chi, bx.c);
    }
    nodes[node_idx].lo = lo;
    nodes[node_idx].hi = hi;
    if (count <= LEAF_SIZE) {
        nodes[node_idx].start = (uint32_t)start;
        nodes[node_idx].count = (uint32_t)count;
        return;
    }
    V3 ext = chi - clo;
    int axis = (ext.x > ext.y && ext.x > ext.z) ? 0 : (ext.y > ext.z ? 1 : 2);
    float axis_ext = ext[axis];
    if (axis_ext < 1e-9f) {
        nodes[node_idx].start = (uint32_t)start;
        nodes[node_idx].count = (uint32_t)count;
        return;
    }
    float scale = (float)N_BINS / axis_ext;
    V3 bin_lo[N_BINS], bin_hi[N_BINS];
    size_t bin_n[N_BINS];
    for (int i = 0; i < N_BINS; ++i) {
        bin_lo[i] = V3::splat(3.40282347e38f);
        bin_hi[i] = V3::splat(-3.40282347e38f);
        bin_n[i] = 0;
    }
    for (size_t i = start; i < start + count; ++i) {
        const BoxC& bx = boxes[order[i]];
        size_t bi = bin_of(bx.c[axis], clo[axis], scale);
        bin_lo[bi] = vmin(bin_lo[bi], bx.lo);
        bin_hi[bi] = vmax(bin_hi[bi], bx.hi);
        bin_n[bi] += 1;
    }
    float left_area[N_BINS];
    size_t left_cnt[N_BINS];
    V3 al = V3::splat(3.40282347e38f), ah = V3::splat(-3.40282347e38f);
    size_t ac = 0;
    for (int i = 0; i < N_BINS; ++i) {
        al = vmin(al, bin_lo[i]);
        ah = vmax(ah, bin_hi[i]);
        ac += bin_n[i];
        left_area[i] = sa_of(al, ah);
        left_cnt[i] = ac;
    }
    float best_cost = 3.40282347e38f;
    size_t best_split = N_BINS / 2;
    V3 bl = V3::splat(3.40282347e38f), bh = V3::splat(-3.40282347e38f);
    size_t bc = 0;
    for (int i = N_BINS - 1; i >= 1; --i) {
        bl = vmin(bl, bin_lo[i]);
        bh = vmax(bh, bin_hi[i]);
        bc += bin_n[i];
        size_t lc = left_cnt[i - 1];
        if (lc == 0 || bc == 0) continue;
        float cost = left_area[i - 1] * (float)lc + sa_of(bl, bh) * (float)bc;
        if (cost < best_cost) {
            best_cost = cost;
            best_split = (size_t)i;
        }
    }
    size_t mid = 0;
    for (size_t i = 0; i < count; ++i) {
        V3 c = boxes[order[start + i]].c;
        size_t bi = bin_of(c[axis], clo[axis], scale);
        if (bi < best_split) {
            std::swap(order[start + i], order[start + mid]);
            mid += 1;
        }
    }
    if (mid == 0 || mid == count) mid = count / 2;

    BvhNode blank;
    size_t left = nodes.size();
    nodes.push_back(blank);
    build_recursive(nodes, order, boxes, left, start, mid);
    size_t right = nodes.size();
    nodes.push_back(blank);
    nodes[node_idx].count = 0;
    nodes[node_idx].right = (uint32_t)right;
    build_recursive(nodes, order, boxes, right, start + mid, count - mid);
}

// bvh.rs:53-91
void Bvh::build(const std::vector<Object>& objects) {
    nodes.clear();
    order.clear();
    if (objects.empty()) {
        empty = true;
        return;
    }
    std::vector<BoxC> boxes;
    boxes.reserve(objects.size());
    for (const Object& o : objects) {
        V3 lo, hi;
        o.prim.bounds(lo, hi);
        V3 e = V3::splat(o.blend);
        lo = lo - e;
        hi = hi + e;
        boxes.push_back({lo, hi, (lo + hi) * 0.5f});
    }
    for (uint32_t i = 0; i < (uint32_t)objects.size(); ++i) order.push_back(i);
    nodes.reserve(objects.size() * 2);
    nodes.push_back(BvhNode());
    build_recursive(nodes, order, boxes, 0, 0, objects.size());
    empty = false;
}

// ------------------------------------------------------------ scene.rs ----
V3 QuadLight::center() const { return (verts[0] + verts[1] + verts[2] + verts[3]) * 0.25f; }
V3 QuadLight::normal() const { return normalize(cross(verts[1] - verts[0], verts[3] - verts[0])); }
float QuadLight::area() const {
    float a = length(cross(verts[1] - verts[0], verts[3] - verts[0]));
    float b = length(cross(verts[3] - verts[2], verts[1] - verts[2]));
    return 0.5f * (a + b);
}

// scene.rs:106-148
bool RenderCfg::validate(std::string& err) const {
    char buf[256];
    if (width == 0 || height == 0) {
        err = "width and height must be at least 1";
        return false;
    }
    if (width > 16384u || height > 16384u) {
        snprintf(buf, sizeof buf, "image is %ux%u, which exceeds the %u px limit on either side", width, height,
                 16384u);
        err = buf;
        return false;
    }
    uint64_t px = (uint64_t)width * (uint64_t)height;
    if (px > 40000000ull) {
        snprintf(buf, sizeof buf, "image is %llu pixels (%ux%u); the limit is %llu", (unsigned long long)px, width,
                 height, 40000000ull);
        err = buf;
        return false;
    }
    if (surfels == 0) {
        err = "surfels must be at least 1";
        return false;
    }
    if (surfels > 2000000ull) {
        snprintf(buf, sizeof buf, "surfels is %llu; the limit is %llu", (unsigned long long)surfels, 2000000ull);
        err = buf;
        return false;
    }
    if (bounces == 0) {
        err = "bounces must be at least 1";
        return false;
    }
    if (bounces > 4096u) {
        snprintf(buf, sizeof buf, "bounces is %u; the limit is %u", bounces, 4096u);
        err = buf;
        return false;
    }
    if (!std::isfinite(exposure) || exposure <= 0.0f) {
        snprintf(buf, sizeof buf, "exposure must be a positive finite number, got %g", (double)exposure);
        err = buf;
        return false;
    }
    return true;
}

// scene.rs:191-208
DistHit Scene::dist_mat(V3 p) const {
    COUNT(t_count.sdf_evals++);
    DistHit best{3.40282347e38f, 0u};
    for (const Object& o : planes) {
        float d = o.dist(p);
        if (d < best.d) best = DistHit{d, o.mat};
    }
    if (use_bvh) {
        // bvh.rs:100-150
        if (bvh.empty) return best;
        uint32_t stack[64];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            uint32_t ni = stack[--sp];
            const BvhNode& nd = bvh.nodes[ni];
            if (aabb_dist(p, nd.lo, nd.hi) >= best.d) continue;
            if (nd.count > 0) {
                for (uint32_t k = nd.start; k < nd.start + nd.count; ++k) {
                    const Object& o = objects[bvh.order[k]];
                    float d = o.dist(p);
                    if (d < best.d) {
                        best.d = d;
                        best.mat = o.mat;
                    }
                }
            } else {
                uint32_t l = ni + 1, r = nd.right;
                float dl = aabb_dist(p, bvh.nodes[l].lo, bvh.nodes[l].hi);
                float dr = aabb_dist(p, bvh.nodes[r].lo, bvh.nodes[r].hi);
                if (dl < dr) {
                    stack[sp++] = r;
                    stack[sp++] = l;
                } else {
                    stack[sp++] = l;
                    stack[sp++] = r;
                }
            }
        }
    } else {
        // bvh.rs:155-163
        for (const Object& o : objects) {
            float d = o.dist(p);
            if (d < best.d) {
                best.d = d;
                best.mat = o.mat;
            }
        }
    }
    return best;
}

// scene.rs:218-236
V3 Scene::normal(V3 p) const {
    const float H = 5e-4f;
    static const V3 K[4] = {V3(1.0f, -1.0f, -1.0f), V3(-1.0f, -1.0f, 1.0f), V3(-1.0f, 1.0f, -1.0f),
                            V3(1.0f, 1.0f, 1.0f)};
    V3 n(0.0f, 0.0f, 0.0f);
    for (int i = 0; i < 4; ++i) n += K[i] * dist(p + K[i] * H);
    float l = length(n);
    if (l > 1e-12f) return n / l;
    return V3(0.0f, 1.0f, 0.0f);
}

Material Scene::material(uint32_t id) const {
    if (id < materials.size()) return materials[id];
    return Material();
}

// ------------------------------------------------------------- parser ----
// scene.rs:247-300
static std::vector<std::string> tokenize(const std::string& src) {
    std::vector<std::string> out;
    std::string cur;
    bool in_str = false;
    size_t i = 0;
    while (i < src.size()) {
        char c = src[i++];
        if (in_str) {
            if (c == '"') {
                out.push_back("\"" + cur);
                cur.clear();
                in_str = false;
            } else {
                cur.push_back(c);
            }
            continue;
        }
        if (c == '#') {
            while (i < src.size()) {
                if (src[i++] == '\n') break;
            }
            continue;
        }
        if (c == '"') {
            if (!cur.empty()) {
                out.push_back(cur);
                cur.clear();
            }
            in_str = true;
            continue;
        }
        if (strchr("{}[],:", c) != nullptr && c != '\0') {
            if (!cur.empty()) {
                out.push_back(cur);
                cur.clear();
            }
            out.push_back(std::string(1, c));
            continue;
        }
        if (c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f') {
            if (!cur.empty()) {
                out.push_back(cur);
                cur.clear();
            }
            continue;
        }
        cur.push_back(c);
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

// Rust's `str::parse::<f32>` grammar: optional sign, then "inf", "infinity",
// "nan" (any case) or a decimal with optional fraction and exponent. No hex,
// no surrounding whitespace. Conversion is correctly rounded, as is strtof.
static bool rust_parse_f32(const std::string& s, float& out) {
    size_t i = 0, n = s.size();
    if (n == 0) return false;
    if (s[0] == '+' || s[0] == '-') i = 1;
    std::string rest = s.substr(i);
    std::string low;
    for (char ch : rest) low.push_back((char)tolower((unsigned char)ch));
    if (low == "inf" || low == "infinity" || low == "nan") {
        float v = (low == "nan") ? NAN : INFINITY;
        out = (s[0] == '-') ? -v : v;
        return true;
    }
    size_t digits = 0, j = i;
    while (j < n && isdigit((unsigned char)s[j])) { ++j; ++digits; }
    if (j < n && s[j] == '.') {
        ++j;
        while (j < n && isdigit((unsigned char)s[j])) { ++j; ++digits; }
    }
    if (digits == 0) return false;
    if (j < n && (s[j] == 'e' || s[j] == 'E')) {
        ++j;
        if (j < n && (s[j] == '+' || s[j] == '-')) ++j;
        size_t ed = 0;
        while (j < n && isdigit((unsigned char)s[j])) { ++j; ++ed; }
        if (ed == 0) return false;
    }
    if (j != n) return false;
    out = strtof(s.c_str(), nullptr);
    return true;
}

struct Parser {  // scene.rs:302-363
    std::vector<std::string> t;
    size_t i = 0;
    std::string err;

    const std::string* peek() const { return i < t.size() ? &t[i] : nullptr; }
    bool next_tok(std::string& v) {
        if (i >= t.size()) {
            err = "unexpected end of file";
            return false;
        }
        v = t[i++];
        return true;
    }
    bool expect(const char* s) {
        std::string n;
        if (!next_tok(n)) return false;
        if (n == s) return true;
        err = std::string("expected `") + s + "`, found `" + n + "`";
        return false;
    }
    bool flt(float& v) {
        std::string n;
        if (!next_tok(n)) return false;
        if (!rust_parse_f32(n, v)) {
            err = "expected number, found `" + n + "`";
            return false;
        }
        return true;
    }
    void skip_comma() {
        if (peek() && *peek() == ",") ++i;
    }
    bool vec3(V3& v) {
        float x, y, z;
        if (!expect("[")) return false;
        if (!flt(x)) return false;
        skip_comma();
        if (!flt(y)) return false;
        skip_comma();
        if (!flt(z)) return false;
        skip_comma();
        if (!expect("]")) return false;
        v = V3(x, y, z);
        return true;
    }
    bool ident(std::string& v) {
        std::string n;
        if (!next_tok(n)) return false;
        size_t k = 0;
        while (k < n.size() && n[k] == '"') ++k;
        v = n.substr(k);
        return true;
    }
    // Returns 1 with a key, 0 at a closing brace, -1 on error.
    int key(std::string& k) {
        if (peek() && *peek() == "}") {
            ++i;
            return 0;
        }
        if (!next_tok(k)) return -1;
        if (!expect(":")) return -1;
        return 1;
    }
};

// scene.rs:573-601
static void world_bounds(const Scene& sc, V3& lo_out, V3& hi_out) {
    V3 lo = V3::splat(3.40282347e38f), hi = V3::splat(-3.40282347e38f);
    for (const Object& o : sc.objects) {
        V3 a, b;
        if (o.prim.bounds(a, b)) {
            lo = vmin(lo, a);
            hi = vmax(hi, b);
        }
    }
    for (const QuadLight& l : sc.lights) {
        for (int k = 0; k < 4; ++k) {
            lo = vmin(lo, l.verts[k]);
            hi = vmax(hi, l.verts[k]);
        }
    }
    for (const SphereLight& l : sc.sphere_lights) {  // [ext]
        lo = vmin(lo, l.c - V3::splat(l.r));
        hi = vmax(hi, l.c + V3::splat(l.r));
    }
    if (lo.x > hi.x) {
        lo_out = V3::splat(-5.0f);
        hi_out = V3::splat(5.0f);
        return;
    }
    bool has_planes = !sc.planes.empty();
    float diag = length(hi - lo);
    float pad = has_planes ? diag * 0.25f : diag * 0.02f;
    lo_out = lo - V3::splat(pad);
    hi_out = hi + V3::splat(pad);
}

// scene.rs:365-571
bool parse_scene(const std::string& src, Scene& sc, std::string& err) {
    Parser p;
    p.t = tokenize(src);
    sc = Scene();
    sc.materials.push_back(Material());
    std::map<std::string, uint32_t> mat_ids;

#define TRY(x)              \
    do {                    \
        if (!(x)) {         \
            err = p.err;    \
            return false;   \
        }                   \
    } while (0)

    while (p.peek()) {
        std::string block = *p.peek();
        p.i += 1;
        std::string k;
        int kr;
        if (block == "camera") {
            TRY(p.expect("{"));
            while ((kr = p.key(k)) == 1) {
                if (k == "pos") TRY(p.vec3(sc.camera.pos));
                else if (k == "look") TRY(p.vec3(sc.camera.look));
                else if (k == "up") TRY(p.vec3(sc.camera.up));
                else if (k == "fov") TRY(p.flt(sc.camera.fov));
                else {
                    err = "unknown camera key `" + k + "`";
                    return false;
                }
                p.skip_comma();
            }
            TRY(kr == 0);
        } else if (block == "render") {
            TRY(p.expect("{"));
            while ((kr = p.key(k)) == 1) {
                float v;
                if (k == "width") { TRY(p.flt(v)); sc.cfg.width = as_u32(v); }
                else if (k == "height") { TRY(p.flt(v)); sc.cfg.height = as_u32(v); }
                else if (k == "surfels") { TRY(p.flt(v)); sc.cfg.surfels = as_usize(v); }
                else if (k == "bounces") { TRY(p.flt(v)); sc.cfg.bounces = as_u32(v); }
                else if (k == "exposure") { TRY(p.flt(v)); sc.cfg.exposure = v; }
                else {
                    err = "unknown render key `" + k + "`";
                    return false;
                }
                p.skip_comma();
            }
            TRY(kr == 0);
        } else if (block == "material") {
            std::string name;
            TRY(p.ident(name));
            Material m;
            TRY(p.expect("{"));
            while ((kr = p.key(k)) == 1) {
                float v;
                if (k == "albedo") TRY(p.vec3(m.albedo));
                else if (k == "roughness") { TRY(p.flt(v)); m.roughness = clampf(v, 0.02f, 1.0f); }
                else if (k == "metallic") { TRY(p.flt(v)); m.metallic = clampf(v, 0.0f, 1.0f); }
                else if (k == "emissive") TRY(p.vec3(m.emissive));
                else {
                    err = "unknown material key `" + k + "`";
                    return false;
                }
                p.skip_comma();
            }
            TRY(kr == 0);
            mat_ids[name] = (uint32_t)sc.materials.size();
            sc.materials.push_back(m);
        } else if (block == "light") {
            QuadLight l;
            l.emit = V3::splat(10.0f);
            TRY(p.expect("{"));
            while ((kr = p.key(k)) == 1) {
                if (k == "verts") {
                    TRY(p.expect("["));
                    for (int q = 0; q < 4; ++q) {
                        TRY(p.vec3(l.verts[q]));
                        p.skip_comma();
                    }
                    TRY(p.expect("]"));
                } else if (k == "emit") {
                    TRY(p.vec3(l.emit));
                } else {
                    err = "unknown light key `" + k + "`";
                    return false;
                }
                p.skip_comma();
            }
            TRY(kr == 0);
            sc.lights.push_back(l);
        } else if (block == "sphere_light") {  // [ext]
            SphereLight l;
            l.r = 0.25f;
            l.emit = V3::splat(10.0f);
            TRY(p.expect("{"));
            while ((kr = p.key(k)) == 1) {
                if (k == "center") TRY(p.vec3(l.c));
                else if (k == "radius") TRY(p.flt(l.r));
                else if (k == "emit") TRY(p.vec3(l.emit));
                else {
                    err = "unknown sphere_light key `" + k + "`";
                    return false;
                }
                p.skip_comma();
            }
            TRY(kr == 0);
            sc.sphere_lights.push_back(l);
        } else if (block == "sphere" || block == "box" || block == "plane" || block == "capsule" ||
                   block == "torus" || block == "cylinder" || block == "cone") {
            uint32_t mat = 0;
            std::vector<Prim> subtract;
            V3 center(0.0f, 0.0f, 0.0f), size(1.0f, 1.0f, 1.0f), normal(0.0f, 1.0f, 0.0f);
            V3 a(0.0f, 0.0f, 0.0f), b(0.0f, 1.0f, 0.0f);
            float radius = 1.0f, round = 0.0f, height = 0.0f, major = 1.0f, minor = 0.25f, radius_top = 0.0f;
            float rotate_y = 0.0f, smooth = 0.0f;  // [ext]
            bool has_rot = false;
            TRY(p.expect("{"));
            while ((kr = p.key(k)) == 1) {
                if (k == "center") TRY(p.vec3(center));
                else if (k == "radius") TRY(p.flt(radius));
                else if (k == "size") TRY(p.vec3(size));
                else if (k == "round") TRY(p.flt(round));
                else if (k == "normal") { TRY(p.vec3(normal)); normal = normalize(normal); }
                else if (k == "height") TRY(p.flt(height));
                else if (k == "a") TRY(p.vec3(a));
                else if (k == "b") TRY(p.vec3(b));
                else if (k == "major") TRY(p.flt(major));
                else if (k == "minor") TRY(p.flt(minor));
                else if (k == "radius_top") TRY(p.flt(radius_top));
                else if (k == "mat") {
                    std::string nm;
                    TRY(p.ident(nm));
                    auto it = mat_ids.find(nm);
                    if (it == mat_ids.end()) {
                        err = "unknown material `" + nm + "`";
                        return false;
                    }
                    mat = it->second;
                } else if (k == "subtract_sphere") {
                    V3 c;
                    float r;
                    TRY(p.expect("["));
                    TRY(p.vec3(c));
                    p.skip_comma();
                    TRY(p.flt(r));
                    p.skip_comma();
                    TRY(p.expect("]"));
                    Prim s;
                    s.type = P_SPHERE;
                    s.c = c;
                    s.r = r;
                    subtract.push_back(s);
                } else if (k == "subtract_cylinder") {  // [ext]
                    V3 ca, cb;
                    float r;
                    TRY(p.expect("["));
                    TRY(p.vec3(ca));
                    p.skip_comma();
                    TRY(p.vec3(cb));
                    p.skip_comma();
                    TRY(p.flt(r));
                    p.skip_comma();
                    TRY(p.expect("]"));
                    Prim s;
                    s.type = P_CYLINDER;
                    s.a = ca;
                    s.b = cb;
                    s.r = r;
                    subtract.push_back(s);
                } else if (k == "rotate_y") {  // [ext]
                    TRY(p.flt(rotate_y));
                    has_rot = true;
                } else if (k == "smooth") {  // [ext]
                    TRY(p.flt(smooth));
                } else {
                    err = "unknown shape key `" + k + "`";
                    return false;
                }
                p.skip_comma();
            }
            TRY(kr == 0);
            Prim pr;
            if (block == "sphere") {
                pr.type = P_SPHERE;
                pr.c = center;
                pr.r = radius;
            } else if (block == "box") {
                pr.type = P_ROUNDBOX;
                pr.c = center;
                pr.b = size * 0.5f;
                pr.r = fminr(round, min_element(size) * 0.499f);
                if (has_rot && rotate_y != 0.0f) {
                    float th = rotate_y * (PI_F / 180.0f);
                    pr.rot_c = std::cos(th);
                    pr.rot_s = std::sin(th);
                    pr.rotated = true;
                }
            } else if (block == "plane") {
                pr.type = P_PLANE;
                pr.n = normal;
                pr.h = height;
            } else if (block == "capsule") {
                pr.type = P_CAPSULE;
                pr.a = a;
                pr.b = b;
                pr.r = radius;
            } else if (block == "cylinder") {
                pr.type = P_CYLINDER;
                pr.a = a;
                pr.b = b;
                pr.r = radius;
            } else if (block == "cone") {
                pr.type = P_CONE;
                pr.a = a;
                pr.b = b;
                pr.r = radius;
                pr.r2 = radius_top;
            } else {
                pr.type = P_TORUS;
                pr.c = center;
                pr.h = major;
                pr.r2 = minor;
            }
            Object obj;
            obj.prim = pr;
            obj.subtract = subtract;
            obj.mat = mat;
            obj.blend = 0.0f;
            obj.smooth = smooth > 0.0f ? smooth : 0.0f;
            if (pr.type == P_PLANE) sc.planes.push_back(obj);
            else sc.objects.push_back(obj);
        } else {
            err = "unknown block `" + block + "`";
            return false;
        }
    }
#undef TRY
    if (sc.lights.empty() && sc.sphere_lights.empty()) {
        err = "scene has no `light` block";
        return false;
    }
    if (!sc.cfg.validate(err)) return false;
    sc.bvh.build(sc.objects);
    world_bounds(sc, sc.lo, sc.hi);
    return true;
}

}  // namespace orc
