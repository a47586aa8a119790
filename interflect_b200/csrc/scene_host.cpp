// Host side of the scene stage: .rad parser (scene.rs:247-571), world bounds
// (scene.rs:573-601), binned-SAH BVH build (bvh.rs:53-309), and flattening
// into the device program blob.
//
// Built with -ffp-contract=off: every f32 expression here (primitive bounds,
// SAH costs, light and camera constants) must round exactly as the
// reference's unfused f32 arithmetic does, because the device reuses these
// values bit for bit.
#include "scene_host.h"

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>

namespace ifx {

// ---------------------------------------------------------------- math ----
static inline F3 add(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline F3 mul(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
static inline F3 divs(F3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
static inline F3 splat(float s) { return {s, s, s}; }
static inline float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float len3(F3 a) { return std::sqrt(dot3(a, a)); }
static inline F3 norm3(F3 a) { return mul(a, 1.0f / len3(a)); }
static inline F3 cross3(F3 a, F3 b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
static inline F3 min3(F3 a, F3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
static inline F3 max3(F3 a, F3 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
static inline float comp(F3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
// Rust f32::clamp: NaN passes through.
static inline float clampr(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
static const float kPi = 3.14159265358979323846f;
static const float kMax = 3.40282347e38f;

// Rust `f32 as u32` / `as usize`: truncating, saturating, NaN -> 0.
static inline uint32_t sat_u32(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)x;
}
static inline uint64_t sat_u64(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 18446744073709551616.0f) return ~0ull;
    return (uint64_t)x;
}

// ------------------------------------------------------- primitive AABB ----
// sdf.rs:128-148 (planes return false).
static bool prim_bounds(const HPrim& p, F3& lo, F3& hi) {
    switch (p.kind) {
        case K_SPHERE:
            lo = sub(p.c, splat(p.r));
            hi = add(p.c, splat(p.r));
            return true;
        case K_BOX:
            lo = sub(p.c, p.half);
            hi = add(p.c, p.half);
            return true;
        case K_BOX_ROT: {
            // AABB of a box rotated about +y, padded by 1e-6 relative.
            float ex = (std::fabs(p.rot_c) * p.half.x + std::fabs(p.rot_s) * p.half.z) * 1.000001f;
            float ez = (std::fabs(p.rot_s) * p.half.x + std::fabs(p.rot_c) * p.half.z) * 1.000001f;
            F3 e{ex, p.half.y, ez};
            lo = sub(p.c, e);
            hi = add(p.c, e);
            return true;
        }
        case K_PLANE:
            return false;
        case K_CAPSULE:
        case K_CYLINDER:
            lo = sub(min3(p.a, p.b), splat(p.r));
            hi = add(max3(p.a, p.b), splat(p.r));
            return true;
        case K_TORUS: {
            F3 e{p.major + p.minor, p.minor, p.major + p.minor};
            lo = sub(p.c, e);
            hi = add(p.c, e);
            return true;
        }
        case K_CONE: {
            float rr = std::fmax(p.r, p.r_top);
            lo = sub(min3(p.a, p.b), splat(rr));
            hi = add(max3(p.a, p.b), splat(rr));
            return true;
        }
    }
    return false;
}

// ------------------------------------------------------------------ BVH ----
namespace {
struct ObjBox {
    F3 lo, hi, c;
};
const int kBins = 12;        // bvh.rs:23
const size_t kLeafSize = 4;  // bvh.rs:24

float surface_area(F3 lo, F3 hi) {  // bvh.rs:226-232
    if (lo.x > hi.x) return 0.0f;
    F3 d = sub(hi, lo);
    return 2.0f * (d.x * d.y + d.y * d.z + d.z * d.x);
}

size_t bin_index(float c, float clo, float scale) {
    uint64_t b = sat_u64((c - clo) * scale);
    return b < (uint64_t)(kBins - 1) ? (size_t)b : (size_t)(kBins - 1);
}

// bvh.rs:166-309: recursive binned SAH; the left child is allocated right
// after its parent and its subtree is completed before the right child.
void build_node(std::vector<DNode>& nodes, std::vector<uint32_t>& order, const std::vector<ObjBox>& boxes,
                size_t ni, size_t start, size_t count) {
    F3 lo = splat(kMax), hi = splat(-kMax), clo = splat(kMax), chi = splat(-kMax);
    for (size_t i = start; i < start + count; ++i) {
        const ObjBox& b = boxes[order[i]];
        lo = min3(lo, b.lo);
        hi = max3(hi, b.hi);
        clo = min3(clo, b.c);
        chi = max3(chi, b.c);
    }
    DNode& nd = nodes[ni];
    nd.lo[0] = lo.x; nd.lo[1] = lo.y; nd.lo[2] = lo.z;
    nd.hi[0] = hi.x; nd.hi[1] = hi.y; nd.hi[2] = hi.z;
    auto make_leaf = [&]() {
        nodes[ni].count = (int32_t)count;
        nodes[ni].link = (int32_t)start;
    };
    if (count <= kLeafSize) {
        make_leaf();
        return;
    }
    F3 ext = sub(chi, clo);
    int axis = (ext.x > ext.y && ext.x > ext.z) ? 0 : (ext.y > ext.z ? 1 : 2);
    float axis_ext = comp(ext, axis);
    if (axis_ext < 1e-9f) {
        make_leaf();
        return;
    }
    float scale = (float)kBins / axis_ext;
    float clo_a = comp(clo, axis);
    F3 blo[kBins], bhi[kBins];
    size_t bn[kBins];
    for (int i = 0; i < kBins; ++i) {
        blo[i] = splat(kMax);
        bhi[i] = splat(-kMax);
        bn[i] = 0;
    }
    for (size_t i = start; i < start + count; ++i) {
        const ObjBox& b = boxes[order[i]];
        size_t k = bin_index(comp(b.c, axis), clo_a, scale);
        blo[k] = min3(blo[k], b.lo);
        bhi[k] = max3(bhi[k], b.hi);
        bn[k] += 1;
    }
    float larea[kBins];
    size_t lcnt[kBins];
    F3 al = splat(kMax), ah = splat(-kMax);
    size_t acc = 0;
    for (int i = 0; i < kBins; ++i) {
        al = min3(al, blo[i]);
        ah = max3(ah, bhi[i]);
        acc += bn[i];
        larea[i] = surface_area(al, ah);
        lcnt[i] = acc;
    }
    float best = kMax;
    size_t split = kBins / 2;
    F3 rl = splat(kMax), rh = splat(-kMax);
    size_t rc = 0;
    for (int i = kBins - 1; i >= 1; --i) {
        rl = min3(rl, blo[i]);
        rh = max3(rh, bhi[i]);
        rc += bn[i];
        size_t lc = lcnt[i - 1];
        if (lc == 0 || rc == 0) continue;
        float cost = larea[i - 1] * (float)lc + surface_area(rl, rh) * (float)rc;
        if (cost < best) {
            best = cost;
            split = (size_t)i;
        }
    }
    size_t mid = 0;
    for (size_t i = 0; i < count; ++i) {
        if (bin_index(comp(boxes[order[start + i]].c, axis), clo_a, scale) < split) {
            std::swap(order[start + i], order[start + mid]);
            ++mid;
        }
    }
    if (mid == 0 || mid == count) mid = count / 2;
    size_t left = nodes.size();
    nodes.push_back(DNode());
    build_node(nodes, order, boxes, left, start, mid);
    size_t right = nodes.size();
    nodes.push_back(DNode());
    nodes[ni].count = 0;
    nodes[ni].link = (int32_t)right;
    build_node(nodes, order, boxes, right, start + mid, count - mid);
}

void build_bvh(HScene& s) {
    s.nodes.clear();
    s.order.clear();
    if (s.objects.empty()) return;
    std::vector<ObjBox> boxes;
    for (const HObject& o : s.objects) {
        F3 lo, hi;
        prim_bounds(o.prim, lo, hi);
        // bvh.rs:62-72: expansion by the object's blend radius, always 0 here.
        lo = sub(lo, splat(0.0f));
        hi = add(hi, splat(0.0f));
        boxes.push_back({lo, hi, mul(add(lo, hi), 0.5f)});
    }
    for (uint32_t i = 0; i < (uint32_t)s.objects.size(); ++i) s.order.push_back(i);
    s.nodes.reserve(s.objects.size() * 2);
    s.nodes.push_back(DNode());
    build_node(s.nodes, s.order, boxes, 0, 0, s.objects.size());
}

// scene.rs:573-601
void compute_bounds(HScene& s) {
    F3 lo = splat(kMax), hi = splat(-kMax);
    for (const HObject& o : s.objects) {
        F3 a, b;
        if (prim_bounds(o.prim, a, b)) {
            lo = min3(lo, a);
            hi = max3(hi, b);
        }
    }
    for (const HQuadLight& l : s.lights)
        for (int k = 0; k < 4; ++k) {
            lo = min3(lo, l.v[k]);
            hi = max3(hi, l.v[k]);
        }
    for (const HSphereLight& l : s.sphere_lights) {
        lo = min3(lo, sub(l.c, splat(l.r)));
        hi = max3(hi, add(l.c, splat(l.r)));
    }
    if (lo.x > hi.x) {
        s.lo = splat(-5.0f);
        s.hi = splat(5.0f);
        return;
    }
    float diag = len3(sub(hi, lo));
    float pad = s.planes.empty() ? diag * 0.02f : diag * 0.25f;
    s.lo = sub(lo, splat(pad));
    s.hi = add(hi, splat(pad));
}

// ----------------------------------------------------------- tokenizer ----
// scene.rs:247-300: '#' comments, quoted strings kept with a leading '"',
// the punctuation {}[],: as single tokens, whitespace separates.
std::vector<std::string> lex(const std::string& src) {
    std::vector<std::string> toks;
    std::string cur;
    auto flush = [&]() {
        if (!cur.empty()) {
            toks.push_back(cur);
            cur.clear();
        }
    };
    size_t i = 0;
    const size_t n = src.size();
    while (i < n) {
        char c = src[i++];
        if (c == '"') {
            flush();
            std::string str("\"");
            bool closed = false;
            while (i < n) {
                char d = src[i++];
                if (d == '"') {
                    closed = true;
                    break;
                }
                str.push_back(d);
            }
            // An unterminated string ends the input; its text is emitted
            // without the leading quote (scene.rs:296-298 flushes the buffer).
            if (closed) toks.push_back(str);
            else if (str.size() > 1) toks.push_back(str.substr(1));
            continue;
        }
        if (c == '#') {
            while (i < n && src[i] != '\n') ++i;
            if (i < n) ++i;
            continue;
        }
        if (c == '{' || c == '}' || c == '[' || c == ']' || c == ',' || c == ':') {
            flush();
            toks.emplace_back(1, c);
            continue;
        }
        if (c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f') {
            flush();
            continue;
        }
        cur.push_back(c);
    }
    flush();
    return toks;
}

// Rust `str::parse::<f32>`: [+-] then inf / infinity / nan (any case) or a
// decimal with optional fraction and exponent; strtof rounds identically.
bool parse_f32(const std::string& s, float& out) {
    size_t i = (!s.empty() && (s[0] == '+' || s[0] == '-')) ? 1 : 0;
    std::string body;
    for (size_t k = i; k < s.size(); ++k) body.push_back((char)std::tolower((unsigned char)s[k]));
    if (body == "inf" || body == "infinity" || body == "nan") {
        float v = body == "nan" ? NAN : INFINITY;
        out = (i == 1 && s[0] == '-') ? -v : v;
        return true;
    }
    size_t j = i, digits = 0;
    while (j < s.size() && std::isdigit((unsigned char)s[j])) ++j, ++digits;
    if (j < s.size() && s[j] == '.') {
        ++j;
        while (j < s.size() && std::isdigit((unsigned char)s[j])) ++j, ++digits;
    }
    if (digits == 0) return false;
    if (j < s.size() && (s[j] == 'e' || s[j] == 'E')) {
        ++j;
        if (j < s.size() && (s[j] == '+' || s[j] == '-')) ++j;
        size_t ed = 0;
        while (j < s.size() && std::isdigit((unsigned char)s[j])) ++j, ++ed;
        if (ed == 0) return false;
    }
    if (j != s.size()) return false;
    out = std::strtof(s.c_str(), nullptr);
    return true;
}

// Token cursor with the reference parser's error messages (scene.rs:302-363).
struct Cursor {
    std::vector<std::string> toks;
    size_t pos = 0;
    std::string err;

    bool at(const char* s) const { return pos < toks.size() && toks[pos] == s; }
    bool done() const { return pos >= toks.size(); }
    bool take(std::string& v) {
        if (done()) {
            err = "unexpected end of file";
            return false;
        }
        v = toks[pos++];
        return true;
    }
    bool want(const char* s) {
        std::string t;
        if (!take(t)) return false;
        if (t == s) return true;
        err = std::string("expected `") + s + "`, found `" + t + "`";
        return false;
    }
    bool number(float& v) {
        std::string t;
        if (!take(t)) return false;
        if (parse_f32(t, v)) return true;
        err = "expected number, found `" + t + "`";
        return false;
    }
    void comma() {
        if (at(",")) ++pos;
    }
    bool vec(F3& v) {
        if (!want("[")) return false;
        if (!number(v.x)) return false;
        comma();
        if (!number(v.y)) return false;
        comma();
        if (!number(v.z)) return false;
        comma();
        return want("]");
    }
    bool name(std::string& v) {
        if (!take(v)) return false;
        size_t k = v.find_first_not_of('"');
        v = k == std::string::npos ? std::string() : v.substr(k);
        return true;
    }
    // 1 = key read, 0 = closing brace, -1 = error.
    int key(std::string& k) {
        if (at("}")) {
            ++pos;
            return 0;
        }
        if (!take(k) || !want(":")) return -1;
        return 1;
    }
};

bool is_shape(const std::string& b) {
    return b == "sphere" || b == "box" || b == "plane" || b == "capsule" || b == "torus" || b == "cylinder" ||
           b == "cone";
}
}  // namespace

// scene.rs:106-148
bool validate_cfg(const HCfg& cfg, std::string& err) {
    char buf[256];
    if (cfg.width == 0 || cfg.height == 0) {
        err = "width and height must be at least 1";
        return false;
    }
    if (cfg.width > 16384u || cfg.height > 16384u) {
        snprintf(buf, sizeof buf, "image is %ux%u, which exceeds the 16384 px limit on either side", cfg.width,
                 cfg.height);
        err = buf;
        return false;
    }
    uint64_t px = (uint64_t)cfg.width * cfg.height;
    if (px > 40000000ull) {
        snprintf(buf, sizeof buf, "image is %llu pixels (%ux%u); the limit is 40000000", (unsigned long long)px,
                 cfg.width, cfg.height);
        err = buf;
        return false;
    }
    if (cfg.surfels == 0) {
        err = "surfels must be at least 1";
        return false;
    }
    if (cfg.surfels > 2000000ull) {
        snprintf(buf, sizeof buf,
                 "surfels is %llu; the limit is 2000000. Values this large ask for tens of gigabytes and cannot "
                 "finish",
                 (unsigned long long)cfg.surfels);
        err = buf;
        return false;
    }
    if (cfg.bounces == 0) {
        err = "bounces must be at least 1";
        return false;
    }
    if (cfg.bounces > 4096u) {
        snprintf(buf, sizeof buf,
                 "bounces is %u; the limit is 4096. The solve converges in tens of bounces, so this only burns CPU",
                 cfg.bounces);
        err = buf;
        return false;
    }
    if (!std::isfinite(cfg.exposure) || cfg.exposure <= 0.0f) {
        snprintf(buf, sizeof buf, "exposure must be a positive finite number, got %g", (double)cfg.exposure);
        err = buf;
        return false;
    }
    return true;
}

// scene.rs:365-571
bool parse_rad(const std::string& src, HScene& s, std::string& err) {
    Cursor cur;
    cur.toks = lex(src);
    s = HScene();
    s.materials.push_back(HMaterial());
    std::map<std::string, uint32_t> mat_ids;
    std::string k;
    int kr = 0;
    auto fail = [&](const std::string& e) {
        err = e;
        return false;
    };
#define NEED(x)                 \
    do {                        \
        if (!(x)) {             \
            err = cur.err;      \
            return false;       \
        }                       \
    } while (0)
#define KEYS_END() NEED(kr == 0)

    while (!cur.done()) {
        std::string block = cur.toks[cur.pos++];
        if (block == "camera") {
            NEED(cur.want("{"));
            while ((kr = cur.key(k)) == 1) {
                if (k == "pos") NEED(cur.vec(s.camera.pos));
                else if (k == "look") NEED(cur.vec(s.camera.look));
                else if (k == "up") NEED(cur.vec(s.camera.up));
                else if (k == "fov") NEED(cur.number(s.camera.fov));
                else return fail("unknown camera key `" + k + "`");
                cur.comma();
            }
            KEYS_END();
        } else if (block == "render") {
            NEED(cur.want("{"));
            while ((kr = cur.key(k)) == 1) {
                float v = 0;
                if (k == "width") { NEED(cur.number(v)); s.cfg.width = sat_u32(v); }
                else if (k == "height") { NEED(cur.number(v)); s.cfg.height = sat_u32(v); }
                else if (k == "surfels") { NEED(cur.number(v)); s.cfg.surfels = sat_u64(v); }
                else if (k == "bounces") { NEED(cur.number(v)); s.cfg.bounces = sat_u32(v); }
                else if (k == "exposure") NEED(cur.number(s.cfg.exposure));
                else return fail("unknown render key `" + k + "`");
                cur.comma();
            }
            KEYS_END();
        } else if (block == "material") {
            std::string nm;
            NEED(cur.name(nm));
            HMaterial m;
            NEED(cur.want("{"));
            while ((kr = cur.key(k)) == 1) {
                float v = 0;
                if (k == "albedo") NEED(cur.vec(m.albedo));
                else if (k == "roughness") { NEED(cur.number(v)); m.roughness = clampr(v, 0.02f, 1.0f); }
                else if (k == "metallic") { NEED(cur.number(v)); m.metallic = clampr(v, 0.0f, 1.0f); }
                else if (k == "emissive") NEED(cur.vec(m.emissive));
                else return fail("unknown material key `" + k + "`");
                cur.comma();
            }
            KEYS_END();
            mat_ids[nm] = (uint32_t)s.materials.size();
            s.materials.push_back(m);
        } else if (block == "light") {
            HQuadLight l;
            for (auto& v : l.v) v = F3{0, 0, 0};
            NEED(cur.want("{"));
            while ((kr = cur.key(k)) == 1) {
                if (k == "verts") {
                    NEED(cur.want("["));
                    for (auto& v : l.v) {
                        NEED(cur.vec(v));
                        cur.comma();
                    }
                    NEED(cur.want("]"));
                } else if (k == "emit") {
                    NEED(cur.vec(l.emit));
                } else {
                    return fail("unknown light key `" + k + "`");
                }
                cur.comma();
            }
            KEYS_END();
            s.lights.push_back(l);
        } else if (block == "sphere_light") {  // extension
            HSphereLight l;
            NEED(cur.want("{"));
            while ((kr = cur.key(k)) == 1) {
                if (k == "center") NEED(cur.vec(l.c));
                else if (k == "radius") NEED(cur.number(l.r));
                else if (k == "emit") NEED(cur.vec(l.emit));
                else return fail("unknown sphere_light key `" + k + "`");
                cur.comma();
            }
            KEYS_END();
            s.sphere_lights.push_back(l);
        } else if (is_shape(block)) {
            HObject obj;
            F3 center{0, 0, 0}, size{1, 1, 1}, normal{0, 1, 0}, a{0, 0, 0}, b{0, 1, 0};
            float radius = 1.0f, round = 0.0f, height = 0.0f, major = 1.0f, minor = 0.25f, radius_top = 0.0f;
            float rotate_y = 0.0f, smooth = 0.0f;
            NEED(cur.want("{"));
            while ((kr = cur.key(k)) == 1) {
                if (k == "center") NEED(cur.vec(center));
                else if (k == "radius") NEED(cur.number(radius));
                else if (k == "size") NEED(cur.vec(size));
                else if (k == "round") NEED(cur.number(round));
                else if (k == "normal") { NEED(cur.vec(normal)); normal = norm3(normal); }
                else if (k == "height") NEED(cur.number(height));
                else if (k == "a") NEED(cur.vec(a));
                else if (k == "b") NEED(cur.vec(b));
                else if (k == "major") NEED(cur.number(major));
                else if (k == "minor") NEED(cur.number(minor));
                else if (k == "radius_top") NEED(cur.number(radius_top));
                else if (k == "mat") {
                    std::string nm;
                    NEED(cur.name(nm));
                    auto it = mat_ids.find(nm);
                    if (it == mat_ids.end()) return fail("unknown material `" + nm + "`");
                    obj.mat = it->second;
                } else if (k == "subtract_sphere") {
                    HPrim sp;
                    sp.kind = K_SPHERE;
                    NEED(cur.want("["));
                    NEED(cur.vec(sp.c));
                    cur.comma();
                    NEED(cur.number(sp.r));
                    cur.comma();
                    NEED(cur.want("]"));
                    obj.subtract.push_back(sp);
                } else if (k == "subtract_cylinder") {  // extension
                    HPrim cy;
                    cy.kind = K_CYLINDER;
                    NEED(cur.want("["));
                    NEED(cur.vec(cy.a));
                    cur.comma();
                    NEED(cur.vec(cy.b));
                    cur.comma();
                    NEED(cur.number(cy.r));
                    cur.comma();
                    NEED(cur.want("]"));
                    obj.subtract.push_back(cy);
                } else if (k == "rotate_y") {  // extension
                    NEED(cur.number(rotate_y));
                } else if (k == "smooth") {  // extension
                    NEED(cur.number(smooth));
                } else {
                    return fail("unknown shape key `" + k + "`");
                }
                cur.comma();
            }
            KEYS_END();
            HPrim& p = obj.prim;
            if (block == "sphere") {
                p.kind = K_SPHERE;
                p.c = center;
                p.r = radius;
            } else if (block == "box") {
                p.kind = K_BOX;
                p.c = center;
                p.half = mul(size, 0.5f);
                p.r = std::fmin(round, std::fmin(size.x, std::fmin(size.y, size.z)) * 0.499f);
                if (rotate_y != 0.0f) {
                    float th = rotate_y * (kPi / 180.0f);
                    p.kind = K_BOX_ROT;
                    p.rot_c = std::cos(th);
                    p.rot_s = std::sin(th);
                }
            } else if (block == "plane") {
                p.kind = K_PLANE;
                p.n = normal;
                p.h = height;
            } else if (block == "capsule" || block == "cylinder") {
                p.kind = block == "capsule" ? K_CAPSULE : K_CYLINDER;
                p.a = a;
                p.b = b;
                p.r = radius;
            } else if (block == "cone") {
                p.kind = K_CONE;
                p.a = a;
                p.b = b;
                p.r = radius;
                p.r_top = radius_top;
            } else {
                p.kind = K_TORUS;
                p.c = center;
                p.major = major;
                p.minor = minor;
            }
            obj.smooth = smooth > 0.0f ? smooth : 0.0f;
            if (p.kind == K_PLANE) s.planes.push_back(obj);
            else s.objects.push_back(obj);
        } else {
            return fail("unknown block `" + block + "`");
        }
    }
#undef NEED
#undef KEYS_END
    if (s.lights.empty() && s.sphere_lights.empty()) return fail("scene has no `light` block");
    if (!validate_cfg(s.cfg, err)) return false;
    build_bvh(s);
    compute_bounds(s);
    return true;
}

float scene_diag(const HScene& s) { return len3(sub(s.hi, s.lo)); }

// ------------------------------------------------------------- flatten ----
// Writes one primitive record, hoisting its p-independent terms.
static DPrim pack_prim(const HPrim& p) {
    DPrim d;
    memset(&d, 0, sizeof d);
    d.kind = p.kind;
    float* v = d.v;
    switch (p.kind) {
        case K_SPHERE:
            v[0] = p.c.x; v[1] = p.c.y; v[2] = p.c.z; v[3] = p.r;
            break;
        case K_BOX:
        case K_BOX_ROT: {
            F3 q = sub(p.half, splat(p.r));  // sdf.rs:58 (b - splat(r))
            v[0] = p.c.x; v[1] = p.c.y; v[2] = p.c.z;
            v[3] = q.x; v[4] = q.y; v[5] = q.z;
            v[6] = p.r; v[7] = p.rot_c; v[8] = p.rot_s;
            break;
        }
        case K_PLANE:
            v[0] = p.n.x; v[1] = p.n.y; v[2] = p.n.z; v[3] = p.h;
            break;
        case K_CAPSULE: {
            F3 ba = sub(p.b, p.a);
            v[0] = p.a.x; v[1] = p.a.y; v[2] = p.a.z;
            v[3] = ba.x; v[4] = ba.y; v[5] = ba.z;
            v[6] = dot3(ba, ba); v[7] = p.r;
            break;
        }
        case K_TORUS:
            v[0] = p.c.x; v[1] = p.c.y; v[2] = p.c.z; v[3] = p.major; v[4] = p.minor;
            break;
        case K_CYLINDER: {
            F3 ba = sub(p.b, p.a);
            float baba = dot3(ba, ba);
            if (baba < 1e-12f) {  // sdf.rs:83-85: a sphere at a
                d.kind = K_SPHERE;
                v[0] = p.a.x; v[1] = p.a.y; v[2] = p.a.z; v[3] = p.r;
                break;
            }
            v[0] = p.a.x; v[1] = p.a.y; v[2] = p.a.z;
            v[3] = ba.x; v[4] = ba.y; v[5] = ba.z;
            v[6] = baba; v[7] = p.r; v[8] = p.r * baba; v[9] = baba * 0.5f;
            break;
        }
        case K_CONE: {
            F3 ba = sub(p.b, p.a);
            float baba = dot3(ba, ba);
            if (baba < 1e-12f) {  // sdf.rs:104-106
                d.kind = K_SPHERE;
                v[0] = p.a.x; v[1] = p.a.y; v[2] = p.a.z; v[3] = std::fmax(p.r, p.r_top);
                break;
            }
            float rba = p.r_top - p.r;
            v[0] = p.a.x; v[1] = p.a.y; v[2] = p.a.z;
            v[3] = ba.x; v[4] = ba.y; v[5] = ba.z;
            v[6] = baba; v[7] = p.r; v[8] = p.r_top; v[9] = rba; v[10] = rba * rba + baba;
            break;
        }
    }
    return d;
}

std::vector<uint8_t> flatten_scene(const HScene& s) {
    // Stored object order: planes, then BVH leaf order.
    std::vector<const HObject*> stored;
    for (const HObject& o : s.planes) stored.push_back(&o);
    for (uint32_t oi : s.order) stored.push_back(&s.objects[oi]);
    std::vector<uint32_t> linear(s.objects.size());
    for (size_t k = 0; k < s.order.size(); ++k) linear[s.order[k]] = (uint32_t)(s.planes.size() + k);

    std::vector<DObject> objs;
    std::vector<DPrim> prims;
    for (const HObject* o : stored) {
        DObject d;
        d.prim = (int32_t)prims.size();
        d.nsub = (int32_t)o->subtract.size();
        d.mat = o->mat;
        d.smooth = o->smooth;
        objs.push_back(d);
        prims.push_back(pack_prim(o->prim));
        for (const HPrim& sp : o->subtract) prims.push_back(pack_prim(sp));
    }
    // Leaves index stored objects: shift by the plane count.
    std::vector<DNode> nodes = s.nodes;
    for (DNode& n : nodes)
        if (n.count > 0) n.link += (int32_t)s.planes.size();

    std::vector<DQuadLight> ql;
    for (const HQuadLight& l : s.lights) {
        DQuadLight d;
        memset(&d, 0, sizeof d);
        for (int k = 0; k < 4; ++k) {
            d.v[k][0] = l.v[k].x; d.v[k][1] = l.v[k].y; d.v[k][2] = l.v[k].z;
        }
        // scene.rs:39-55, shade.rs:62-79
        F3 c = mul(add(add(add(l.v[0], l.v[1]), l.v[2]), l.v[3]), 0.25f);
        F3 e1 = sub(l.v[1], l.v[0]), e2 = sub(l.v[3], l.v[0]);
        F3 nc = cross3(e1, e2);
        F3 n = norm3(nc);
        float a1 = len3(nc);
        float a2 = len3(cross3(sub(l.v[3], l.v[2]), sub(l.v[1], l.v[2])));
        float area = 0.5f * (a1 + a2);
        float radius = std::fmax(std::sqrt(area / kPi), 1e-4f);
        d.center[0] = c.x; d.center[1] = c.y; d.center[2] = c.z; d.center[3] = radius;
        d.normal[0] = n.x; d.normal[1] = n.y; d.normal[2] = n.z; d.normal[3] = area;
        d.emit[0] = l.emit.x; d.emit[1] = l.emit.y; d.emit[2] = l.emit.z;
        d.e1[0] = e1.x; d.e1[1] = e1.y; d.e1[2] = e1.z; d.e1[3] = dot3(e1, e1);
        d.e2[0] = e2.x; d.e2[1] = e2.y; d.e2[2] = e2.z; d.e2[3] = dot3(e2, e2);
        d.ncross[0] = nc.x; d.ncross[1] = nc.y; d.ncross[2] = nc.z;
        ql.push_back(d);
    }
    std::vector<DSphereLight> sl;
    for (const HSphereLight& l : s.sphere_lights) {
        DSphereLight d;
        memset(&d, 0, sizeof d);
        d.c[0] = l.c.x; d.c[1] = l.c.y; d.c[2] = l.c.z; d.c[3] = l.r;
        d.emit[0] = l.emit.x; d.emit[1] = l.emit.y; d.emit[2] = l.emit.z;
        sl.push_back(d);
    }
    std::vector<DMaterial> mats;
    for (const HMaterial& m : s.materials) {
        DMaterial d;
        memset(&d, 0, sizeof d);
        d.albedo[0] = m.albedo.x; d.albedo[1] = m.albedo.y; d.albedo[2] = m.albedo.z; d.albedo[3] = m.roughness;
        d.emissive[0] = m.emissive.x; d.emissive[1] = m.emissive.y; d.emissive[2] = m.emissive.z;
        d.emissive[3] = m.metallic;
        // shade.rs:36-43: kd = albedo * (1 - metallic); f0 = lerp(0.04, albedo, metallic)
        float om = 1.0f - m.metallic;
        d.kd[0] = m.albedo.x * om; d.kd[1] = m.albedo.y * om; d.kd[2] = m.albedo.z * om;
        d.kd[3] = std::fmax(m.roughness * m.roughness, 1e-3f);
        d.f0[0] = 0.04f * om + m.albedo.x * m.metallic;
        d.f0[1] = 0.04f * om + m.albedo.y * m.metallic;
        d.f0[2] = 0.04f * om + m.albedo.z * m.metallic;
        d.f0[3] = (m.roughness < 0.45f || m.metallic > 0.05f) ? 1.0f : 0.0f;  // main.rs:322
        mats.push_back(d);
    }

    BlobHeader h;
    memset(&h, 0, sizeof h);
    h.n_planes = (int32_t)s.planes.size();
    h.n_objects = (int32_t)s.objects.size();
    h.n_prims = (int32_t)prims.size();
    h.n_nodes = (int32_t)nodes.size();
    h.n_lights = (int32_t)ql.size();
    h.n_sphere_lights = (int32_t)sl.size();
    h.n_materials = (int32_t)mats.size();
    h.use_bvh = s.use_bvh ? 1 : 0;
    uint32_t off = align16(sizeof(BlobHeader));
    h.off_objects = off;
    off += align16((uint32_t)(objs.size() * sizeof(DObject)));
    h.off_prims = off;
    off += align16((uint32_t)(prims.size() * sizeof(DPrim)));
    h.off_nodes = off;
    off += align16((uint32_t)(nodes.size() * sizeof(DNode)));
    h.off_lights = off;
    off += align16((uint32_t)(ql.size() * sizeof(DQuadLight)));
    h.off_sphere_lights = off;
    off += align16((uint32_t)(sl.size() * sizeof(DSphereLight)));
    h.off_materials = off;
    off += align16((uint32_t)(mats.size() * sizeof(DMaterial)));
    h.off_linear = off;
    off += align16((uint32_t)(linear.size() * sizeof(uint32_t)));
    h.total_bytes = off;
    std::vector<uint8_t> blob(off, 0);
    memcpy(blob.data(), &h, sizeof h);
    auto put = [&](uint32_t at, const void* src, size_t bytes) {
        if (bytes) memcpy(blob.data() + at, src, bytes);
    };
    put(h.off_objects, objs.data(), objs.size() * sizeof(DObject));
    put(h.off_prims, prims.data(), prims.size() * sizeof(DPrim));
    put(h.off_nodes, nodes.data(), nodes.size() * sizeof(DNode));
    put(h.off_lights, ql.data(), ql.size() * sizeof(DQuadLight));
    put(h.off_sphere_lights, sl.data(), sl.size() * sizeof(DSphereLight));
    put(h.off_materials, mats.data(), mats.size() * sizeof(DMaterial));
    put(h.off_linear, linear.data(), linear.size() * sizeof(uint32_t));
    return blob;
}

// trace.rs:165-177 direction coefficients (identical for every surfel):
// (r cos phi, r sin phi, sqrt(max(1 - u1, 0))) with u1, u2 the base-2 and
// base-3 radical inverses of k + 1.
static float radical_inverse(uint32_t i, uint32_t base) {  // trace.rs:189-199
    float f = 1.0f, r = 0.0f;
    float inv = 1.0f / (float)base;
    while (i > 0) {
        f *= inv;
        r += f * (float)(i % base);
        i /= base;
    }
    return r;
}

SceneConsts scene_consts(const HScene& s) {
    SceneConsts c;
    memset(&c, 0, sizeof c);
    c.lo[0] = s.lo.x; c.lo[1] = s.lo.y; c.lo[2] = s.lo.z;
    c.hi[0] = s.hi.x; c.hi[1] = s.hi.y; c.hi[2] = s.hi.z;
    c.diag = scene_diag(s);
    const float tau = 6.28318530717958647692f;
    for (uint32_t k = 0; k < 16; ++k) {
        float u1 = radical_inverse(k + 1, 2);
        float u2 = radical_inverse(k + 1, 3);
        float r = std::sqrt(u1);
        float phi = tau * u2;
        c.closure[k][0] = r * std::cos(phi);
        c.closure[k][1] = r * std::sin(phi);
        c.closure[k][2] = std::sqrt(std::fmax(1.0f - u1, 0.0f));
    }
    return c;
}

// main.rs:198-210
CamBasis camera_basis(const F3& pos, const F3& look, const F3& up_hint, float fov, uint32_t w, uint32_t h) {
    CamBasis b;
    F3 fwd = norm3(sub(look, pos));
    F3 right = norm3(cross3(fwd, up_hint));
    F3 up = cross3(right, fwd);
    const float rads = kPi / 180.0f;
    b.origin[0] = pos.x; b.origin[1] = pos.y; b.origin[2] = pos.z;
    b.fwd[0] = fwd.x; b.fwd[1] = fwd.y; b.fwd[2] = fwd.z;
    b.right[0] = right.x; b.right[1] = right.y; b.right[2] = right.z;
    b.up[0] = up.x; b.up[1] = up.y; b.up[2] = up.z;
    b.tan_half = std::tan(fov * rads * 0.5f);
    b.aspect = (float)w / (float)h;
    return b;
}

// film.rs:23-31
uint8_t srgb_host(float c) {
    c = clampr(c, 0.0f, 1.0f);
    float v = (c <= 0.0031308f) ? c * 12.92f : 1.055f * std::pow(c, 1.0f / 2.4f) - 0.055f;
    float x = v * 255.0f + 0.5f;
    if (!(x > 0.0f)) return 0;
    if (x >= 255.0f) return 255;
    return (uint8_t)x;
}

void srgb_thresholds(float t[256]) {
    // t[k]: the smallest f32 in [0, 1] whose encoding is >= k; found by
    // bisection over the (ordered) bit patterns of non-negative floats.
    t[0] = -INFINITY;
    uint32_t one;
    float f1 = 1.0f;
    memcpy(&one, &f1, 4);
    for (int k = 1; k < 256; ++k) {
        uint32_t lo = 0, hi = one;  // srgb(bits(hi)) >= k always (255 at 1.0)
        while (lo < hi) {
            uint32_t mid = lo + (hi - lo) / 2;
            float m;
            memcpy(&m, &mid, 4);
            if (srgb_host(m) >= k) hi = mid;
            else lo = mid + 1;
        }
        memcpy(&t[k], &lo, 4);
    }
}

}  // namespace ifx
