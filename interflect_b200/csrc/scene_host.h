// Host side of the scene stage: the .rad parser, the BVH builder and the
// flattening of a parsed scene into the device program blob (layout.h).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "layout.h"

namespace ifx {

struct F3 {
    float x, y, z;
};

// One primitive as written in the scene (sdf.rs:10-48 plus the rotated box).
struct HPrim {
    int32_t kind = K_SPHERE;
    F3 c{0, 0, 0}, half{0, 0, 0}, a{0, 0, 0}, b{0, 1, 0}, n{0, 1, 0};
    float r = 0, r_top = 0, major = 0, minor = 0, h = 0;
    float rot_c = 1, rot_s = 0;
};

struct HObject {
    HPrim prim;
    std::vector<HPrim> subtract;
    uint32_t mat = 0;
    float smooth = 0;
};

struct HMaterial {
    F3 albedo{0.8f, 0.8f, 0.8f};
    float roughness = 0.8f, metallic = 0.0f;
    F3 emissive{0, 0, 0};
};

struct HQuadLight {
    F3 v[4];
    F3 emit{10, 10, 10};
};

struct HSphereLight {
    F3 c{0, 0, 0};
    float r = 0.25f;
    F3 emit{10, 10, 10};
};

struct HCfg {
    uint32_t width = 800, height = 600;
    uint64_t surfels = 20000;
    uint32_t bounces = 12;
    float exposure = 1.0f;
};

struct HCamera {
    F3 pos{0, 2, 6}, look{0, 1, 0}, up{0, 1, 0};
    float fov = 40.0f;
};

struct HScene {
    std::vector<HObject> objects;  // bounded, parse order
    std::vector<HObject> planes;
    std::vector<HMaterial> materials;  // [0] = default
    std::vector<HQuadLight> lights;
    std::vector<HSphereLight> sphere_lights;
    HCamera camera;
    HCfg cfg;
    bool use_bvh = true;
    F3 lo{0, 0, 0}, hi{0, 0, 0};
    // Flattened BVH (bvh.rs:27-36 node semantics) and leaf object order.
    std::vector<DNode> nodes;
    std::vector<uint32_t> order;
};

// scene.rs:365-571. Returns false with a diagnostic on malformed input.
bool parse_rad(const std::string& src, HScene& out, std::string& err);
// scene.rs:106-148
bool validate_cfg(const HCfg& cfg, std::string& err);
float scene_diag(const HScene& s);
// Flattens into the blob described in layout.h.
std::vector<uint8_t> flatten_scene(const HScene& s);
SceneConsts scene_consts(const HScene& s);

// Camera basis of main.rs:198-210.
struct CamBasis {
    float origin[3], fwd[3], right[3], up[3];
    float tan_half, aspect;
};
CamBasis camera_basis(const F3& pos, const F3& look, const F3& up_hint, float fov, uint32_t w, uint32_t h);

// film.rs:23-31 encodes through powf; the GPU reproduces the host's bytes
// exactly by comparing against the 255 input thresholds at which the encoded
// byte steps up (t[k] = smallest f32 c with srgb(c) >= k, k = 1..255).
void srgb_thresholds(float t[256]);
uint8_t srgb_host(float c);

}  // namespace ifx
