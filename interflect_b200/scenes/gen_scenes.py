"""Writes the synthetic benchmark scenes as .rad files (seeded, %.9g floats).

    python -m interflect_b200.scenes.gen_scenes        # rewrites the files next to this script

Scenes (sizes as the benchmark configurations name them):
  c1_cornell.rad          Cornell-style box, 5 inward slabs bounding [-1,1]^3
                          with the front open, a box rotated 15 degrees about y
                          [ext: rotate_y], a sphere r=0.35, a 0.5x0.5 ceiling
                          light (17,12,4); 260x260, 20k surfels, 12 bounces
  c1_cornell_strict.rad   the same with the box unrotated (reference features
                          only)
  c2_product.rad          product scale: a floor plane, a metallic sphere
                          r=0.5, a torus (0.4, 0.12), a capsule (length 0.8,
                          r=0.15), a rounded box and a bowl (a sphere
                          smooth-subtracted with k=0.05 by a smaller sphere
                          [ext: smooth] and drilled by 3 cylinders [ext:
                          subtract_cylinder]); one quad light of emission 10
                          and one sphere light of emission 6 [ext:
                          sphere_light]; albedos U[0.2,0.9] per channel;
                          1920x1080, 200k surfels, 16 bounces
  c2_product_strict.rad   the same objects with reference features only: hard
                          subtraction, sphere drills, two quad lights
  c5_cornell_fill.rad     the differentiation scene: c1_cornell at 512x512
                          with a second, fill light (a sphere light r=0.1 of
                          emission (2.5, 3, 4) near the open front
                          [ext: sphere_light]), so that the gradient has two
                          light emissions
  c3_stress.rad           512 random spheres/boxes/tori (1/3 each, size
                          U[0.1,0.5], albedo U[0.2,0.9]) in [-4,4]^3 inside an
                          enclosing box of 6 slabs, 4 quad lights of emission
                          U[5,20]; 3840x2160, 1M surfels, 24 bounces

"7 SDF primitives" in the product-scale description is read as the five
named objects plus the floor plane and the bowl's inner sphere; the bowl's
three drills are subtractions of the bowl object.
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SEED = 20261203


def f(x) -> str:
    return f"{float(np.float32(x)):.9g}"


def v3(a) -> str:
    return "[" + ", ".join(f(x) for x in a) + "]"


def quad(cx, y, cz, hx, hz, emit) -> str:
    # Counter-clockwise seen from below: the light faces -y.
    verts = [(cx - hx, y, cz - hz), (cx + hx, y, cz - hz), (cx + hx, y, cz + hz), (cx - hx, y, cz + hz)]
    return "light { verts: [" + ", ".join(v3(p) for p in verts) + "], emit: " + v3(emit) + " }\n"


def header(name: str, extra: str = "") -> str:
    return (f"# {name}: generated by interflect_b200/scenes/gen_scenes.py (seed {SEED}).\n"
            + (f"# {extra}\n" if extra else ""))


def c1(rotated: bool) -> str:
    s = header("c1_cornell" + ("" if rotated else "_strict"),
               "extension: rotate_y" if rotated else "reference features only")
    s += "render { width: 260, height: 260, surfels: 20000, bounces: 12, exposure: 1.0 }\n"
    s += "camera { pos: [0, 0, 3.5], look: [0, 0, 0], up: [0, 1, 0], fov: 40 }\n"
    s += 'material "white" { albedo: [0.73, 0.73, 0.73], roughness: 0.9 }\n'
    s += 'material "red" { albedo: [0.63, 0.065, 0.05], roughness: 0.9 }\n'
    s += 'material "green" { albedo: [0.14, 0.45, 0.09], roughness: 0.9 }\n'
    t = 0.1
    s += f'box {{ center: [0, {f(-1 - t / 2)}, 0], size: [2.2, {f(t)}, 2.2], mat: "white" }}\n'
    s += f'box {{ center: [0, {f(1 + t / 2)}, 0], size: [2.2, {f(t)}, 2.2], mat: "white" }}\n'
    s += f'box {{ center: [0, 0, {f(-1 - t / 2)}], size: [2.2, 2.2, {f(t)}], mat: "white" }}\n'
    s += f'box {{ center: [{f(-1 - t / 2)}, 0, 0], size: [{f(t)}, 2.2, 2.2], mat: "red" }}\n'
    s += f'box {{ center: [{f(1 + t / 2)}, 0, 0], size: [{f(t)}, 2.2, 2.2], mat: "green" }}\n'
    rot = ", rotate_y: 15" if rotated else ""
    s += f'box {{ center: [0.35, -0.4, -0.3], size: [0.6, 1.2, 0.6]{rot}, mat: "white" }}\n'
    s += 'sphere { center: [-0.4, -0.65, 0.3], radius: 0.35, mat: "white" }\n'
    s += quad(0.0, 0.99, 0.0, 0.25, 0.25, (17, 12, 4))
    return s


def c5() -> str:
    s = c1(True).replace("render { width: 260, height: 260,", "render { width: 512, height: 512,")
    s = s.replace("# c1_cornell: ", "# c5_cornell_fill: ").replace("# extension: rotate_y", "# extensions: rotate_y, sphere_light")
    s += "sphere_light { center: [-0.55, 0.55, 0.75], radius: 0.1, emit: [2.5, 3, 4] }\n"
    return s


def c2(strict: bool) -> str:
    rng = np.random.default_rng(SEED + 2)
    s = header("c2_product" + ("_strict" if strict else ""),
               "reference features only" if strict else "extensions: smooth, subtract_cylinder, sphere_light")
    s += "render { width: 1920, height: 1080, surfels: 200000, bounces: 16, exposure: 1.0 }\n"
    s += "camera { pos: [0, 1.6, 4.6], look: [0, 0.45, -0.2], up: [0, 1, 0], fov: 40 }\n"
    s += 'material "chrome" { albedo: [0.9, 0.9, 0.9], roughness: 0.1, metallic: 1.0 }\n'
    for name in ("floor", "torus", "capsule", "box", "bowl"):
        a = rng.uniform(0.2, 0.9, 3)
        rough = rng.uniform(0.3, 0.9)
        s += f'material "{name}" {{ albedo: {v3(a)}, roughness: {f(rough)} }}\n'
    s += 'plane { normal: [0, 1, 0], height: 0, mat: "floor" }\n'
    s += 'sphere { center: [-1.2, 0.5, 0.2], radius: 0.5, mat: "chrome" }\n'
    s += 'torus { center: [0.2, 0.12, 1.0], major: 0.4, minor: 0.12, mat: "torus" }\n'
    s += 'capsule { a: [1.3, 0.15, 0.4], b: [1.3, 0.95, 0.4], radius: 0.15, mat: "capsule" }\n'
    s += 'box { center: [0.3, 0.4, -0.5], size: [0.8, 0.8, 0.8], round: 0.08, mat: "box" }\n'
    c = np.array([-0.4, 0.45, -1.5])
    bowl = f'sphere {{ center: {v3(c)}, radius: 0.45, mat: "bowl"'
    inner = c + np.array([0.0, 0.12, 0.0])
    bowl += f", subtract_sphere: [{v3(inner)}, 0.38]"
    for k in range(3):
        ang = np.pi * k / 3.0
        d = np.array([np.cos(ang), 0.0, np.sin(ang)]) * 0.6
        a, b = c + np.array([0, -0.15, 0]) - d, c + np.array([0, -0.15, 0]) + d
        if strict:
            bowl += f", subtract_sphere: [{v3(c + np.array([0, -0.15, 0]) + d * 0.75)}, 0.07]"
        else:
            bowl += f", subtract_cylinder: [{v3(a)}, {v3(b)}, 0.06]"
    if not strict:
        bowl += ", smooth: 0.05"
    s += bowl + " }\n"
    s += quad(0.0, 3.2, 0.0, 0.8, 0.8, (10, 10, 10))
    if strict:
        s += quad(2.2, 2.0, 1.5, 0.22, 0.22, (6, 6, 6))
    else:
        s += "sphere_light { center: [2.2, 2.0, 1.5], radius: 0.25, emit: [6, 6, 6] }\n"
    return s


def stress_scene(rng, name: str, note: str, prims: int, surfels: int, width: int, height: int,
                 bounces: int) -> str:
    """The stress scene's recipe: `prims` random spheres/boxes/tori (1/3
    each, size U[0.1,0.5], albedo U[0.2,0.9]) in [-4,4]^3 inside an enclosing
    box of 6 slabs, 4 quad lights of emission U[5,20]."""
    s = header(name, note)
    s += f"render {{ width: {width}, height: {height}, surfels: {surfels}, bounces: {bounces}, exposure: 1.0 }}\n"
    s += "camera { pos: [0, 0.5, 4.3], look: [0, -0.3, 0], up: [0, 1, 0], fov: 60 }\n"
    s += 'material "wall" { albedo: [0.7, 0.7, 0.68], roughness: 0.9 }\n'
    objs = []
    for i in range(prims):
        kind = rng.integers(0, 3)
        size = rng.uniform(0.1, 0.5)
        c = rng.uniform(-4.0, 4.0, 3)
        a = rng.uniform(0.2, 0.9, 3)
        s += f'material "m{i}" {{ albedo: {v3(a)}, roughness: {f(rng.uniform(0.3, 0.95))} }}\n'
        if kind == 0:
            objs.append(f'sphere {{ center: {v3(c)}, radius: {f(size)}, mat: "m{i}" }}')
        elif kind == 1:
            objs.append(f'box {{ center: {v3(c)}, size: {v3([2 * size] * 3)}, round: {f(0.1 * size)}, mat: "m{i}" }}')
        else:
            objs.append(f'torus {{ center: {v3(c)}, major: {f(size)}, minor: {f(0.3 * size)}, mat: "m{i}" }}')
    w, t = 4.6, 0.2
    for axis in range(3):
        for sign in (-1, 1):
            center = [0.0, 0.0, 0.0]
            center[axis] = sign * (w + t / 2)
            size = [2 * w + 2 * t] * 3
            size[axis] = t
            s += f'box {{ center: {v3(center)}, size: {v3(size)}, mat: "wall" }}\n'
    s += "\n".join(objs) + "\n"
    for k, (x, z) in enumerate(((-2.0, -2.0), (2.0, -2.0), (-2.0, 2.0), (2.0, 2.0))):
        e = rng.uniform(5.0, 20.0)
        s += quad(x, w - 0.02, z, 0.6, 0.6, (e, e, e))
    return s


def c3() -> str:
    return stress_scene(np.random.default_rng(SEED + 3), "c3_stress", "512 random primitives in an enclosing box",
                        512, 1000000, 3840, 2160, 24)


def packed_scenes(count: int = 64, seed: int = SEED + 4) -> list[str]:
    """The batching configuration's many-scene set, generated in memory:
    `count` scenes in the stress scene's style with 8-128 primitives,
    2k-50k surfels requested, square films of 256..1024 pixels (multiples
    of 64) and 24 bounces."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        prims = int(rng.integers(8, 129))
        surfels = int(rng.integers(2000, 50001))
        side = int(rng.integers(4, 17)) * 64
        out.append(stress_scene(rng, f"packed_{i}", f"packed scene {i} of {count} (seed {seed})", prims, surfels,
                                side, side, 24))
    return out


def main() -> None:
    files = {"c1_cornell.rad": c1(True), "c1_cornell_strict.rad": c1(False), "c2_product.rad": c2(False),
             "c2_product_strict.rad": c2(True), "c3_stress.rad": c3(), "c5_cornell_fill.rad": c5()}
    for name, text in files.items():
        with open(os.path.join(HERE, name), "w") as fh:
            fh.write(text)
        print(name, len(text.splitlines()), "lines")


if __name__ == "__main__":
    main()
