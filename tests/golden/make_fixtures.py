"""Regenerates the fixtures in this folder from the reference checkout.

Run in a container that has the reference crate mounted (default path below,
or pass it as the first argument):

    python tests/golden/make_fixtures.py [/path/to/interflect]

It writes
  scenes/*.rad            the reference's own scene files (product, cornell,
                          stress and the four bench scenes) and the scenes its
                          unit tests embed as string constants (closed_box,
                          flush_ceiling_light, minimal)
  golden.json             the stage counts the reference publishes for
                          product.rad (README.md "First render" block and
                          TESTING.md tier 0), parsed from the text

The tests read only these files; nothing at test time touches the reference.
"""
import json
import os
import re
import shutil
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "scenes")


def embedded(rs_file: str, const: str) -> str:
    src = open(os.path.join(REF, "src", rs_file)).read()
    m = re.search(r"const " + const + r': &str = r#"(.*?)"#;', src, re.S)
    if not m:
        raise SystemExit(f"{const} not found in {rs_file}")
    return m.group(1)


def main() -> None:
    os.makedirs(OUT, exist_ok=True)
    for name in ("product", "cornell", "stress"):
        shutil.copyfile(os.path.join(REF, "scenes", name + ".rad"), os.path.join(OUT, name + ".rad"))
    for name in ("box_only", "cornell", "high_albedo", "sphere_only"):
        shutil.copyfile(os.path.join(REF, "scenes", "bench", name + ".rad"),
                        os.path.join(OUT, "bench_" + name + ".rad"))
    for fname, rs, const in (("closed_box.rad", "formfactor.rs", "CLOSED_BOX"),
                             ("flush_ceiling_light.rad", "trace.rs", "FLUSH_CEILING_LIGHT"),
                             ("minimal.rad", "scene.rs", "MINIMAL")):
        with open(os.path.join(OUT, fname), "w") as f:
            f.write(embedded(rs, const))

    readme = open(os.path.join(REF, "README.md")).read()
    block = readme[readme.index("interflect render scenes/product.rad"):]
    g = {}
    m = re.search(r"scene\s+(\d+) objects, (\d+) lights, (\d+) materials, (\d+) bvh nodes", block)
    g["objects"], g["lights"], g["materials"], g["bvh_nodes"] = map(int, m.groups())
    m = re.search(r"film\s+(\d+)x(\d+)", block)
    g["width"], g["height"] = map(int, m.groups())
    m = re.search(r"surfels\s+(\d+) placed of (\d+) requested", block)
    g["surfels_placed"], g["surfels_requested"] = map(int, m.groups())
    m = re.search(r"transfer\s+(\d+) clusters, (\d+) links, row-sum ([0-9.]+), ([0-9.]+)M sdf evals", block)
    g["clusters"], g["links"] = int(m.group(1)), int(m.group(2))
    g["row_sum_3dp"], g["transfer_evals_M_1dp"] = m.group(3), m.group(4)
    m = re.search(r"solve\s+(\d+) bounces, residual ([0-9.e-]+), ([0-9.]+)M sdf evals", block)
    g["bounces"], g["residual_3sf"], g["solve_evals_M_1dp"] = int(m.group(1)), m.group(2), m.group(3)
    m = re.search(r"shade\s+\d+ ms\s+([0-9.]+)M sdf evals\s+(\d+) evals/px", block)
    g["shade_evals_M_1dp"], g["evals_per_px"] = m.group(1), int(m.group(2))
    g["source"] = "reference README.md, First render (interflect 0.1.3, scenes/product.rad, defaults)"
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(g, f, indent=1)
        f.write("\n")
    print(json.dumps(g, indent=1))


if __name__ == "__main__":
    main()
