"""Regenerate the golden fixtures of this directory (run in the development container).

reference_kats.json: known answers copied, by parsing the text of the reference's own
tests, from crates/vork-render/src/path_sampler.rs:84-91 (Joe-Kuo dimension-4 direction
numbers and the first Sobol points in eighths) and
crates/vork-render/src/environment/brdf_tests.rs:97-104 (BRDF atlas texels).
display_standard.npz: Blender 5.2.1 "Standard" view samples computed directly by
OpenColorIO, read from crates/vork-render/data/device-reference.json (family "standard",
displays Display P3, Rec.2100-PQ and Rec.2100-HLG at 1000 cd/m2 peak, 100 cd/m2 white;
the reference checks its std/standard view against them in
crates/vork-render/src/display_program_tests.rs:126-150,205-235).
sampler_harness.npz: the four sampler groups of the reference's GPU parity harness
(path_sampler.rs:266-276: 64*47 invocations, index id%300 of 300, pixel
(id/300*7, id/300*13+1), stream 0x5eed, vertex id%5), computed by the oracle's
table-form sampler (path_sampler.rs:12-79), which is itself pinned by the KATs above.
"""
import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path("/root/reference/crates/vork-render/src")


def display_kats():
    data = json.loads((REF.parent / "data" / "device-reference.json").read_text())
    out = {}
    for row in data["standard"]:
        key = row["display"].replace(".", "").replace("-", "_").replace(" ", "_").lower()
        out[key + "_input"] = np.asarray([s["input"] for s in row["samples"]], np.float64)
        out[key + "_output"] = np.asarray([s["output"] for s in row["samples"]], np.float64)
    return out


def reference_kats():
    sampler = (REF / "path_sampler.rs").read_text()
    pub = re.search(r"let published = \[(.*?)\];", sampler).group(1)
    published = [int(x.strip().rstrip("u32"), 16) for x in pub.split(",")]
    exp = re.search(r"let expected = \[(\[.*?\])\];", sampler, re.S).group(1)
    points = json.loads("[" + exp + "]")
    brdf = (REF / "environment" / "brdf_tests.rs").read_text()
    block = re.search(r"for \(x, y, expected\) in \[(.*?)\] \{", brdf, re.S).group(1)
    texels = []
    for x, y, e in re.findall(r"\((\d+),\s*(\d+),\s*([^)]*?)\)", block):
        e = e.strip()
        val = 1.0 - float(np.log(2.0)) if "LN_2" in e else float(e.rstrip("."))
        texels.append([int(x), int(y), val])
    tol = float(re.search(r"\(pixel\[0\] - expected\)\.abs\(\) < ([0-9.]+)", brdf).group(1))
    return {"source": {"sobol": "crates/vork-render/src/path_sampler.rs:84-91",
                       "brdf": "crates/vork-render/src/environment/brdf_tests.rs:97-104"},
            "sobol_dim4_directions": published, "sobol_first_points_eighths": points,
            "brdf_texels": texels, "brdf_tolerance": tol}


def sampler_harness():
    sys.path.insert(0, str(HERE.parent.parent))
    from oracle import pyoracle as O
    ids = np.arange(64 * 47, dtype=np.uint32)
    index = ids % 300
    p = ids // 300
    px, py = p * 7, p * 13 + 1
    v = ids % 5
    out = {}
    for name, slot in [("camera", None), ("scatter", 0), ("light", 1), ("mesh", 2), ("environment", 3), ("decisions", 4)]:
        groups = np.zeros_like(ids) if slot is None else 1 + v * 5 + slot
        out[name] = O.sampler_bits(px, py, index, groups, 300, 0x5EED, mode=1)
    return dict(px=px, py=py, index=index, vertex=v, **out)


if __name__ == "__main__":
    (HERE / "reference_kats.json").write_text(json.dumps(reference_kats(), indent=1) + "\n")
    np.savez_compressed(HERE / "sampler_harness.npz", **sampler_harness())
    np.savez_compressed(HERE / "display_standard.npz", **display_kats())
    print("wrote", HERE / "reference_kats.json", HERE / "sampler_harness.npz", HERE / "display_standard.npz")
