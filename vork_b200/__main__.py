"""`python -m vork_b200 render scene.json --out image.png`: the std/path route of
`vork render scene.json --profile std/path --out x.png` for the supported scene subset
(scene_json.py): load, install, path-trace on the GPU, display transform (std/standard),
PNG.  `--linear out.npy` also keeps the linear RGBA mean; `--exr out.exr` writes it as a
float OpenEXR (png_output.rs:291-366), with the denoiser guide planes when `--guides`."""
from __future__ import annotations

import argparse
import sys

import numpy as np

from . import Profile, Renderer, display, exr, scene_json


def render_command(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m vork_b200 render", description=__doc__)
    ap.add_argument("scene", help="scene document (version 2)")
    ap.add_argument("--out", required=True, help="PNG path")
    ap.add_argument("--samples", type=int, default=Profile.samples)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--depth", type=int, default=None, help="every bounce budget = depth (the reference's test hook)")
    ap.add_argument("--width", type=int, default=None)
    ap.add_argument("--height", type=int, default=None)
    ap.add_argument("--display", default="srgb", choices=sorted(display.DISPLAYS))
    ap.add_argument("--exposure", type=float, default=0.0)
    ap.add_argument("--gamma", type=float, default=1.0)
    ap.add_argument("--bits", type=int, default=8, choices=[8, 16])
    ap.add_argument("--linear", default=None, help="also save the linear RGBA mean (.npy)")
    ap.add_argument("--exr", default=None, help="also write the linear RGBA mean as a float OpenEXR")
    ap.add_argument("--guides", action="store_true", help="with --exr: add the denoiser guide planes")
    ap.add_argument("--exr-compression", default="zip", choices=sorted(exr.COMPRESSION))
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    sc = scene_json.load(a.scene, a.width, a.height)
    prof = Profile.reference_transport(a.depth, a.samples, seed=a.seed) if a.depth else Profile(samples=a.samples, seed=a.seed)
    with Renderer(a.device) as r, r.install(sc) as s:
        res = s.render(prof, guides=bool(a.exr and a.guides))
        codes = display.display(r, res.image, a.display, a.exposure, a.gamma, bits=a.bits)
    display.write_png(a.out, codes, a.display)
    if a.linear:
        np.save(a.linear, res.image)
    if a.exr:
        exr.write_exr(a.exr, exr.channels_of(res.image, res.guide_albedo, res.guide_normal), compression=a.exr_compression)
    st = res.stats
    print(f"{a.out}: {sc.camera.width}x{sc.camera.height}, {a.samples} spp, {st['paths'] / max(st['render_ms'], 1e-6) / 1e3:.1f} M paths/s",
          file=sys.stderr)
    return 0


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv or argv[0] != "render":
        print("usage: python -m vork_b200 render scene.json --out image.png [options]", file=sys.stderr)
        return 2
    return render_command(argv[1:])


if __name__ == "__main__":
    sys.exit(main())
