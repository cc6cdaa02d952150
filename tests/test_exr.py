"""Float OpenEXR output (png_output.rs:291-366): round trip of every compression, channel
naming and header attributes, no GPU."""
import struct

import numpy as np
import pytest

from vork_b200 import exr


@pytest.mark.parametrize("compression", ["none", "zips", "zip"])
def test_round_trip_is_exact(tmp_path, compression):
    rng = np.random.default_rng(3)
    h, w = 37, 53                      # ragged: the last ZIP block holds 5 scanlines
    img = rng.normal(size=(h, w, 4)).astype(np.float32)
    img[3, 4, 0] = np.inf; img[5, 6, 1] = -0.0
    ga = rng.random((h, w, 4)).astype(np.float32)
    gn = rng.normal(size=(h, w, 4)).astype(np.float32)
    path = tmp_path / f"x_{compression}.exr"
    exr.write_exr(path, exr.channels_of(img, ga, gn), compression=compression)
    ch, attrs = exr.read_exr(path)
    assert list(ch) == sorted(["A", "B", "G", "R", "guide_albedo.A", "guide_albedo.B", "guide_albedo.G", "guide_albedo.R",
                                "guide_normal.X", "guide_normal.Y", "guide_normal.Z"])
    for i, k in enumerate("RGBA"):
        assert np.array_equal(ch[k].view(np.uint32), img[..., i].view(np.uint32))
        assert np.array_equal(ch[f"guide_albedo.{k}"], ga[..., i])
    for i, k in enumerate("XYZ"):
        assert np.array_equal(ch[f"guide_normal.{k}"], gn[..., i])
    assert attrs["compression"][1][0] == exr.COMPRESSION[compression][0]
    assert attrs["vork:color_space"][1] == b"Linear Rec.709"
    assert attrs["vork:reference_domain"][1] == b"scene"
    assert struct.unpack("<8f", attrs["chromaticities"][1]) == pytest.approx(exr.REC709)


def test_header_layout_and_compression_pays(tmp_path):
    img = np.zeros((64, 64, 4), np.float32)
    img[..., 3] = 1.0
    a, b = tmp_path / "a.exr", tmp_path / "b.exr"
    exr.write_exr(a, exr.channels_of(img), compression="none")
    exr.write_exr(b, exr.channels_of(img), compression="zip")
    raw = a.read_bytes()
    assert struct.unpack_from("<ii", raw, 0) == (20000630, 2)          # magic, version 2 (scanline)
    assert b.stat().st_size < a.stat().st_size / 10
    with pytest.raises(ValueError):
        exr.write_exr(a, {"R": np.zeros((2, 2)), "G": np.zeros((3, 2))})
