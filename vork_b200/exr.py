"""Scene-linear OpenEXR output of a render: the reference's float EXR path
(crates/vork-render/src/png_output.rs:291-366, encode_exr_clock / write_exr).

The beauty image goes in the default layer as R, G, B, A; every other plane is
`<name>.<channel>` (the denoiser guides as guide_albedo.{R,G,B,A} and
guide_normal.{X,Y,Z}, depth as Z).  Channels are 32-bit float, sorted by name as
OpenEXR requires; the header names the storage colour (chromaticities of the Rec.709
primaries and D65 white, `vork:color_space` "Linear Rec.709",
`vork:reference_domain` "scene").  Compression: NONE, ZIPS (one scanline per zlib
block) or ZIP (16 scanlines per block, the reference's default codec) with OpenEXR's
predictor and byte interleave.  Written from the file format's published layout
(magic, version, attribute header, line offset table, scanline chunks).
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

MAGIC = 20000630
COMPRESSION = {"none": (0, 1), "zips": (2, 1), "zip": (3, 16)}
REC709 = (0.64, 0.33, 0.30, 0.60, 0.15, 0.06, 0.3127, 0.3290)


def _attr(name: str, kind: str, data: bytes) -> bytes:
    return name.encode() + b"\0" + kind.encode() + b"\0" + struct.pack("<i", len(data)) + data


def _text(s: str) -> bytes:
    return s.encode()


def _predict_interleave(raw: bytes) -> bytes:
    """OpenEXR's ZIP preconditioning: split even/odd bytes, then delta-code the bytes."""
    b = np.frombuffer(raw, np.uint8)
    t = np.concatenate([b[0::2], b[1::2]])
    d = t.astype(np.int16)
    d[1:] = (t[1:].astype(np.int16) - t[:-1].astype(np.int16) + 128) & 0xFF
    return d.astype(np.uint8).tobytes()


def _unpredict_deinterleave(data: bytes) -> bytes:
    d = np.frombuffer(data, np.uint8).astype(np.int64)
    steps = np.concatenate([d[:1], d[1:] - 128])
    t = (np.cumsum(steps) & 0xFF).astype(np.uint8)
    half = (len(t) + 1) // 2
    out = np.empty(len(t), np.uint8)
    out[0::2] = t[:half]
    out[1::2] = t[half:]
    return out.tobytes()


def channels_of(image: np.ndarray, guide_albedo=None, guide_normal=None, depth=None) -> dict:
    """The channel planes of a render result: beauty RGBA, optional guides and depth."""
    ch = {k: image[..., i] for i, k in enumerate("RGBA")}
    if guide_albedo is not None:
        ch.update({f"guide_albedo.{k}": guide_albedo[..., i] for i, k in enumerate("RGBA")})
    if guide_normal is not None:
        ch.update({f"guide_normal.{k}": guide_normal[..., i] for i, k in enumerate("XYZ")})
    if depth is not None:
        ch["Z"] = depth
    return ch


def write_exr(path, channels: dict, compression: str = "zip", color_space: str = "Linear Rec.709",
              reference_domain: str = "scene") -> None:
    """Write `channels` ({name: (H, W) float array}, all the same size) as one float layer."""
    if compression not in COMPRESSION:
        raise ValueError(f"compression must be one of {sorted(COMPRESSION)}")
    names = sorted(channels)
    if not names:
        raise ValueError("no channels")
    planes = [np.ascontiguousarray(channels[n], np.float32) for n in names]
    h, w = planes[0].shape
    if any(p.shape != (h, w) for p in planes):
        raise ValueError("channel size mismatch")
    code, lines = COMPRESSION[compression]
    chlist = b"".join(n.encode() + b"\0" + struct.pack("<iB3xii", 2, 0, 1, 1) for n in names) + b"\0"
    box = struct.pack("<iiii", 0, 0, w - 1, h - 1)
    header = struct.pack("<ii", MAGIC, 2)
    header += _attr("channels", "chlist", chlist)
    header += _attr("chromaticities", "chromaticities", struct.pack("<8f", *REC709))
    header += _attr("compression", "compression", bytes([code]))
    header += _attr("dataWindow", "box2i", box)
    header += _attr("displayWindow", "box2i", box)
    header += _attr("lineOrder", "lineOrder", bytes([0]))
    header += _attr("pixelAspectRatio", "float", struct.pack("<f", 1.0))
    header += _attr("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0))
    header += _attr("screenWindowWidth", "float", struct.pack("<f", 1.0))
    header += _attr("vork:color_space", "string", _text(color_space))
    header += _attr("vork:reference_domain", "string", _text(reference_domain))
    header += b"\0"
    stack = np.stack(planes, 1)          # (H, C, W): per scanline, each channel's run of pixels
    chunks = []
    for y0 in range(0, h, lines):
        raw = stack[y0:y0 + lines].tobytes()
        if code != 0:
            packed = zlib.compress(_predict_interleave(raw), 6)
            raw = packed if len(packed) < len(raw) else raw
        chunks.append(struct.pack("<ii", y0, len(raw)) + raw)
    table_at = len(header)
    offsets, at = [], table_at + 8 * len(chunks)
    for c in chunks:
        offsets.append(at)
        at += len(c)
    with open(path, "wb") as f:
        f.write(header)
        f.write(struct.pack(f"<{len(offsets)}Q", *offsets))
        for c in chunks:
            f.write(c)


def read_exr(path) -> tuple[dict, dict]:
    """(channels, attributes) of a scanline float EXR written by write_exr (test reader)."""
    data = open(path, "rb").read()
    magic, version = struct.unpack_from("<ii", data, 0)
    if magic != MAGIC:
        raise ValueError("not an OpenEXR file")
    at, attrs = 8, {}
    while data[at] != 0:
        e = data.index(b"\0", at); name = data[at:e].decode(); at = e + 1
        e = data.index(b"\0", at); kind = data[at:e].decode(); at = e + 1
        (size,) = struct.unpack_from("<i", data, at); at += 4
        attrs[name] = (kind, data[at:at + size]); at += size
    at += 1
    raw_ch = attrs["channels"][1]
    names, p = [], 0
    while raw_ch[p] != 0:
        e = raw_ch.index(b"\0", p); names.append(raw_ch[p:e].decode()); p = e + 1 + 16
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    code = attrs["compression"][1][0]
    lines = {0: 1, 2: 1, 3: 16}[code]
    n_chunks = (h + lines - 1) // lines
    offsets = struct.unpack_from(f"<{n_chunks}Q", data, at)
    out = np.empty((h, len(names), w), np.float32)
    for off in offsets:
        y, size = struct.unpack_from("<ii", data, off)
        body = data[off + 8:off + 8 + size]
        n_lines = min(lines, h - y)
        expect = n_lines * len(names) * w * 4
        if code != 0 and size < expect:
            body = _unpredict_deinterleave(zlib.decompress(body))
        out[y:y + n_lines] = np.frombuffer(body, np.float32).reshape(n_lines, len(names), w)
    attributes = {k: v for k, v in attrs.items()}
    return {n: out[:, i, :] for i, n in enumerate(names)}, attributes
