"""Display stage and image files: the resolved linear image through vkb_display (vork's
std/standard view, crates/vork-render/shaders/resolve.slang and libraries/std/standard.slang)
and a PNG writer tagged as vork tags its pictures (crates/vork-render/src/png_output.rs:184-215:
an sRGB chunk for sRGB, a cICP chunk for Display P3 and Rec.2100)."""
from __future__ import annotations

import ctypes as C
import struct
import zlib

import numpy as np

from . import abi

DISPLAYS = {"srgb": abi.DISPLAY_SRGB, "display_p3": abi.DISPLAY_P3, "rec2100_pq": abi.DISPLAY_REC2100_PQ,
            "rec2100_hlg": abi.DISPLAY_REC2100_HLG}
# cICP (colour primaries, transfer, matrix, full range) per destination (png_output.rs:184-192).
CICP = {abi.DISPLAY_P3: bytes([12, 13, 0, 1]), abi.DISPLAY_REC2100_PQ: bytes([9, 16, 0, 1]),
        abi.DISPLAY_REC2100_HLG: bytes([9, 18, 0, 1])}


def display(renderer, image: np.ndarray, display: str | int = "srgb", exposure: float = 0.0, gamma: float = 1.0,
            peak_luminance: float = 1000.0, reference_white: float = 100.0, bits: int = 8, unassociate: bool = False) -> np.ndarray:
    """(H, W, 4) linear RGBA float32 -> (H, W, 4) code values (uint8, uint16 or float32) on the GPU."""
    img = np.ascontiguousarray(image, np.float32)
    h, w = img.shape[:2]
    p = abi.VkbDisplayParams()
    p.display = DISPLAYS[display] if isinstance(display, str) else int(display)
    p.exposure, p.gamma, p.peak_luminance, p.reference_white = exposure, gamma, peak_luminance, reference_white
    p.bits, p.unassociate = bits, 1 if unassociate else 0
    out = np.empty((h, w, 4), {8: np.uint8, 16: np.uint16, 32: np.float32}[bits])
    abi.check(renderer.lib.vkb_display(renderer.h, C.byref(p), img.ctypes.data_as(C.c_void_p), 0, w, h,
                                       out.ctypes.data_as(C.c_void_p), 0))
    return out


def _chunk(kind: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data) & 0xFFFFFFFF)


def png_bytes(codes: np.ndarray, display: str | int = "srgb") -> bytes:
    """An RGBA PNG of 8- or 16-bit code values, tagged for its display."""
    codes = np.ascontiguousarray(codes)
    h, w, ch = codes.shape
    assert ch == 4 and codes.dtype in (np.uint8, np.uint16)
    depth = 8 if codes.dtype == np.uint8 else 16
    disp = DISPLAYS[display] if isinstance(display, str) else int(display)
    raw = codes.astype(">u2").tobytes() if depth == 16 else codes.tobytes()
    stride = w * 4 * depth // 8
    rows = b"".join(b"\x00" + raw[y * stride:(y + 1) * stride] for y in range(h))
    out = [b"\x89PNG\r\n\x1a\n", _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, 6, 0, 0, 0))]
    out.append(_chunk(b"cICP", CICP[disp]) if disp in CICP else _chunk(b"sRGB", b"\x00"))
    out += [_chunk(b"IDAT", zlib.compress(rows, 6)), _chunk(b"IEND", b"")]
    return b"".join(out)


def write_png(path, codes: np.ndarray, display: str | int = "srgb") -> None:
    with open(path, "wb") as f:
        f.write(png_bytes(codes, display))


def read_png(path_or_bytes) -> tuple[np.ndarray, dict]:
    """Read back an RGBA PNG written by png_bytes (filter type 0 rows): codes and chunk tags."""
    data = path_or_bytes if isinstance(path_or_bytes, bytes) else open(path_or_bytes, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, tags = 8, b"", {}
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        if zlib.crc32(kind + body) & 0xFFFFFFFF != struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]:
            raise ValueError(f"bad CRC in {kind!r}")
        if kind == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
        elif kind == b"IDAT":
            idat += body
        else:
            tags[kind.decode()] = body
        pos += 12 + n
    raw = zlib.decompress(idat)
    stride = w * 4 * depth // 8
    rows = [raw[y * (stride + 1) + 1:(y + 1) * (stride + 1)] for y in range(h)]
    assert all(raw[y * (stride + 1)] == 0 for y in range(h))
    arr = np.frombuffer(b"".join(rows), ">u2" if depth == 16 else np.uint8).reshape(h, w, 4)
    return arr.astype(np.uint16 if depth == 16 else np.uint8), tags
