"""ORACLE (test infrastructure only): CPU restatement of the display stage used by the
tests to check the CUDA display kernel (vork_b200/csrc/vkb_display.cuh).  The product
never imports this module.

Follows the reference's std/standard view (libraries/std/standard.slang:1-33) with the
encodings of libraries/std/view.slang:3-41 (sRGB, ST 2084, BT.2100 HLG), for a linear
Rec.709 working space (view_linear_rec709, view.slang:44-63, is the identity there),
and the resolve stage's unorm quantisation (crates/vork-render/shaders/resolve.slang:13)
and unassociated display colour (resolve.slang:140-145).  Pinned by the reference's
direct OpenColorIO samples (tests/golden/display_standard.npz).
"""
from __future__ import annotations

import numpy as np

SRGB, DISPLAY_P3, REC2100_PQ, REC2100_HLG = 0, 1, 2, 3
TO_P3 = np.array([[.82246197, .17753803, 0.], [.03319420, .96680580, 0.], [.01708263, .07239744, .91051993]])
TO_2020 = np.array([[.62740390, .32928304, .04331307], [.06909729, .91954040, .01136232], [.01639144, .08801331, .89559525]])


def encode_srgb(c):   # view.slang:7-9
    c = np.asarray(c, np.float64)
    return np.where(c > .0031308, 1.055 * np.power(np.maximum(c, 0.), 1. / 2.4) - .055, 12.92 * c)


def decode_srgb(c):   # view.slang:3-5
    c = np.asarray(c, np.float64)
    return np.where(c > .04045, np.power(np.maximum((c + .055) / 1.055, 0.), 2.4), c / 12.92)


def encode_pq(nits):  # view.slang:11-14
    l = np.power(np.maximum(nits, 0.) / 10000., .1593017578125)
    return np.power((.8359375 + 18.8515625 * l) / (1. + 18.6875 * l), 78.84375)


def encode_hlg(nits, peak):  # view.slang:18-25
    relative = peak / 1000.
    gamma = 1.2 + .42 * .30102999566 * np.log2(relative) if 400. <= peak <= 2000. else 1.2 * 1.111 ** np.log2(relative)
    light = np.maximum(nits, 0.) / peak
    y = np.maximum(light @ np.array([.2627, .6780, .0593]), 1e-4 / 3. ** gamma)
    scene = light * np.power(y, (1. - gamma) / gamma)[..., None]
    return np.where(scene <= 1. / 12., np.sqrt(3. * np.maximum(scene, 0.)),
                    .17883277 * np.log(np.maximum(12. * scene - .28466892, .000001)) + .55991073)


def standard(rgb, display=SRGB, exposure=0.0, gamma=1.0, peak=1000.0, white=100.0):
    """std/standard (standard.slang:24-33): linear Rec.709 (n, 3) -> display code values."""
    c = np.asarray(rgb, np.float64) * 2.0 ** exposure
    mapped = encode_srgb(c)
    if display == SRGB:
        if gamma != 1.0:
            mapped = np.power(np.maximum(mapped, 0.), 1. / gamma)
        return mapped
    if gamma != 1.0:
        c = decode_srgb(np.power(np.maximum(mapped, 0.), 1. / gamma))
    if display == DISPLAY_P3:
        return encode_srgb(c @ TO_P3.T)
    nits = np.clip(c @ TO_2020.T * white, 0., peak)
    return encode_pq(nits) if display == REC2100_PQ else encode_hlg(nits, peak)


def display(rgba, display=SRGB, exposure=0.0, gamma=1.0, peak=1000.0, white=100.0, bits=8, unassociate=False):
    """Linear RGBA (h, w, 4) -> quantised code values: unorm round(saturate(v) * (2^bits - 1)),
    alpha passed through the same quantisation; bits 32 returns float codes."""
    img = np.asarray(rgba, np.float64)
    rgb = img[..., :3].copy()
    a = img[..., 3:4]
    if unassociate:
        rgb = np.where(a > 0., rgb / np.where(a > 0., a, 1.), rgb)
    codes = standard(rgb.reshape(-1, 3), display, exposure, gamma, peak, white).reshape(rgb.shape)
    out = np.concatenate([codes, a], -1)
    if bits == 32:
        return out.astype(np.float32)
    scale = float((1 << bits) - 1)
    q = np.round(np.clip(out, 0., 1.) * scale)
    return q.astype(np.uint8 if bits == 8 else np.uint16)
