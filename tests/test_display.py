"""Display stage: the std/standard oracle against the reference's OpenColorIO samples,
the PNG writer, and (GPU) the CUDA display kernel against the oracle."""
from pathlib import Path

import numpy as np
import pytest

from oracle import display as D
from vork_b200 import display as V

GOLDEN = Path(__file__).parent / "golden" / "display_standard.npz"


@pytest.mark.parametrize("key,disp,ceiling", [("display_p3", D.DISPLAY_P3, 1.0), ("rec2100_pq", D.REC2100_PQ, 0.7518271),
                                               ("rec2100_hlg", D.REC2100_HLG, 1.0)])
def test_standard_view_matches_the_reference_ocio_samples(key, disp, ceiling):
    # display_program_tests.rs:126-150,205-235: non-negative inputs, code values clamped to
    # [0, 1] (PQ to its 1000 cd/m2 code), worst error below 5e-4.
    g = np.load(GOLDEN)
    x, y = g[key + "_input"], g[key + "_output"]
    ok = (x >= 0).all(1)
    assert ok.sum() > 600
    out = np.clip(D.standard(x[ok], disp), 0.0, ceiling)
    assert np.abs(out - np.clip(y[ok], 0.0, ceiling)).max() < 5e-4


def test_srgb_standard_is_the_srgb_transfer_and_quantises_like_resolve():
    x = np.array([[0.0, 0.0031308, 0.5], [1.0, 2.0, -0.1]])
    codes = D.standard(x)
    assert np.allclose(codes[0], [0.0, 12.92 * 0.0031308, 1.055 * 0.5 ** (1 / 2.4) - 0.055])
    assert codes[1, 0] == pytest.approx(1.0) and codes[1, 2] < 0
    img = np.concatenate([x.reshape(1, 2, 3), np.ones((1, 2, 1))], -1)
    q = D.display(img, bits=8)
    assert q.dtype == np.uint8 and q[0, 1].tolist() == [255, 255, 0, 255]
    assert D.display(img, bits=16)[0, 0, 2] == round((1.055 * 0.5 ** (1 / 2.4) - 0.055) * 65535)


@pytest.mark.parametrize("bits,display", [(8, "srgb"), (16, "display_p3"), (16, "rec2100_pq")])
def test_png_round_trip_and_tags(tmp_path, bits, display):
    rng = np.random.default_rng(bits)
    codes = rng.integers(0, (1 << bits) - 1, (7, 5, 4)).astype(np.uint8 if bits == 8 else np.uint16)
    V.write_png(tmp_path / "x.png", codes, display)
    back, tags = V.read_png(tmp_path / "x.png")
    assert np.array_equal(back, codes)
    if display == "srgb":
        assert tags["sRGB"] == b"\x00" and "cICP" not in tags
    else:
        assert tags["cICP"] == V.CICP[V.DISPLAYS[display]]


@pytest.mark.gpu
@pytest.mark.parametrize("display", ["srgb", "display_p3", "rec2100_pq", "rec2100_hlg"])
def test_display_kernel_matches_the_oracle(renderer, display):
    g = np.load(GOLDEN)
    rng = np.random.default_rng(3)
    x = np.concatenate([g["display_p3_input"], rng.uniform(0, 4, (371, 3)), rng.exponential(0.2, (1000, 3))])
    img = np.concatenate([x, rng.uniform(0.2, 1, (len(x), 1))], 1).astype(np.float32).reshape(40, 50, 4)
    d = V.DISPLAYS[display]
    for kw in ({}, {"exposure": 0.5, "gamma": 1.8}):
        f = V.display(renderer, img, display, bits=32, **kw)
        fo = D.display(img, d, bits=32, **kw)
        # Finite codes agree to float precision of the transfer functions.
        assert np.allclose(f, fo, rtol=2e-5, atol=2e-6), np.abs(f - fo).max()
        q = V.display(renderer, img, display, bits=16, **kw)
        qo = D.display(img, d, bits=16, **kw)
        assert np.abs(q.astype(int) - qo.astype(int)).max() <= 1
    u = V.display(renderer, img, display, bits=8, unassociate=True)
    assert np.abs(u.astype(int) - D.display(img, d, bits=8, unassociate=True).astype(int)).max() <= 1


@pytest.mark.gpu
def test_display_rejects_bad_arguments_and_flags_nonfinite(renderer):
    from vork_b200 import abi
    img = np.zeros((2, 2, 4), np.float32)
    with pytest.raises(abi.VkbError):
        V.display(renderer, img, 9)
    img[0, 0, 1] = np.nan
    with pytest.raises(abi.VkbError) as e:
        V.display(renderer, img)
    assert e.value.status == abi.VKB_NONFINITE
