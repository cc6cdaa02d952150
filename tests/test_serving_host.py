"""Host logic of the serving driver (no GPU): the request mix and per-request views."""
import numpy as np

from vork_b200 import scene as S
from vork_b200.serving import request_mix, view


def test_request_mix_resolutions_and_sequences():
    reqs = request_mix(2000, 6, seed=1, frames=24, spp_range=(8, 128), bounces=8, pixels_range=(256 * 256, 1920 * 1080))
    px = np.array([r.width * r.height for r in reqs], np.float64)
    assert all(16 <= r.width <= 1920 and 16 <= r.height <= 1080 for r in reqs)
    assert px.min() >= 0.9 * 256 * 256 * 0.56 and px.max() <= 1920 * 1080
    # log-uniform pixel counts: the median sits near the geometric mean of the range
    assert abs(np.log(np.median(px)) - 0.5 * np.log(256 * 256 * 1920 * 1080)) < 0.35
    seq = np.mean([r.frames == 24 for r in reqs])
    assert 0.17 < seq < 0.23 and all(r.frames in (1, 24) for r in reqs)
    spp = np.array([r.profile.samples for r in reqs])
    assert spp.min() >= 8 and spp.max() <= 128
    assert set(r.scene_index for r in reqs) == set(range(6))
    again = request_mix(2000, 6, seed=1, frames=24, spp_range=(8, 128), bounces=8, pixels_range=(256 * 256, 1920 * 1080))
    assert [(r.width, r.height, r.frames, r.profile.seed) for r in reqs] == [(r.width, r.height, r.frames, r.profile.seed) for r in again]


def test_view_keeps_the_vertical_field_of_view():
    cam = S.look_at((0, 1, -5), (0, 0, 0), fov_y_degrees=40, width=1920, height=1080)
    v = view(cam, 640, 640)
    assert (v.width, v.height) == (640, 640)
    assert v.proj_y == cam.proj_y and abs(v.proj_x - cam.proj_y) < 1e-6
    assert list(v.eye) == list(cam.eye) and list(v.forward) == list(cam.forward)
    assert (cam.width, cam.height) == (1920, 1080)          # the scene's own camera is untouched
