"""Serving: requests admitted between waves share the device; each result equals the
request rendered alone (continuous batching changes scheduling, never the image)."""
import numpy as np
import pytest

from vork_b200 import Profile, abi, scene as S
from vork_b200.serving import Server, poisson_load, request_mix

pytestmark = pytest.mark.gpu


def _scenes(renderer):
    out = []
    for k, (w, h, n) in enumerate([(96, 64, 3), (160, 120, 20), (64, 64, 1)]):
        out.append(renderer.install(S.spheres_scene(num_spheres=n, seed=k, width=w, height=h, grid_cells=16)))
    return out


def test_requests_in_the_mix_equal_alone(renderer):
    scenes = _scenes(renderer)
    try:
        reqs = [(scenes[0], Profile.reference_transport(4, 8)), (scenes[1], Profile.reference_transport(6, 12, seed=4)),
                (scenes[2], Profile.reference_transport(8, 5)), (scenes[1], Profile.reference_transport(5, 3, seed=11)),
                (scenes[0], Profile.reference_transport(4, 16, seed=2))]
        with Server(renderer, max_jobs=3, wave_capacity=40000) as srv:
            ids = [srv.submit(*reqs[0]), srv.submit(*reqs[1])]
            srv.step()                                   # two running, the next arrive mid-flight
            ids += [srv.submit(*reqs[2]), srv.submit(*reqs[3])]
            srv.step()
            ids.append(srv.submit(*reqs[4]))
            srv.run_until_idle()
            assert all(srv.state(i) == 2 for i in ids)
            for rid, (inst, prof) in zip(ids, reqs):
                assert np.array_equal(srv.images[rid], inst.render(prof).image)
    finally:
        for s in scenes:
            s.close()


def test_memory_budget_admission_and_rejection(renderer):
    scenes = _scenes(renderer)
    try:
        cap = 160 * 120  # one sample of the larger scene per wave: requests span several waves
        with Server(renderer, memory_budget_bytes=1 << 40, max_jobs=8, wave_capacity=cap) as big:
            wave = big.step()["used_bytes"]
        budget = wave + scenes[1].info()["scene_bytes"] + 160 * 120 * 32 + 4096   # room for one of the larger requests
        with Server(renderer, memory_budget_bytes=budget, max_jobs=8, wave_capacity=cap) as srv:
            a = srv.submit(scenes[1], Profile.reference_transport(4, 4))
            b = srv.submit(scenes[1], Profile.reference_transport(4, 4, seed=3))
            st = srv.step()
            assert st["running"] == 1 and st["queued"] == 1 and st["peak_bytes"] <= budget
            srv.run_until_idle()
            assert srv.state(a) == 2 and srv.state(b) == 2
            huge = S.spheres_scene(num_spheres=2, width=2048, height=2048)
            with renderer.install(huge) as h:
                with pytest.raises(abi.VkbError):
                    srv.submit(h, Profile.reference_transport(4, 1))
    finally:
        for s in scenes:
            s.close()


def test_poisson_load_reports_latency(renderer):
    scenes = _scenes(renderer)
    try:
        reqs = request_mix(12, len(scenes), seed=1, frames=3, spp_range=(2, 6), bounces=4)
        with Server(renderer, max_jobs=16) as srv:
            r = poisson_load(srv, scenes, reqs, rate=50.0, seed=2, timeout_s=120)
        assert r["requests"] == 12 and 0 < r["p50_s"] <= r["p99_s"] and r["throughput_paths_s"] > 0
    finally:
        for s in scenes:
            s.close()
