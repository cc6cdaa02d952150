"""Serving: requests admitted between waves share the device; each result equals the
request rendered alone (continuous batching changes scheduling, never the image)."""
import numpy as np
import pytest

from vork_b200 import Profile, abi, scene as S
from vork_b200.serving import Server, fifo_load, poisson_load, request_mix, view

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


def test_forks_and_views_in_the_mix_equal_alone(renderer):
    # A fork owns its instances and TLAS: moving them leaves the base alone, renders the
    # same image as a fresh install of the moved scene, and requests through forks and
    # through per-request cameras equal those renders done alone.
    sc = S.spheres_scene(num_spheres=12, seed=3, width=96, height=96, grid_cells=16)
    moved = S.spheres_scene(num_spheres=12, seed=3, width=96, height=96, grid_cells=16)
    moved.instance_rows = sc.instance_rows.copy()
    moved.instance_rows[:12, 1, 3] += 0.7
    base = renderer.install(sc)
    fork = base.fork()
    try:
        before = base.render(Profile.reference_transport(4, 4)).image
        fork.update_instances(moved.instance_rows, policy=1)
        assert np.array_equal(base.render(Profile.reference_transport(4, 4)).image, before)
        with renderer.install(moved) as fresh:
            assert np.array_equal(fork.render(Profile.reference_transport(4, 4)).image,
                                  fresh.render(Profile.reference_transport(4, 4)).image)
        wide, small = view(sc.camera, 160, 90), view(sc.camera, 48, 64)
        reqs = [(base, Profile.reference_transport(4, 6), wide), (fork, Profile.reference_transport(5, 4, seed=9), small),
                (fork, Profile.reference_transport(4, 3, seed=2), None), (base, Profile.reference_transport(6, 5, seed=5), small)]
        with Server(renderer, max_jobs=4, wave_capacity=30000) as srv:
            ids = [srv.submit(*q) for q in reqs[:2]]
            srv.step()
            ids += [srv.submit(*q) for q in reqs[2:]]
            srv.run_until_idle()
            for rid, (inst, prof, cam) in zip(ids, reqs):
                img = srv.images[rid]
                alone = inst.render(prof, camera=cam).image
                assert img.shape == alone.shape and np.array_equal(img, alone)
        assert srv.images[ids[0]].shape == (90, 160, 4)
        with pytest.raises(abi.VkbError):
            base.close()                                   # a live fork keeps its base
    finally:
        fork.close()
        base.close()


def test_animated_sequences_and_the_fifo_baseline(renderer):
    # Sequences on an animated scene render frame by frame through forks; the plain FIFO
    # arm serves the same arrivals; both report every request.
    sc = S.spheres_scene(num_spheres=8, seed=1, width=64, height=64, grid_cells=8)
    rows = [sc.instance_rows.copy() for _ in range(3)]
    for f, r in enumerate(rows):
        r[:8, 1, 3] += 0.2 * f
    scenes = [renderer.install(sc), renderer.install(S.spheres_scene(num_spheres=3, seed=2, width=48, height=48, grid_cells=8))]
    try:
        reqs = request_mix(10, len(scenes), seed=4, frames=3, spp_range=(2, 4), bounces=4, pixels_range=(32 * 32, 96 * 96))
        assert any(r.frames == 3 and r.scene_index == 0 for r in reqs)
        with Server(renderer, max_jobs=8) as srv:
            a = poisson_load(srv, scenes, reqs, rate=100.0, seed=3, timeout_s=120, animations={0: rows})
        b = fifo_load(scenes, reqs, rate=100.0, seed=3, timeout_s=120, animations={0: rows})
        for res in (a, b):
            assert res["requests"] == 10 and 0 < res["p50_s"] <= res["p99_s"] and res["throughput_paths_s"] > 0
        assert a["throughput_paths_s"] > 0 and b["wall_s"] > 0
    finally:
        for s_ in scenes:
            s_.close()
