"""Batched previews: many jobs share one wavefront (vkb_render_batch) with results
equal to rendering each job alone; the autotuner picks a wave shape."""
import numpy as np
import pytest

from vork_b200 import Profile, scene as S

pytestmark = pytest.mark.gpu


def _jobs(renderer, count, seed=3, max_side=192):
    items = []
    for sc, spp, depth in S.preview_jobs(count, seed=seed, max_side=max_side):
        items.append((renderer.install(sc), Profile.reference_transport(depth, spp)))
    return items


def test_batch_results_equal_single_renders(renderer):
    items = _jobs(renderer, 6)
    try:
        images, stats = renderer.render_batch(items)
        assert stats["paths"] == sum(i.scene.camera.width * i.scene.camera.height * p.samples for i, p in items)
        assert stats["traversal_overflows"] == 0
        for (inst, prof), img in zip(items, images):
            alone = inst.render(prof).image
            assert np.array_equal(img, alone)
        # The same scene twice in one batch, with different sample ranges and seeds.
        inst, prof = items[0]
        a = Profile.reference_transport(prof.bounces[0], prof.samples, sample_count=2)
        b = Profile.reference_transport(prof.bounces[0], prof.samples, seed=9)
        (ia, ib), _ = renderer.render_batch([(inst, a), (inst, b)])
        (fa, fb), _ = renderer.render_batch([(inst, a), (inst, b)], flags=4)
        assert np.array_equal(fa, ia) and np.array_equal(fb, ib)
        assert np.array_equal(ia, inst.render(a).image) and np.array_equal(ib, inst.render(b).image)
    finally:
        for inst, _ in items:
            inst.close()


def test_autotune_picks_a_candidate_and_keeps_results(renderer):
    items = _jobs(renderer, 3, seed=5, max_side=128)
    try:
        before = [inst.render(p).image for inst, p in items]
        r = renderer.autotune(items)
        assert r["best_ms"] > 0 and len(r["tried"]) == 15   # 5 capacities x 3 grids
        assert r["best_capacity"] in [c for c, _, _ in r["tried"]]
        after, _ = renderer.render_batch(items)
        for x, y in zip(before, after):
            assert np.array_equal(x, y)
    finally:
        for inst, _ in items:
            inst.close()


def test_overlapped_batch_waves_equal_one_stream(renderer):
    # Jobs of 2^25 paths and more take several waves of the default 32 Mi-slot wavefront:
    # their waves alternate between two streams, and every image equals the one-stream run.
    from vork_b200 import abi
    items = []
    for k, (side, spp) in enumerate([(1024, 16), (768, 24), (512, 40)]):
        sc = S.spheres_scene(num_spheres=16, seed=20 + k, width=side, height=side, grid_cells=8)
        items.append((renderer.install(sc), Profile.reference_transport(4, spp)))
    try:
        a, sa = renderer.render_batch(items)
        b, sb = renderer.render_batch(items, flags=abi.PROFILE_SERIAL_WAVES)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
        assert sa["extension_rays"] == sb["extension_rays"] and sa["shadow_rays"] == sb["shadow_rays"]
    finally:
        for inst, _ in items:
            inst.close()
