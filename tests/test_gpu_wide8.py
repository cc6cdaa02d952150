"""Compressed 8-wide BLASes (VKB_BLAS_WIDE8) on the GPU: the same closest and any hits as
the 4-wide nodes and the FP64 oracle, the same images, and the batch/server rules."""
import copy

import numpy as np
import pytest

from vork_b200 import Profile, abi, scene as S
from vork_b200.serving import Server

pytestmark = pytest.mark.gpu


def _wide8(sc):
    w = copy.copy(sc)
    w.blas_format = abi.BLAS_WIDE8
    return w


def _rays(n, lo, hi, seed, reach=None):
    rng = np.random.default_rng(seed)
    org = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3)); d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = np.full((n, 1), 1e30) if reach is None else rng.uniform(*reach, (n, 1))
    return np.concatenate([org, d, tmax], 1).astype(np.float32)


@pytest.mark.parametrize("which", ["spheres", "flock"])
def test_hits_equal_the_4wide_nodes_and_the_oracle(renderer, oracle, which):
    if which == "spheres":
        sc = S.spheres_scene()
        rays, reach = _rays(20000, -2, 12, 11), _rays(20000, -2, 12, 12, (0.2, 12.0))
    else:
        sc, _ = S.flock_scene(num_birds=20000, width=64, height=36, terrain_cells=300, terrain_size=400.0)
        rays, reach = _rays(20000, (-150, 0, -150), (150, 120, 150), 13), _rays(20000, (-150, 0, -150), (150, 120, 150), 14, (1.0, 200.0))
    with renderer.install(sc) as a, renderer.install(_wide8(sc)) as b:
        t4, ids4, uv4 = a.trace(rays)
        t8, ids8, uv8 = b.trace(rays)
        occ4, occ8 = a.occluded(reach), b.occluded(reach)
    same = np.all(ids4 == ids8, axis=1)
    print(which, "8-wide vs 4-wide: closest ids equal", same.mean(), "any-hit equal", np.mean(occ4 == occ8), "hits", np.mean(ids4[:, 0] != 0xFFFFFFFF))
    # Equal-distance ties may resolve to another triangle; nothing else differs.
    assert same.mean() >= 1 - 1e-3
    assert np.array_equal(t4[same], t8[same]) and np.array_equal(uv4[same], uv8[same])
    assert np.mean(occ4 != occ8) <= 1e-3
    if which == "spheres":
        t_ref, ids_ref, _ = oracle.OracleScene(sc).trace(rays, fp64=True)
        assert np.mean(np.any(ids8 != ids_ref, axis=1)) <= 2e-3


def test_images_equal_the_4wide_nodes(renderer):
    sc = S.spheres_scene(num_spheres=24, seed=3, width=96, height=96, grid_cells=16)
    prof = Profile.reference_transport(4, 8)
    with renderer.install(sc) as a, renderer.install(_wide8(sc)) as b:
        ra, rb = a.render(prof), b.render(prof)
    close = np.all(np.abs(ra.image - rb.image) <= 1e-6 * (1 + np.abs(ra.image)), axis=-1)
    print("8-wide image: pixels equal to the 4-wide image", close.mean())
    assert close.mean() >= 0.999 and rb.stats["traversal_overflows"] == 0


def test_batches_share_a_format_and_the_server_takes_4wide(renderer):
    a_sc = S.spheres_scene(num_spheres=6, seed=5, width=32, height=32, grid_cells=8)
    b_sc = S.spheres_scene(num_spheres=8, seed=6, width=40, height=24, grid_cells=8)
    prof = Profile.reference_transport(4, 4)
    with renderer.install(_wide8(a_sc)) as a8, renderer.install(_wide8(b_sc)) as b8, renderer.install(a_sc) as a4:
        alone = [a8.render(prof).image, b8.render(prof).image]
        imgs, _ = renderer.render_batch([(a8, prof), (b8, prof)], flags=4)
        assert np.array_equal(imgs[0], alone[0]) and np.array_equal(imgs[1], alone[1])
        with pytest.raises(Exception):
            renderer.render_batch([(a8, prof), (a4, prof)], flags=4)
        with Server(renderer, max_jobs=4, wave_capacity=20000) as srv:
            with pytest.raises(Exception):
                srv.submit(a8, prof)
