"""GPU-built BLASes (VKB_BLAS_BUILD_LBVH / _PLOC: the TLAS's Morton-ordered builders run per
mesh at install) give the same closest and any hits and the same images as the host SAH
trees, and install far faster."""
import copy

import numpy as np
import pytest

from vork_b200 import Profile, abi, scene as S

pytestmark = pytest.mark.gpu


def _built(sc, builder):
    b = copy.copy(sc)
    b.blas_builder = builder
    return b


def _rays(n, lo, hi, seed, reach=None):
    rng = np.random.default_rng(seed)
    org = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3)); d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = np.full((n, 1), 1e30) if reach is None else rng.uniform(*reach, (n, 1))
    return np.concatenate([org, d, tmax], 1).astype(np.float32)


@pytest.mark.parametrize("builder", [abi.BLAS_BUILD_LBVH, abi.BLAS_BUILD_PLOC])
@pytest.mark.parametrize("which", ["spheres", "flock"])
def test_gpu_built_blases_give_the_same_hits(renderer, which, builder):
    if which == "spheres":
        sc = S.spheres_scene()
        rays, reach = _rays(20000, -2, 12, 31), _rays(20000, -2, 12, 32, (0.2, 12.0))
    else:
        sc, _ = S.flock_scene(num_birds=20000, width=64, height=36, terrain_cells=300, terrain_size=400.0)
        rays, reach = _rays(20000, (-150, 0, -150), (150, 120, 150), 33), _rays(20000, (-150, 0, -150), (150, 120, 150), 34, (1.0, 200.0))
    with renderer.install(sc) as a, renderer.install(_built(sc, builder)) as b:
        ta, ida, uva = a.trace(rays)
        tb, idb, uvb = b.trace(rays)
        oa, ob = a.occluded(reach), b.occluded(reach)
        ia, ib = a.info(), b.info()
    same = np.all(ida == idb, axis=1)
    print(which, builder, "closest ids equal", same.mean(), "any-hit equal", np.mean(oa == ob),
          "install ms SAH", ia["install_ms"], "GPU", ib["install_ms"])
    # Equal-distance ties may resolve to another triangle; nothing else differs.
    assert same.mean() >= 1 - 1e-3
    assert np.array_equal(ta[same], tb[same]) and np.array_equal(uva[same], uvb[same])
    assert np.mean(oa != ob) <= 1e-3
    assert ib["blas_host_ms"] == 0.0


def test_gpu_built_blases_give_the_same_images(renderer):
    sc = S.spheres_scene(num_spheres=24, seed=3, width=96, height=96, grid_cells=16)
    prof = Profile.reference_transport(4, 8)
    with renderer.install(sc) as a, renderer.install(_built(sc, abi.BLAS_BUILD_PLOC)) as b:
        ra, rb = a.render(prof), b.render(prof)
    close = np.all(np.abs(ra.image - rb.image) <= 1e-6 * (1 + np.abs(ra.image)), axis=-1)
    print("GPU-built BLAS image: pixels equal to the SAH image", close.mean())
    assert close.mean() >= 0.999 and rb.stats["traversal_overflows"] == 0


def test_gpu_builders_refuse_the_8wide_format(renderer):
    sc = _built(S.spheres_scene(num_spheres=4, width=16, height=16, grid_cells=4), abi.BLAS_BUILD_LBVH)
    sc.blas_format = abi.BLAS_WIDE8
    with pytest.raises(abi.VkbError):
        renderer.install(sc)
