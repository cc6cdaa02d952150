"""TLAS leaf boxes (CPU): the world box of an instance is the box of its mesh box's 8
transformed corners intersected with the box of its transformed bounding sphere.  The
oracle restates that computation bit for bit (the GPU TLAS Morton codes are checked
against it), so these checks on the oracle's boxes hold for the build's."""
import numpy as np

from vork_b200 import scene


def _random_rows(rng, n, max_translate):
    """(n, 3, 4) float32 object->world rows: random rotation, non-uniform scale and shear
    from a random matrix, translation up to max_translate."""
    rows = np.empty((n, 3, 4), np.float32)
    for i in range(n):
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        lin = q @ np.diag(rng.uniform(0.02, 8.0, 3)) @ (np.eye(3) + 0.3 * rng.normal(size=(3, 3)))
        rows[i, :, :3] = lin
        rows[i, :, 3] = rng.uniform(-max_translate, max_translate, 3)
    return rows


def _scene(rng, n_inst, max_translate):
    meshes = [scene.geodesic_sphere(3, jitter=0.2, seed=1), scene.uv_sphere(1.0, 12, 6)]
    long = scene.geodesic_sphere(2, jitter=0.0, seed=2)
    long.positions = (long.positions * np.array([0.2, 0.2, 3.0], np.float32) + np.array([5.0, -1.0, 2.0], np.float32)).astype(np.float32)
    meshes.append(long)
    rows = _random_rows(rng, n_inst, max_translate)
    mesh_ids = (np.arange(n_inst) % len(meshes)).astype(np.uint32)
    cam = scene.look_at(eye=(0.0, 0.0, -10.0), target=(0.0, 0.0, 0.0), width=8, height=8)
    return scene.Scene(meshes, rows, mesh_ids, np.zeros(n_inst, np.uint32), [scene.material()], [], cam, scene.environment())


def _world_vertices(sc, i):
    m = sc.meshes[int(sc.instance_mesh[i])]
    r = sc.instance_rows[i].astype(np.float64)
    return m.positions.astype(np.float64) @ r[:, :3].T + r[:, 3]


def test_instance_boxes_contain_their_transformed_meshes(oracle):
    rng = np.random.default_rng(11)
    for max_translate in (1.0, 1e3):
        sc = _scene(rng, 300, max_translate)
        lo, hi = oracle.OracleScene(sc, fp32=True, fp64=False).instance_boxes()
        for i in range(len(sc.instance_mesh)):
            w = _world_vertices(sc, i)
            # fp32 corners of the mesh box may round by an ulp; the sphere part is widened.
            slack = 2.0 ** -22 * np.maximum(np.abs(w).max(0), 1.0)
            assert (w.min(0) >= lo[i].astype(np.float64) - slack).all(), (max_translate, i)
            assert (w.max(0) <= hi[i].astype(np.float64) + slack).all(), (max_translate, i)


def test_sphere_term_tightens_rotated_round_meshes(oracle):
    # For round meshes under rotation the transformed sphere's box is well inside the box
    # of the rotated mesh box; the exact box of the transformed vertices bounds it below.
    rng = np.random.default_rng(12)
    sc = _scene(rng, 300, 10.0)
    lo, hi = oracle.OracleScene(sc, fp32=True, fp64=False).instance_boxes()
    area = lambda e: e[:, 0] * e[:, 1] + e[:, 1] * e[:, 2] + e[:, 2] * e[:, 0]
    round_ids = [i for i in range(len(sc.instance_mesh)) if sc.instance_mesh[i] == 0]
    corners_area, built_area, exact_area = [], [], []
    for i in round_ids:
        m = sc.meshes[0]
        r = sc.instance_rows[i].astype(np.float64)
        blo, bhi = m.positions.min(0).astype(np.float64), m.positions.max(0).astype(np.float64)
        c = np.array([[x, y, z] for x in (blo[0], bhi[0]) for y in (blo[1], bhi[1]) for z in (blo[2], bhi[2])]) @ r[:, :3].T + r[:, 3]
        w = _world_vertices(sc, i)
        corners_area.append(area((c.max(0) - c.min(0))[None])[0])
        built_area.append(area((hi[i] - lo[i]).astype(np.float64)[None])[0])
        exact_area.append(area((w.max(0) - w.min(0))[None])[0])
    corners_area, built_area, exact_area = map(np.asarray, (corners_area, built_area, exact_area))
    assert (built_area <= corners_area * (1 + 1e-5)).all()
    assert (built_area >= exact_area * (1 - 1e-5)).all()
    assert built_area.mean() < 0.9 * corners_area.mean()
