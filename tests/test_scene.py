"""Synthetic generators: std tessellation rules, determinism, winding (CPU only)."""
import numpy as np

from vork_b200 import scene


def _face_normals(m):
    p = m.positions.astype(np.float64)
    i = m.indices
    return np.cross(p[i[:, 1]] - p[i[:, 0]], p[i[:, 2]] - p[i[:, 0]])


def test_uv_sphere_matches_std_tessellation():
    m = scene.uv_sphere()
    assert m.num_triangles == 960 and m.positions.shape[0] == 17 * 33
    n = _face_normals(m)
    c = m.positions[m.indices].mean(1)
    assert np.all(np.einsum("ij,ij->i", n, c) > 0)  # outward counter-clockwise


def test_grid_faces_up_and_counts():
    g = scene.grid((10.0, 10.0), (64, 64))
    assert g.num_triangles == 8192
    assert np.all(_face_normals(g)[:, 1] > 0)


def test_geodesic_sphere_has_500_outward_triangles():
    m = scene.geodesic_sphere(5, jitter=0.1, seed=3)
    assert m.num_triangles == 500
    c = m.positions[m.indices].mean(1)
    assert np.all(np.einsum("ij,ij->i", _face_normals(m), c) > 0)


def test_spheres_scene_is_deterministic_and_in_range():
    a, b = scene.spheres_scene(), scene.spheres_scene()
    assert np.array_equal(a.instance_rows, b.instance_rows)
    rows = a.instance_rows[:64]
    assert np.all((rows[:, :, 3] >= 0) & (rows[:, :, 3] <= 10))
    assert np.all((rows[:, 0, 0] >= 0.2) & (rows[:, 0, 0] <= 1.0))
    metal = np.array([m.base_metalness for m in a.materials[:64]])
    assert set(np.unique(metal)) <= {0.0, 1.0} and 5 <= metal.sum() <= 35
    assert a.num_triangles == 64 * 960 + 8192
    l = a.lights[0]
    area = np.linalg.norm(np.cross(l.emitter_u[:3], l.emitter_v[:3]))
    assert abs(l.radiance[0] / (np.pi * area) - 20.0) < 1e-4


def test_pcg32_reference_sequence():
    # O'Neill's pcg32-demo with seed 42, sequence 54 starts 0xa15c02b7, 0x7b47f409.
    r = scene.Pcg32(42, 54)
    assert [r.next_u32() for _ in range(2)] == [0xA15C02B7, 0x7B47F409]
