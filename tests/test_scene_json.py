"""The scene-document loader (vork scene v2 subset) against hand-computed expectations, and
(GPU) a loaded document rendered against the oracle."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from vork_b200 import Profile, scene as S, scene_json as J

FIXTURE = Path(__file__).parent / "golden" / "scene_subset.json"


def _doc():
    return json.loads(FIXTURE.read_text())


def test_loads_meshes_instances_and_materials():
    sc = J.load(FIXTURE)
    # floor, 3 instanced balls, cube, plate; four distinct meshes (grid, sphere, box, buffer triangle)
    assert len(sc.instance_rows) == 6 and len(sc.meshes) == 4
    assert sc.meshes[1].num_triangles == S.uv_sphere(1.0, 24, 12).num_triangles
    assert np.array_equal(sc.meshes[1].positions, S.uv_sphere(1.0, 24, 12).positions)
    assert sc.meshes[0].num_triangles == 2 * 8 * 8
    # Instance world = group TRS x instance TRS (group: translate (0,0.2,-1), yaw 0.5).
    g = np.eye(4); g[:3, :3] = J.euler_matrix([0, 0.5, 0]); g[:3, 3] = [0, 0.2, -1]
    inst = np.eye(4); inst[:3, :3] = J.quat_matrix([0, 0.3826834, 0, 0.9238795]) * 0.4; inst[:3, 3] = [0, 0.5, 0]
    assert np.allclose(sc.instance_rows[2], (g @ inst)[:3], atol=1e-6)
    # Materials: named ones shared, the inline one double-sided; default material on the plate.
    mats = [sc.materials[i] for i in sc.instance_material]
    assert mats[1].base_metalness == 1.0 and mats[1].specular_roughness == pytest.approx(0.25)
    assert mats[4].flags == 2 and list(mats[4].base_color) == pytest.approx([0.2, 0.5, 0.8])
    assert list(mats[5].base_color) == pytest.approx([0.8, 0.8, 0.8]) and mats[5].specular_roughness == pytest.approx(0.3)
    # A buffer mesh without normals gets its face normal (winding 0, 2, 1 faces +y).
    assert np.allclose(sc.meshes[3].normals, [[0, 1, 0]] * 3)


def test_camera_is_std_camera_aimed_at_its_target():
    sc = J.load(FIXTURE)
    c = sc.camera
    eye, fwd = np.array(c.eye), np.array(c.forward)
    want = np.array([0, 0.5, 0]) - np.array([4, 3, 6])
    assert np.allclose(fwd, want / np.linalg.norm(want), atol=1e-6)
    assert abs(np.dot(c.right, [0, 1, 0])) < 1e-6 and np.allclose(np.cross(c.right, c.up), -fwd, atol=1e-6)
    # camera.slang:25-31 at aspect 4/3, lens 35, 36 mm sensor: height = 36 / (4/3).
    aspect = 160 / 120
    assert c.proj_y == pytest.approx(2 * 35 / (36 / aspect)) and c.proj_x == pytest.approx(c.proj_y / aspect)
    assert (c.width, c.height) == (160, 120) and c.near_plane == pytest.approx(0.1)


def test_lights_follow_the_reference_evaluation():
    sc = J.load(FIXTURE)
    key, sun, bulb, spot = sc.lights
    # rectangle: kind 3, radiance = colour x energy, emitter axes = frame axes x size, aimed at the origin
    assert key.position[3] == 3.0 and list(key.radiance[:3]) == pytest.approx([700, 644, 560])
    d = -np.array([-3.0, 5.0, 4.0]); d /= np.linalg.norm(d)
    assert np.allclose(key.direction[:3], d, atol=1e-6)
    assert np.linalg.norm(key.emitter_u[:3]) == pytest.approx(4.0) and np.linalg.norm(key.emitter_v[:3]) == pytest.approx(2.0)
    assert key.params[1] == pytest.approx(0.5 * math.sqrt(16 + 4)) and key.direction[3] == pytest.approx(math.cos(math.pi / 4))
    # sun: kind 0, default angle 0.526 deg -> half angle; energy as irradiance
    assert sun.position[3] == 0.0 and sun.params[1] == pytest.approx(math.radians(0.526) / 2)
    assert list(sun.radiance[:3]) == pytest.approx([2.5] * 3)
    assert np.allclose(sun.direction[:3], J.euler_matrix([-1.0, 0.3, 0]) @ [0, 0, -1], atol=1e-6)
    # point: kind 1, radius; spot: kind 2, aimed at the cube node, Blender blend on the cosine
    assert bulb.position[3] == 1.0 and bulb.params[1] == pytest.approx(0.1)
    assert spot.position[3] == 2.0
    outer = math.pi / 8
    assert spot.direction[3] == pytest.approx(math.cos(outer))
    assert spot.radiance[3] == pytest.approx(math.cos(math.acos(math.cos(outer) + (1 - math.cos(outer)) * 0.15)))
    assert list(sc.environment.radiance) == pytest.approx([0.15, 0.2, 0.3])


@pytest.mark.parametrize("edit,match", [
    (lambda d: d["nodes"].append({"type": "asset", "file": "x.glb"}), "asset"),
    (lambda d: d["materials"]["clay"]["inputs"].update(coat_weight=1.0), "coat_weight"),
    (lambda d: d["geometry"].update(ball={"std": "torus"}), "torus"),
    (lambda d: d.update(version=1), "version 2"),
    (lambda d: d["nodes"][-1]["material"]["inputs"].update(use_dof=True), "depth-of-field"),
    (lambda d: d["nodes"].append({"type": "mesh", "geometry": "nothing"}), "nothing"),
])
def test_outside_the_subset_is_refused(edit, match):
    d = _doc()
    edit(d)
    with pytest.raises(J.SceneSubsetError, match=match):
        J.load(d)


def test_resolution_override_and_background_colour():
    d = _doc()
    d["render"]["background"] = [0.1, 0.2, 0.3]
    sc = J.load(d, width=64, height=32)
    assert (sc.camera.width, sc.camera.height) == (64, 32)
    assert list(sc.environment.background) == pytest.approx([0.1, 0.2, 0.3]) and sc.environment.camera_sees_environment == 0


@pytest.mark.gpu
def test_loaded_document_renders_like_the_oracle(renderer, oracle):
    sc = J.load(FIXTURE, width=96, height=72)
    prof = Profile.reference_transport(4, 16)
    o = oracle.OracleScene(sc, fp32=True, fp64=False)
    ref, _ = o.render(prof.c(), fp64=False)
    with renderer.install(sc) as s:
        img = s.render(prof).image
    assert np.isfinite(img).all()
    m, mr = img[..., :3].mean((0, 1)), ref[..., :3].mean((0, 1))
    assert np.all(np.abs(m / mr - 1) < 0.01), (m, mr)


@pytest.mark.gpu
def test_render_command_writes_a_tagged_png(tmp_path):
    from vork_b200 import __main__ as cli, display as V
    out = tmp_path / "scene.png"
    assert cli.main(["render", str(FIXTURE), "--out", str(out), "--samples", "4", "--depth", "4", "--width", "64",
                     "--height", "48", "--linear", str(tmp_path / "lin.npy")]) == 0
    codes, tags = V.read_png(out)
    lin = np.load(tmp_path / "lin.npy")
    assert codes.shape == (48, 64, 4) and tags["sRGB"] == b"\x00"
    from oracle import display as D
    assert np.abs(codes.astype(int) - D.display(lin, bits=8).astype(int)).max() <= 1
    assert codes[..., :3].max() > 0
