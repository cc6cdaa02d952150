"""vork scene documents (version 2) for the backend: the subset the path's configurations use.

Reads the scene JSON that `vork render scene.json` takes (crates/vork-scene/src/v2/mod.rs:
version, render, nodes, buffers, geometry, materials) and returns an installable `Scene`:

* nodes (`node.rs:41-120,173-230`): glTF TRS written on the node (quaternion or
  `{"euler": [x, y, z]}`, R = Rz Ry Rx, `node.rs:395-430`), children, `target` aiming at a
  point or a named node (`crates/vork-render/src/targets.rs:62-92`: look-to frame with +Y up,
  +Z when the view is within 0.999 of vertical), and the kinds
  - `mesh`: `geometry` by name or inline, `materials` by name or inline (one per mesh),
    `instances` with TRANSLATION / ROTATION / SCALE buffers (`geometry.rs:171-178`);
  - `light`: sun, point, spot, rectangle, ellipse evaluated to light records as
    `crates/vork-render/src/lights.rs:53-170` does (defaults from `light.rs:14-36` and
    `constants.rs`), and an environment light's constant colour x energy as the world;
  - `camera`: std/camera's pinhole with its inputs (`libraries/std/camera.slang:6-36`:
    lens 50 mm, 36 x 24 mm sensor, auto fit, clip 0.1..1000);
  - `node`: a group;
* geometry (`geometry.rs:83-131`): inline or named buffers POSITION (vec3), NORMAL (vec3,
  else area-weighted vertex normals), u32 `indices` (else a triangle soup), or the std
  generators `{"std": "sphere" | "grid" | "box", ...}` of crates/vork-std/src/sdk.js;
* materials (`material.rs:279-300`): the OpenPBR inputs of the built subset (base_weight,
  base_color, base_metalness, specular_weight, specular_color, specular_roughness,
  specular_ior) and `double_sided`;
* render (`render.rs:75-110`): resolution, camera, background (environment, a colour, or
  transparent).

Anything outside the subset (assets, text, programs, textures, animation, other inputs)
raises SceneSubsetError naming it, instead of rendering something else.
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

from . import abi
from . import scene as S

SUPPORTED_INPUTS = {"base_weight", "base_color", "base_metalness", "specular_weight", "specular_color",
                    "specular_roughness", "specular_ior"}
BUFFER_WIDTH = {"f32": 1, "i32": 1, "u32": 1, "vec2": 2, "vec3": 3, "vec4": 4, "uvec4": 4, "mat4": 16}
UP_PARALLEL = 0.999               # crates/vork-render/src/constants.rs:69
SUN_ANGLE = math.radians(0.526)   # crates/vork-scene/src/v2/constants.rs:86-88
SPOT_SIZE, SPOT_BLEND = math.pi / 4, 0.15
ENVIRONMENT_COLOR = (0.05, 0.05, 0.05)


class SceneSubsetError(ValueError):
    """The document uses something outside the subset this backend renders."""


# ----------------------------------------------------------------------------- math
def quat_matrix(q):
    x, y, z, w = (float(v) for v in q)
    n = math.sqrt(x * x + y * y + z * z + w * w)
    if n < 1e-8:
        raise SceneSubsetError("zero-length rotation")
    x, y, z, w = x / n, y / n, z / n, w / n
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def euler_matrix(e):
    x, y, z = (float(v) for v in e)
    rx = np.array([[1, 0, 0], [0, math.cos(x), -math.sin(x)], [0, math.sin(x), math.cos(x)]])
    ry = np.array([[math.cos(y), 0, math.sin(y)], [0, 1, 0], [-math.sin(y), 0, math.cos(y)]])
    rz = np.array([[math.cos(z), -math.sin(z), 0], [math.sin(z), math.cos(z), 0], [0, 0, 1]])
    return rz @ ry @ rx


def rotation_of(r):
    if r is None:
        return np.eye(3)
    if isinstance(r, dict):
        if set(r) != {"euler"}:
            raise SceneSubsetError(f"rotation {r!r}: a quaternion or {{'euler': [x, y, z]}}")
        return euler_matrix(r["euler"])
    return quat_matrix(r)


def trs(node):
    m = np.eye(4)
    t = node.get("translation", [0.0, 0.0, 0.0])
    s = node.get("scale", [1.0, 1.0, 1.0])
    m[:3, :3] = rotation_of(node.get("rotation")) @ np.diag([float(v) for v in s])
    m[:3, 3] = [float(v) for v in t]
    return m


def look_to_frame(eye, direction, up):
    """Columns x, y, z of the camera-to-world frame of a right-handed look-to view."""
    f = direction / np.linalg.norm(direction)
    x = np.cross(f, up)
    x /= np.linalg.norm(x)
    y = np.cross(x, f)
    return np.stack([x, y, -f], 1)


def aimed(world, target, parent_world, node):
    """targets.rs:62-92: a look-to frame at the node's origin, times its own rotation, the
    parent's stretch and its scale."""
    eye = world[:3, 3]
    d = np.asarray(target, np.float64) - eye
    if float(d @ d) <= 1e-10:
        raise SceneSubsetError(f"node {node.get('name', '')!r}: target coincides with the node origin")
    d /= np.linalg.norm(d)
    up = np.array([0.0, 0.0, 1.0]) if abs(d[1]) > UP_PARALLEL else np.array([0.0, 1.0, 0.0])
    frame = look_to_frame(eye, d, up)
    p = parent_world[:3, :3]
    x = p[:, 0] / max(np.linalg.norm(p[:, 0]), 1e-30)
    y = p[:, 1] - x * (x @ p[:, 1])
    y /= max(np.linalg.norm(y), 1e-30)
    stretch = np.stack([x, y, np.cross(x, y)], 1).T @ p
    out = np.eye(4)
    out[:3, :3] = frame @ rotation_of(node.get("rotation")) @ stretch @ np.diag([float(v) for v in node.get("scale", [1, 1, 1])])
    out[:3, 3] = eye
    return out


def node_view(world):
    """values.rs:1208-1255: the orthonormal view frame of a node (right, up, -forward)."""
    direction = -world[:3, 2] / np.linalg.norm(world[:3, 2])
    up = world[:3, 1] / np.linalg.norm(world[:3, 1])
    if abs(direction @ up) > UP_PARALLEL:
        up = world[:3, 2] / np.linalg.norm(world[:3, 2])
        if abs(direction @ up) > UP_PARALLEL:
            up = world[:3, 0] / np.linalg.norm(world[:3, 0])
    return look_to_frame(world[:3, 3], direction, up)


# ----------------------------------------------------------------------------- document
class _Loader:
    def __init__(self, doc, base: Path | None):
        if doc.get("version") != 2:
            raise SceneSubsetError("only scene version 2 documents are read")
        comp = doc.get("composition")
        if comp and comp.get("space", "3d") != "3d":
            raise SceneSubsetError("2D canvas documents are outside the subset")
        for key in ("animation", "programs", "images", "simulation", "propagation"):
            if doc.get(key):
                raise SceneSubsetError(f"scene.{key} is outside the subset")
        self.doc, self.base = doc, base
        self.buffers = doc.get("buffers", {})
        self.geometry = doc.get("geometry", {})
        self.materials = doc.get("materials", {})
        self.meshes, self.mesh_keys = [], {}
        self.mats, self.mat_keys = [], {}
        self.rows, self.mesh_ids, self.mat_ids = [], [], []
        self.lights, self.env = [], None
        self.cameras = []

    # buffers ------------------------------------------------------------------
    def buffer(self, ref, what):
        b = self.buffers.get(ref) if isinstance(ref, str) else ref
        if b is None:
            raise SceneSubsetError(f"{what}: unknown buffer {ref!r}")
        if "data" not in b or b.get("file") or b.get("grid") or b.get("dims"):
            raise SceneSubsetError(f"{what}: only inline `data` buffers are read")
        width = BUFFER_WIDTH.get(b.get("type"))
        if width is None:
            raise SceneSubsetError(f"{what}: buffer type {b.get('type')!r}")
        arr = np.asarray(b["data"], np.float64)
        return arr.reshape(-1) if width == 1 else arr.reshape(-1, width)

    # geometry -----------------------------------------------------------------
    def mesh(self, ref):
        key = ref if isinstance(ref, str) else id(ref)
        if key in self.mesh_keys:
            return self.mesh_keys[key]
        g = self.geometry.get(ref) if isinstance(ref, str) else ref
        if g is None:
            raise SceneSubsetError(f"unknown geometry {ref!r}")
        mesh = self.std_mesh(g) if "std" in g else self.buffer_mesh(g, ref)
        self.meshes.append(mesh)
        self.mesh_keys[key] = len(self.meshes) - 1
        return self.mesh_keys[key]

    def std_mesh(self, g):
        kind = g["std"]
        opts = {k: v for k, v in g.items() if k != "std"}
        if kind == "sphere":
            bad = set(opts) - {"radius", "segments", "rings"}
            if bad:
                raise SceneSubsetError(f"std sphere options {sorted(bad)}")
            return S.uv_sphere(float(opts.get("radius", 1.0)), int(opts.get("segments", 32)), int(opts.get("rings", 16)))
        if kind == "grid":
            bad = set(opts) - {"size", "segments"}
            if bad:
                raise SceneSubsetError(f"std grid options {sorted(bad)}")
            return S.grid(tuple(float(v) for v in opts.get("size", [2, 2])), tuple(int(v) for v in opts.get("segments", [1, 1])))
        if kind == "box":
            bad = set(opts) - {"size"}
            if bad:
                raise SceneSubsetError(f"std box options {sorted(bad)}")
            return box(tuple(float(v) for v in opts.get("size", [2, 2, 2])))
        raise SceneSubsetError(f"std geometry {kind!r} is outside the subset (sphere, grid, box)")

    def buffer_mesh(self, g, ref):
        if g.get("topology", "triangles") != "triangles":
            raise SceneSubsetError(f"geometry {ref!r}: only triangles")
        for key in ("face_vertex_counts", "subdivision", "curve_vertex_counts", "widths", "material_ranges", "morphs"):
            if g.get(key):
                raise SceneSubsetError(f"geometry {ref!r}: `{key}` is outside the subset")
        attrs = g.get("attributes", {})
        if "POSITION" not in attrs:
            raise SceneSubsetError(f"geometry {ref!r}: no POSITION")
        pos = self.buffer(attrs["POSITION"], "POSITION")
        idx = self.buffer(g["indices"], "indices").astype(np.int64) if g.get("indices") is not None else np.arange(len(pos))
        if len(idx) % 3 or (len(idx) and (idx.min() < 0 or idx.max() >= len(pos))):
            raise SceneSubsetError(f"geometry {ref!r}: indices are not whole triangles of its vertices")
        tri = idx.reshape(-1, 3)
        if "NORMAL" in attrs:
            nrm = self.buffer(attrs["NORMAL"], "NORMAL")
        else:
            nrm = np.zeros_like(pos)
            fn = np.cross(pos[tri[:, 1]] - pos[tri[:, 0]], pos[tri[:, 2]] - pos[tri[:, 0]])
            for k in range(3):
                np.add.at(nrm, tri[:, k], fn)
            nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-30)
        return S.Mesh(pos.astype(np.float32), nrm.astype(np.float32), tri.astype(np.uint32))

    # materials ----------------------------------------------------------------
    def material(self, ref):
        key = ref if isinstance(ref, str) else json.dumps(ref, sort_keys=True)
        if key in self.mat_keys:
            return self.mat_keys[key]
        m = self.materials.get(ref) if isinstance(ref, str) else ref
        if m is None:
            raise SceneSubsetError(f"unknown material {ref!r}")
        if m.get("program") not in (None, "std/openpbr"):
            raise SceneSubsetError(f"material program {m.get('program')!r} is outside the subset")
        inputs = m.get("inputs", {})
        bad = set(inputs) - SUPPORTED_INPUTS
        if bad:
            raise SceneSubsetError(f"material inputs {sorted(bad)} are outside the subset")
        for k, v in inputs.items():
            if isinstance(v, dict):
                raise SceneSubsetError(f"material input {k!r}: only constant values")
        mat = S.material(inputs.get("base_color", [0.8, 0.8, 0.8]), inputs.get("specular_roughness", 0.3),
                         inputs.get("base_metalness", 0.0), bool(m.get("double_sided", False)))
        mat.base_weight = float(inputs.get("base_weight", 1.0))
        mat.specular_weight = float(inputs.get("specular_weight", 1.0))
        mat.specular_color[:] = [float(v) for v in inputs.get("specular_color", [1.0, 1.0, 1.0])]
        mat.specular_ior = float(inputs.get("specular_ior", 1.5))
        self.mats.append(mat)
        self.mat_keys[key] = len(self.mats) - 1
        return self.mat_keys[key]

    # nodes --------------------------------------------------------------------
    def walk(self, nodes, parent, named, out):
        for node in nodes:
            local = trs(node)
            world = parent @ local
            target = node.get("target")
            if target is not None:
                if isinstance(target, str) and target not in named:
                    raise SceneSubsetError(f"target {target!r} is not a node")
                point = named[target][:3, 3] if isinstance(target, str) else target
                world = aimed(world, point, parent, node)
            out.append((node, world))
            self.walk(node.get("children", []), world, named, out)

    def names(self, nodes, parent, named):
        for node in nodes:
            world = parent @ trs(node)
            if node.get("name"):
                named[node["name"]] = world
            self.names(node.get("children", []), world, named)

    def run(self, width=None, height=None):
        named = {}
        self.names(self.doc.get("nodes", []), np.eye(4), named)
        placed = []
        self.walk(self.doc.get("nodes", []), np.eye(4), named, placed)
        for node, world in placed:
            kind = node.get("type", "node")
            if kind == "mesh":
                self.add_mesh(node, world)
            elif kind == "light":
                self.add_light(node, world)
            elif kind == "camera":
                self.cameras.append((node, world))
            elif kind != "node":
                raise SceneSubsetError(f"node type {kind!r} is outside the subset")
        render = self.doc.get("render", {})
        res = render.get("resolution", [1920, 1080])
        w, h = int(width or res[0]), int(height or res[1])
        cam = self.camera(render.get("camera"), w, h)
        if not self.rows:
            raise SceneSubsetError("the scene has no mesh")
        env = self.environment(render.get("background", "environment"))
        rows = np.stack(self.rows).astype(np.float32)
        return S.Scene(self.meshes, rows, np.asarray(self.mesh_ids, np.uint32), np.asarray(self.mat_ids, np.uint32),
                       self.mats, self.lights, cam, env, name=str(self.doc.get("name", "scene")))

    def add_mesh(self, node, world):
        for key in ("skin", "morph_weights"):
            if node.get(key):
                raise SceneSubsetError(f"mesh `{key}` is outside the subset")
        mesh = self.mesh(node["geometry"])
        mats = node.get("materials", [])
        if len(mats) > 1:
            raise SceneSubsetError("one material per mesh (material ranges are outside the subset)")
        mat = self.material(mats[0] if mats else {"inputs": {}})
        inst = node.get("instances")
        if inst is None:
            locals_ = [np.eye(4)]
        else:
            attrs = inst.get("attributes", {})
            bad = set(attrs) - {"TRANSLATION", "ROTATION", "SCALE"}
            if bad:
                raise SceneSubsetError(f"instance attributes {sorted(bad)} are outside the subset")
            t = self.buffer(attrs["TRANSLATION"], "TRANSLATION") if "TRANSLATION" in attrs else None
            r = self.buffer(attrs["ROTATION"], "ROTATION") if "ROTATION" in attrs else None
            s = self.buffer(attrs["SCALE"], "SCALE") if "SCALE" in attrs else None
            counts = {len(a) for a in (t, r, s) if a is not None}
            if inst.get("count") is not None:
                counts.add(int(self.buffer(inst["count"], "count")[0]) if not isinstance(inst["count"], int) else inst["count"])
            if len(counts) != 1:
                raise SceneSubsetError("instance attribute lengths differ")
            n = counts.pop()
            locals_ = []
            for i in range(n):
                m = np.eye(4)
                rot = quat_matrix(r[i]) if r is not None else np.eye(3)
                m[:3, :3] = rot @ np.diag(s[i] if s is not None else [1.0, 1.0, 1.0])
                if t is not None:
                    m[:3, 3] = t[i]
                locals_.append(m)
        for m in locals_:
            wm = world @ m
            self.rows.append(wm[:3, :4])
            self.mesh_ids.append(mesh)
            self.mat_ids.append(mat)

    def add_light(self, node, world):
        shape = node.get("shape")
        color = node.get("color")
        if node.get("temperature") is not None or node.get("image") or node.get("medium") or node.get("material"):
            raise SceneSubsetError("light temperature, images, media and materials are outside the subset")
        if shape == "environment":
            energy = float(node.get("energy", 1.0))
            c = color if color is not None else ENVIRONMENT_COLOR
            self.env = [float(v) * energy for v in c]
            return
        energy = float(node.get("energy", 1.0 if shape == "sun" else 10.0))
        color = [float(v) for v in (color if color is not None else [1.0, 1.0, 1.0])]
        frame = node_view(world)
        direction = frame @ np.array([0.0, 0.0, -1.0])
        l = S._light_base()
        if shape == "sun":
            kind, size, inner, outer = 0.0, float(node.get("angle", SUN_ANGLE)) * 0.5, 0.0, 0.0
        elif shape == "point":
            kind, size, inner, outer = 1.0, float(node.get("radius", 0.0)), 0.0, math.pi / 4
        elif shape == "spot":
            spot, blend = float(node.get("spot_size", SPOT_SIZE)), float(node.get("spot_blend", SPOT_BLEND))
            oc = math.cos(spot * 0.5)
            kind, size = 2.0, float(node.get("radius", 0.0))
            inner, outer = math.acos(min(1.0, max(-1.0, oc + (1.0 - oc) * blend))), spot * 0.5
        elif shape in ("rectangle", "ellipse"):
            kind, inner, outer = 3.0, 0.0, math.pi / 4
            width = float(node.get("size", 1.0))
            height = float(node.get("size_y", width))
            u = frame @ np.array([1.0, 0.0, 0.0]) * np.linalg.norm(world[:3, 0]) * width
            v = frame @ np.array([0.0, 1.0, 0.0]) * np.linalg.norm(world[:3, 1]) * height
            l.emitter_u[:] = [float(u[0]), float(u[1]), float(u[2]), 1.0 if shape == "ellipse" else 0.0]
            l.emitter_v[:] = [float(v[0]), float(v[1]), float(v[2]), 0.0]
            size = 0.5 * math.sqrt(float(u @ u + v @ v))
            if float(np.linalg.norm(np.cross(u, v))) == 0.0:
                energy = 0.0
        else:
            raise SceneSubsetError(f"light shape {shape!r}")
        pos = world[:3, 3]
        l.position[:] = [float(pos[0]), float(pos[1]), float(pos[2]), kind]
        l.direction[:] = [float(direction[0]), float(direction[1]), float(direction[2]), math.cos(outer)]
        l.radiance[:] = [color[0] * energy, color[1] * energy, color[2] * energy, math.cos(inner)]
        l.params[:] = [0.0, size, 0.0, 0.0]
        l.projection[:] = [math.tan(outer), 0.0, 0.0, 0.0]
        self.lights.append(l)

    def camera(self, name, w, h):
        cams = [c for c in self.cameras if name is None or c[0].get("name") == name]
        if not cams:
            raise SceneSubsetError(f"no camera {name!r}" if name else "the scene has no camera")
        node, world = cams[0]
        mat = node.get("material")
        inputs = {}
        if mat is not None:
            if isinstance(mat, str) or mat.get("program") not in (None, "std/camera"):
                raise SceneSubsetError("camera materials other than inline std/camera inputs are outside the subset")
            inputs = mat.get("inputs", {})
        if inputs.get("projection", "persp") != "persp" or inputs.get("use_dof", False) or any(inputs.get("shift", [0, 0])):
            raise SceneSubsetError("orthographic, depth-of-field and shifted cameras are outside the subset")
        lens = float(inputs.get("lens", 50.0))
        sw, sh = float(inputs.get("sensor_width", 36.0)), float(inputs.get("sensor_height", 24.0))
        fit = inputs.get("fit", "auto")
        aspect = w / h
        span = aspect if fit == "horizontal" else (1.0 if fit == "vertical" else max(aspect, 1.0))
        sensor = sh if fit == "vertical" else sw
        height = sensor / span                      # camera.slang:26-31
        frame = node_view(world)
        cam = abi.VkbCamera()
        cam.eye[:] = [float(v) for v in world[:3, 3]]
        cam.right[:] = [float(v) for v in frame[:, 0]]
        cam.up[:] = [float(v) for v in frame[:, 1]]
        cam.forward[:] = [float(v) for v in -frame[:, 2]]
        cam.proj_x = 2.0 * lens / (height * aspect)
        cam.proj_y = 2.0 * lens / height
        cam.near_plane, cam.far_plane = float(inputs.get("clip_start", 0.1)), float(inputs.get("clip_end", 1000.0))
        cam.width, cam.height = w, h
        return cam

    def environment(self, background):
        radiance = self.env if self.env is not None else [0.0, 0.0, 0.0]
        if isinstance(background, list):
            return S.environment(radiance, background=[float(v) for v in background], camera_sees=False)
        if background == "transparent":
            return S.environment(radiance, background=[0.0, 0.0, 0.0], camera_sees=False)
        if background != "environment":
            raise SceneSubsetError(f"background {background!r}")
        return S.environment(radiance)


def box(size=(2.0, 2.0, 2.0)) -> S.Mesh:
    """sdk.js:135-155: six faces of two triangles each, per-face normals."""
    faces = [((1, 0, 0), (0, 0, -1), (0, 1, 0)), ((-1, 0, 0), (0, 0, 1), (0, 1, 0)),
             ((0, 1, 0), (1, 0, 0), (0, 0, -1)), ((0, -1, 0), (1, 0, 0), (0, 0, 1)),
             ((0, 0, 1), (1, 0, 0), (0, 1, 0)), ((0, 0, -1), (-1, 0, 0), (0, 1, 0))]
    pos, nrm, idx = [], [], []
    for n, u, v in faces:
        base = len(pos)
        for y in (-1, 1):
            for x in (-1, 1):
                pos.append([(n[k] + u[k] * x + v[k] * y) * size[k] / 2 for k in range(3)])
                nrm.append(n)
        idx += [(base + 0, base + 1, base + 3), (base + 0, base + 3, base + 2)]
    return S.Mesh(np.asarray(pos, np.float32), np.asarray(nrm, np.float32), np.asarray(idx, np.uint32))


def load(source, width: int | None = None, height: int | None = None) -> S.Scene:
    """A scene document (path, JSON text or parsed dict) -> Scene (resolution overridable)."""
    base = None
    if isinstance(source, dict):
        doc = source
    elif isinstance(source, (str, Path)) and Path(str(source)).exists():
        base = Path(str(source)).resolve().parent
        raw = Path(str(source)).read_bytes()
        doc = json.loads(raw.decode("utf-8-sig"))
    else:
        doc = json.loads(str(source))
    return _Loader(doc, base).run(width, height)
