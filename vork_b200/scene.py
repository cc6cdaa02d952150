"""Seeded synthetic scenes for the std/path configurations, and their C descriptors.

Geometry follows vork's std library tessellation rules: the Y-up UV sphere with 32
longitudes x 16 rings (crates/vork-std/src/sdk.js:157-181, 960 triangles) and the
centred XZ grid facing +Y (sdk.js:350-370).  Lights are packed as `Light` records the
way crates/vork-render/src/lights.rs:53-170 packs them (area light: kind 3, edge vectors
u = X*width, v = Y*height of the light frame, radiance = colour*energy, emitted radiance
radiance/(pi*area), shaders/emitter.slang:143).  No public dataset is involved: every
input is generated here from a fixed seed.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi

# ----------------------------------------------------------------------------- PCG32
_PCG_MULT = 6364136223846793005
_MASK64 = (1 << 64) - 1


class Pcg32:
    """O'Neill's PCG32 (XSH-RR), seeded like the reference implementation's pcg32_srandom."""

    def __init__(self, seed: int = 0, seq: int = 0xDA3E39CB94B95BDB):
        self.state = 0
        self.inc = ((seq << 1) | 1) & _MASK64
        self.next_u32()
        self.state = (self.state + seed) & _MASK64
        self.next_u32()

    def next_u32(self) -> int:
        old = self.state
        self.state = (old * _PCG_MULT + self.inc) & _MASK64
        xorshifted = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xorshifted >> rot) | (xorshifted << ((-rot) & 31))) & 0xFFFFFFFF

    def uniform(self, lo: float = 0.0, hi: float = 1.0) -> float:
        return lo + (hi - lo) * ((self.next_u32() >> 8) * (1.0 / 16777216.0))


# ----------------------------------------------------------------------------- meshes
@dataclass
class Mesh:
    positions: np.ndarray  # (V,3) float32
    normals: np.ndarray    # (V,3) float32
    indices: np.ndarray    # (T,3) uint32

    @property
    def num_triangles(self) -> int:
        return int(self.indices.shape[0])


def uv_sphere(radius: float = 1.0, longitude: int = 32, rings: int = 16) -> Mesh:
    """sdk.js:157-181: vertices per ring and longitude (seam duplicated), tri(a,b+1,b), tri(a,a+1,b+1)."""
    pos, nrm = [], []
    for y in range(rings + 1):
        a = y * math.pi / rings
        for x in range(longitude + 1):
            az = (0 if x == longitude else x) * 2 * math.pi / longitude
            c, s = math.cos(az), math.sin(az)
            n = (0.0, 1.0, 0.0) if y == 0 else ((0.0, -1.0, 0.0) if y == rings else (math.sin(a) * c, math.cos(a), math.sin(a) * s))
            nrm.append(n)
            pos.append(tuple(v * radius for v in n))
    idx = []
    for y in range(rings):
        for x in range(longitude):
            a = y * (longitude + 1) + x
            b = a + longitude + 1
            if y < rings - 1:
                idx.append((a, b + 1, b))
            if y > 0:
                idx.append((a, a + 1, b + 1))
    return Mesh(np.asarray(pos, np.float32), np.asarray(nrm, np.float32), np.asarray(idx, np.uint32))


def grid(size=(2.0, 2.0), segments=(1, 1)) -> Mesh:
    """sdk.js:350-370: XZ grid facing +Y, centred; tri(a,c,a+1), tri(a+1,c,c+1)."""
    nx, nz = segments
    pos, nrm = [], []
    for z in range(nz + 1):
        for x in range(nx + 1):
            pos.append(((x / nx - 0.5) * size[0], 0.0, (z / nz - 0.5) * size[1]))
            nrm.append((0.0, 1.0, 0.0))
    idx = []
    for z in range(nz):
        for x in range(nx):
            a = z * (nx + 1) + x
            c = a + nx + 1
            idx.append((a, c, a + 1))
            idx.append((a + 1, c, c + 1))
    return Mesh(np.asarray(pos, np.float32), np.asarray(nrm, np.float32), np.asarray(idx, np.uint32))


def height_grid(heights: np.ndarray, size: float) -> Mesh:
    """A displaced XZ grid (terrain) with smooth normals from central differences."""
    n = heights.shape[0] - 1
    xs = (np.arange(n + 1, dtype=np.float64) / n - 0.5) * size
    X, Z = np.meshgrid(xs, xs, indexing="xy")
    pos = np.stack([X, heights, Z], -1).reshape(-1, 3)
    h = heights
    dx = np.gradient(h, axis=1) / (size / n)
    dz = np.gradient(h, axis=0) / (size / n)
    nrm = np.stack([-dx, np.ones_like(h), -dz], -1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    a = (np.arange(n)[None, :] + (n + 1) * np.arange(n)[:, None]).reshape(-1)
    c = a + n + 1
    idx = np.stack([np.stack([a, c, a + 1], -1), np.stack([a + 1, c, c + 1], -1)], 1).reshape(-1, 3)
    return Mesh(pos.astype(np.float32), nrm.reshape(-1, 3).astype(np.float32), idx.astype(np.uint32))


def geodesic_sphere(frequency: int = 5, jitter: float = 0.0, seed: int = 0) -> Mesh:
    """Icosahedron with each face split into frequency^2 triangles (20*f^2: 500 at f=5),
    projected to the unit sphere, radially jittered by a seeded amount."""
    t = (1 + 5 ** 0.5) / 2
    V = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                  (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], np.float64)
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
         (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts: dict = {}
    pos: list = []
    idx: list = []

    def vid(p):
        key = tuple(np.round(p / np.linalg.norm(p), 9))
        if key not in verts:
            verts[key] = len(pos)
            pos.append(p / np.linalg.norm(p))
        return verts[key]

    f = frequency
    for a, b, c in F:
        A, B, Cc = V[a], V[b], V[c]
        grid_ids = {}
        for i in range(f + 1):
            for j in range(f + 1 - i):
                p = A + (B - A) * (i / f) + (Cc - A) * (j / f)
                grid_ids[(i, j)] = vid(p)
        for i in range(f):
            for j in range(f - i):
                idx.append((grid_ids[(i, j)], grid_ids[(i + 1, j)], grid_ids[(i, j + 1)]))
                if j < f - i - 1:
                    idx.append((grid_ids[(i + 1, j)], grid_ids[(i + 1, j + 1)], grid_ids[(i, j + 1)]))
    P = np.asarray(pos)
    if jitter > 0:
        rng = np.random.default_rng(seed)
        P = P * (1.0 + jitter * (rng.random(len(P))[:, None] * 2 - 1))
    I = np.asarray(idx, np.uint32)
    # outward winding
    p0, p1, p2 = P[I[:, 0]], P[I[:, 1]], P[I[:, 2]]
    flip = np.einsum("ij,ij->i", np.cross(p1 - p0, p2 - p0), p0 + p1 + p2) < 0
    I[flip] = I[flip][:, [0, 2, 1]]
    N = P / np.linalg.norm(P, axis=1, keepdims=True)
    return Mesh(P.astype(np.float32), N.astype(np.float32), I)


# ----------------------------------------------------------------------------- records
def material(base_color=(0.8, 0.8, 0.8), roughness=0.3, metalness=0.0, double_sided=False) -> abi.VkbMaterial:
    """OpenPBR 1.1.1 defaults (crates/vork-scene/openpbr-params.md:22-30) with the given inputs."""
    m = abi.VkbMaterial()
    m.base_weight = 1.0
    m.base_color[:] = [float(v) for v in base_color]
    m.base_metalness = float(metalness)
    m.specular_weight = 1.0
    m.specular_color[:] = [1.0, 1.0, 1.0]
    m.specular_roughness = float(roughness)
    m.specular_ior = 1.5
    m.emission_luminance = 0.0
    m.emission_color[:] = [1.0, 1.0, 1.0]
    m.flags = 2 if double_sided else 0
    return m


def emissive(color=(1.0, 1.0, 1.0), luminance=1.0, double_sided=False) -> abi.VkbMaterial:
    """A black surface emitting colour x luminance (OpenPBR emission_color, emission_luminance)
    on its front side, or on both sides when double sided."""
    m = material((0.0, 0.0, 0.0), 1.0, 0.0, double_sided)
    m.base_weight = 0.0
    m.specular_weight = 0.0
    m.emission_luminance = float(luminance)
    m.emission_color[:] = [float(v) for v in color]
    return m


ALL_RAYS = abi.RAY_CAMERA | abi.RAY_SHADOW | abi.RAY_DIFFUSE | abi.RAY_SPECULAR | abi.RAY_TRANSMISSION | abi.RAY_VOLUME


def _light_base() -> abi.VkbLight:
    l = abi.VkbLight()
    l.shadow_offsets[0] = ALL_RAYS | abi.LIGHT_LINK_ALL         # contribution: visible to every ray, all links
    l.shadow_offsets[1] = 0xFFFFFFFF                             # illuminates every group
    l.shadow_offsets[2] = abi.LIGHT_RAY_SHADOWED | abi.LIGHT_RAY_SHADOWED_BY_ALL
    l.shadow_offsets[3] = 0xFFFFFFFF
    return l


def area_light(center, normal, u_axis, width, height, radiance, color=(1.0, 1.0, 1.0)) -> abi.VkbLight:
    """Rectangle light emitting along `normal` with radiance `radiance`: energy = radiance*pi*area (lights.rs:99-127)."""
    n = np.asarray(normal, np.float64); n /= np.linalg.norm(n)
    u = np.asarray(u_axis, np.float64); u -= n * np.dot(u, n); u /= np.linalg.norm(u)
    v = np.cross(n, u)  # light frame: -Z along the emission direction, X = u, Y = v
    area = width * height
    energy = radiance * math.pi * area
    l = _light_base()
    l.position[:] = [float(center[0]), float(center[1]), float(center[2]), 3.0]
    l.direction[:] = [float(n[0]), float(n[1]), float(n[2]), math.cos(math.pi / 4)]
    l.radiance[:] = [color[0] * energy, color[1] * energy, color[2] * energy, 1.0]
    eu, ev = u * width, v * height
    l.params[:] = [0.0, 0.5 * math.sqrt(float(np.dot(eu, eu) + np.dot(ev, ev))), 0.0, 0.0]
    l.emitter_u[:] = [float(eu[0]), float(eu[1]), float(eu[2]), 0.0]
    l.emitter_v[:] = [float(ev[0]), float(ev[1]), float(ev[2]), 0.0]
    l.projection[:] = [math.tan(math.pi / 4), 0.0, 0.0, 0.0]
    return l


def sun_light(direction, angle_degrees=0.526, energy=3.0, color=(1.0, 1.0, 1.0)) -> abi.VkbLight:
    """Sun: kind 0, params.y = half the angular diameter, direction = travel direction of its light."""
    d = np.asarray(direction, np.float64); d /= np.linalg.norm(d)
    l = _light_base()
    l.position[:] = [0.0, 0.0, 0.0, 0.0]
    l.direction[:] = [float(d[0]), float(d[1]), float(d[2]), 1.0]
    l.radiance[:] = [color[0] * energy, color[1] * energy, color[2] * energy, 1.0]
    l.params[:] = [0.0, math.radians(angle_degrees) * 0.5, 0.0, 0.0]
    l.projection[:] = [0.0, 0.0, 0.0, 0.0]
    return l


def look_at(eye, target, up=(0.0, 1.0, 0.0), fov_y_degrees=45.0, width=256, height=256, near=0.05, far=1e4) -> abi.VkbCamera:
    e = np.asarray(eye, np.float64); t = np.asarray(target, np.float64)
    f = t - e; f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    if np.linalg.norm(r) < 1e-6:  # looking along `up`: take any perpendicular
        r = np.cross(f, (0.0, 0.0, 1.0) if abs(f[2]) < 0.9 else (1.0, 0.0, 0.0))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    cam = abi.VkbCamera()
    cam.eye[:] = [float(x) for x in e]
    cam.right[:] = [float(x) for x in r]
    cam.up[:] = [float(x) for x in u]
    cam.forward[:] = [float(x) for x in f]
    p11 = 1.0 / math.tan(math.radians(fov_y_degrees) / 2)
    cam.proj_y = p11
    cam.proj_x = p11 / (width / height)
    cam.near_plane, cam.far_plane = near, far
    cam.width, cam.height = width, height
    return cam


def rows_from(scale, translate) -> np.ndarray:
    """3x4 object->world rows of a uniform scale then translation."""
    r = np.zeros((3, 4), np.float32)
    r[0, 0] = r[1, 1] = r[2, 2] = scale
    r[:, 3] = translate
    return r


# ----------------------------------------------------------------------------- scene
@dataclass
class Scene:
    meshes: list
    instance_rows: np.ndarray       # (N,3,4) float32
    instance_mesh: np.ndarray       # (N,) uint32
    instance_material: np.ndarray   # (N,) uint32
    materials: list
    lights: list
    camera: abi.VkbCamera
    environment: abi.VkbEnvironment
    name: str = "scene"
    tlas_builder: int = abi.TLAS_LBVH
    env_image: "EnvironmentImage | None" = None
    blas_format: int = abi.BLAS_WIDE4
    blas_builder: int = abi.BLAS_BUILD_SAH
    _keep: list = field(default_factory=list, repr=False)

    @property
    def num_triangles(self) -> int:
        return int(sum(self.meshes[m].num_triangles for m in self.instance_mesh))

    def desc(self) -> abi.VkbSceneDesc:
        """The C descriptor; the arrays it points at stay alive with this Scene."""
        keep = []
        mesh_arr = (abi.VkbMesh * max(1, len(self.meshes)))()
        for i, m in enumerate(self.meshes):
            p = np.ascontiguousarray(m.positions, np.float32)
            n = np.ascontiguousarray(m.normals, np.float32)
            ix = np.ascontiguousarray(m.indices, np.uint32)
            keep += [p, n, ix]
            mesh_arr[i].positions = abi.fptr(p)
            mesh_arr[i].normals = abi.fptr(n)
            mesh_arr[i].indices = abi.uptr(ix)
            mesh_arr[i].num_vertices = p.shape[0]
            mesh_arr[i].num_triangles = ix.shape[0]
        rows = np.ascontiguousarray(self.instance_rows, np.float32).reshape(-1)
        im = np.ascontiguousarray(self.instance_mesh, np.uint32)
        imat = np.ascontiguousarray(self.instance_material, np.uint32)
        mats = (abi.VkbMaterial * max(1, len(self.materials)))(*self.materials)
        lights = (abi.VkbLight * max(1, len(self.lights)))(*self.lights)
        keep += [mesh_arr, rows, im, imat, mats, lights]
        d = abi.VkbSceneDesc()
        d.meshes = C.cast(mesh_arr, C.POINTER(abi.VkbMesh))
        d.num_meshes = len(self.meshes)
        d.num_instances = int(im.shape[0])
        d.instance_rows = abi.fptr(rows)
        d.instance_mesh = abi.uptr(im)
        d.instance_material = abi.uptr(imat)
        d.materials = C.cast(mats, C.POINTER(abi.VkbMaterial))
        d.num_materials = len(self.materials)
        d.lights = C.cast(lights, C.POINTER(abi.VkbLight))
        d.num_lights = len(self.lights)
        d.camera = self.camera
        d.environment = self.environment
        d.tlas_builder = self.tlas_builder
        d.blas_format = self.blas_format
        d.blas_builder = self.blas_builder
        if self.env_image is not None:
            img = np.ascontiguousarray(self.env_image.rgba, np.float32)
            e = abi.VkbEnvironmentImage()
            e.rgba = abi.fptr(img)
            e.height, e.width = int(img.shape[0]), int(img.shape[1])
            e.strength = float(self.env_image.strength)
            e.color[:] = [float(v) for v in self.env_image.color]
            e.rotation[:] = [float(v) for v in np.asarray(self.env_image.rotation, np.float64).reshape(9)]
            keep += [img, e]
            d.environment_image = C.pointer(e)
        self._keep = keep
        return d


@dataclass
class EnvironmentImage:
    """A lat-long linear RGBA environment (row 0 at the +y pole) with its strength,
    colour and 3x3 rotation (a world direction d looks up normalize(d R))."""
    rgba: np.ndarray
    strength: float = 1.0
    color: tuple = (1.0, 1.0, 1.0)
    rotation: np.ndarray = field(default_factory=lambda: np.eye(3))


def sky_image(width: int = 256, height: int = 128, sun_dir=(0.4, 0.8, 0.45), sun_radiance: float = 400.0,
              sun_radius_deg: float = 3.0, seed: int = 0) -> np.ndarray:
    """A procedural lat-long sky: a blue-to-white gradient, a warm ground, seeded
    low-frequency cloud noise and a small bright disc around `sun_dir`."""
    rng = np.random.default_rng(seed)
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    theta = np.pi * v[:, None]
    phi = 2 * np.pi * (u[None, :] - 0.5)
    d = np.stack([np.sin(theta) * np.cos(phi), np.cos(theta) * np.ones_like(phi), np.sin(theta) * np.sin(phi)], -1)
    up = np.clip(d[..., 1], -1, 1)
    sky = np.where(up[..., None] > 0, (1 - up[..., None]) * np.array([0.9, 0.95, 1.0]) + up[..., None] * np.array([0.25, 0.45, 0.9]),
                   np.array([0.3, 0.25, 0.2]) * (1 + up[..., None]))
    noise = rng.random((8, 16))
    ny = np.minimum((v * 8).astype(int), 7)[:, None]
    nx = np.minimum((u * 16).astype(int), 15)[None, :]
    sky = sky * (0.8 + 0.4 * noise[ny, nx])[..., None]
    s = np.asarray(sun_dir, np.float64); s /= np.linalg.norm(s)
    disc = np.einsum("hwc,c->hw", d, s) > np.cos(np.radians(sun_radius_deg))
    sky[disc] = sun_radiance * np.array([1.0, 0.93, 0.85])
    rgba = np.concatenate([sky, np.ones(sky.shape[:2] + (1,))], -1)
    return rgba.astype(np.float32)


def environment(radiance=(0.0, 0.0, 0.0), exposure=1.0, background=(0.0, 0.0, 0.0), camera_sees=True) -> abi.VkbEnvironment:
    e = abi.VkbEnvironment()
    e.radiance[:] = [float(v) for v in radiance]
    e.exposure = float(exposure)
    e.background[:] = [float(v) for v in background]
    e.camera_sees_environment = 1 if camera_sees else 0
    return e


def spheres_scene(num_spheres: int = 64, seed: int = 0, width: int = 256, height: int = 256, cube: float = 10.0,
                  grid_cells: int = 64, light_radiance: float = 20.0) -> Scene:
    """Plain method, small: spheres at seeded uniform positions in a cube, radii U[0.2,1.0],
    a grid_cells^2-quad ground, albedo U[0.1,0.9]^3, roughness U[0.05,1.0], metallic
    Bernoulli(0.3), one rectangular area light of radiance `light_radiance`."""
    rng = Pcg32(seed)
    sphere = uv_sphere(1.0)
    ground = grid((cube, cube), (grid_cells, grid_cells))
    rows, mesh_ids, mats = [], [], []
    materials = []
    for i in range(num_spheres):
        c = (rng.uniform(0, cube), rng.uniform(0, cube), rng.uniform(0, cube))
        r = rng.uniform(0.2, 1.0)
        col = (rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9))
        rough = rng.uniform(0.05, 1.0)
        metal = 1.0 if rng.uniform() < 0.3 else 0.0
        materials.append(material(col, rough, metal))
        rows.append(rows_from(r, c))
        mesh_ids.append(0)
        mats.append(i)
    col = (rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9))
    rough = rng.uniform(0.05, 1.0)
    materials.append(material(col, rough, 0.0))
    rows.append(rows_from(1.0, (cube / 2, 0.0, cube / 2)))
    mesh_ids.append(1)
    mats.append(num_spheres)
    light = area_light(center=(cube / 2, cube * 1.4, cube / 2), normal=(0, -1, 0), u_axis=(1, 0, 0), width=cube * 0.4,
                       height=cube * 0.4, radiance=light_radiance)
    cam = look_at(eye=(cube / 2, cube * 0.75, -cube * 0.9), target=(cube / 2, cube * 0.3, cube / 2), fov_y_degrees=50.0,
                  width=width, height=height, near=0.05, far=1000.0)
    return Scene([sphere, ground], np.stack(rows).astype(np.float32), np.asarray(mesh_ids, np.uint32),
                 np.asarray(mats, np.uint32), materials, [light], cam, environment(), name=f"spheres{num_spheres}")


# ----------------------------------------------------------------------------- plain method, large
def lamp_scene(width: int = 128, height: int = 96, seed: int = 0, lamps: int = 3, spheres: int = 8, double_sided=False):
    """A floor with diffuse and glossy spheres lit by emissive quads facing down and one
    small emissive sphere (no analytic lights, black world): every light comes through
    surface emission and the mesh next-event strategy."""
    rng = np.random.default_rng(seed)
    meshes = [grid((12.0, 12.0), (4, 4)), grid((1.0, 1.0), (2, 2)), uv_sphere(1.0)]
    rows, mesh_ids, mat_ids = [rows_from(1.0, (0.0, 0.0, 0.0))], [0], [0]
    materials = [material((0.75, 0.75, 0.75), 0.8, 0.0)]
    for k in range(lamps):
        w, d = rng.uniform(0.6, 1.8, 2)
        r = np.zeros((3, 4), np.float32)
        r[0, 0], r[1, 1], r[2, 2] = w, -1.0, -d          # scale in x/z, flipped to face -Y (det > 0)
        r[:, 3] = (rng.uniform(-3.5, 3.5), rng.uniform(2.5, 4.0), rng.uniform(-3.5, 3.5))
        rows.append(r); mesh_ids.append(1); mat_ids.append(len(materials))
        materials.append(emissive(tuple(rng.uniform(0.4, 1.0, 3)), float(rng.uniform(4.0, 20.0)), double_sided))
    rows.append(rows_from(0.3, (rng.uniform(-2.0, 2.0), 1.2, rng.uniform(-2.0, 2.0))))
    mesh_ids.append(2); mat_ids.append(len(materials))
    materials.append(emissive((1.0, 0.6, 0.3), 30.0))
    for k in range(spheres):
        rad = float(rng.uniform(0.3, 0.8))
        rows.append(rows_from(rad, (rng.uniform(-4.0, 4.0), rad, rng.uniform(-4.0, 4.0))))
        mesh_ids.append(2); mat_ids.append(len(materials))
        materials.append(material(tuple(rng.uniform(0.2, 0.9, 3)), float(rng.uniform(0.1, 0.7)), float(k % 3 == 0)))
    cam = look_at((0.0, 5.5, 9.0), (0.0, 0.8, 0.0), width=width, height=height, fov_y_degrees=50)
    return Scene(meshes, np.stack(rows).astype(np.float32), np.asarray(mesh_ids, np.uint32), np.asarray(mat_ids, np.uint32),
                 materials, [], cam, environment((0.0, 0.0, 0.0)), name="lamps")


def value_noise_heights(cells: int, size: float, seed: int = 0, amplitude: float = 30.0, octaves: int = 6) -> np.ndarray:
    """(cells+1)^2 heights of seeded fBm value noise (smoothstep-interpolated lattice values)."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, 1.0, cells + 1)
    h = np.zeros((cells + 1, cells + 1))
    freq, amp = 4, amplitude
    for _ in range(octaves):
        lattice = rng.uniform(-1, 1, (freq + 2, freq + 2))
        u = xs * freq
        i = np.minimum(u.astype(np.int64), freq)
        f = u - i
        f = f * f * (3 - 2 * f)
        a = lattice[i][:, i]; b = lattice[i + 1][:, i]; c = lattice[i][:, i + 1]; d = lattice[i + 1][:, i + 1]
        fz, fx = f[:, None], f[None, :]
        h += amp * ((a * (1 - fz) + b * fz) * (1 - fx) + (c * (1 - fz) + d * fz) * fx)
        freq *= 2
        amp *= 0.5
    return h


class Flock:
    """Seeded boid flock (cohesion, alignment, separation) over a uniform grid of cells.

    Each boid steers toward its cell's mean position and velocity and away from the
    cell mean when crowded, plus a weak pull toward the flock centre.  Cell sums use
    one sort per frame, O(N log N)."""

    def __init__(self, n: int, seed: int = 0, center=(0.0, 60.0, 0.0), extent=(240.0, 60.0, 240.0), cell: float = 4.0):
        rng = np.random.default_rng(seed)
        self.center = np.asarray(center, np.float64)
        self.extent = np.asarray(extent, np.float64)
        self.pos = self.center + (rng.random((n, 3)) - 0.5) * self.extent
        ang = rng.uniform(0, 2 * np.pi, n)
        self.vel = np.stack([np.cos(ang), rng.uniform(-0.2, 0.2, n), np.sin(ang)], 1) * 8.0
        self.cell = cell

    def step(self, dt: float = 1.0 / 24.0):
        key = np.floor(self.pos / self.cell).astype(np.int64)
        k = (key[:, 0] * 73856093) ^ (key[:, 1] * 19349663) ^ (key[:, 2] * 83492791)
        _, inv, counts = np.unique(k, return_inverse=True, return_counts=True)
        cnt = counts[inv][:, None].astype(np.float64)
        mean_p = np.stack([np.bincount(inv, self.pos[:, a]) for a in range(3)], 1)[inv] / cnt
        mean_v = np.stack([np.bincount(inv, self.vel[:, a]) for a in range(3)], 1)[inv] / cnt
        cohesion = (mean_p - self.pos) * 0.5
        alignment = (mean_v - self.vel) * 0.8
        separation = (self.pos - mean_p) * np.minimum(cnt, 8.0) * 0.6
        centre = (self.center - self.pos) / self.extent * 4.0
        self.vel += (cohesion + alignment + separation + centre) * dt
        speed = np.linalg.norm(self.vel, axis=1, keepdims=True)
        self.vel *= np.clip(speed, 4.0, 14.0) / np.maximum(speed, 1e-6)
        self.pos += self.vel * dt

    def rows(self, length: float = 0.35, width: float = 0.14) -> np.ndarray:
        """(N,3,4) object->world rows: the bird's long axis along its velocity."""
        f = self.vel / np.linalg.norm(self.vel, axis=1, keepdims=True)
        up = np.array([0.0, 1.0, 0.0])
        r = np.cross(up, f)
        r /= np.maximum(np.linalg.norm(r, axis=1, keepdims=True), 1e-9)
        u = np.cross(f, r)
        out = np.empty((len(f), 3, 4), np.float32)
        out[:, :, 0] = r * width
        out[:, :, 1] = u * width
        out[:, :, 2] = f * length
        out[:, :, 3] = self.pos
        return out


def flock_scene(num_birds: int = 1_000_000, seed: int = 0, width: int = 1920, height: int = 1080,
                terrain_cells: int = 1000, terrain_size: float = 1000.0, num_materials: int = 16):
    """Plain method, large: `num_birds` instances of a seeded 500-triangle geodesic
    (icosphere-derived) mesh placed by a boid flock, a 2*terrain_cells^2-triangle
    noise-displaced terrain, materials drawn as in the small configuration, a sun and a
    constant environment light.  Returns (Scene, Flock); Flock.step()/rows() give the
    following animation frames."""
    rng = Pcg32(seed)
    bird = geodesic_sphere(5, jitter=0.12, seed=seed)
    terrain = height_grid(value_noise_heights(terrain_cells, terrain_size, seed=seed + 1), terrain_size)
    materials = []
    for _ in range(num_materials):
        col = (rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9))
        rough = rng.uniform(0.05, 1.0)
        metal = 1.0 if rng.uniform() < 0.3 else 0.0
        materials.append(material(col, rough, metal))
    materials.append(material((0.32, 0.28, 0.22), 0.85, 0.0))
    flock = Flock(num_birds, seed=seed + 2)
    rows = np.concatenate([flock.rows(), rows_from(1.0, (0.0, 0.0, 0.0))[None]], 0)
    mesh_ids = np.zeros(num_birds + 1, np.uint32)
    mesh_ids[-1] = 1
    mat_ids = (np.arange(num_birds + 1, dtype=np.uint64) * 2654435761 % num_materials).astype(np.uint32)
    mat_ids[-1] = num_materials
    sun = sun_light(direction=(-0.35, -0.8, 0.45), angle_degrees=0.526, energy=3.0, color=(1.0, 0.95, 0.88))
    cam = look_at(eye=(0.0, 75.0, -330.0), target=(0.0, 48.0, 0.0), fov_y_degrees=40.0, width=width, height=height,
                  near=0.1, far=1e5)
    env = environment(radiance=(0.18, 0.26, 0.42))
    sc = Scene([bird, terrain], rows, mesh_ids, mat_ids, materials, [sun], cam, env, name="flock")
    return sc, flock


# ----------------------------------------------------------------------------- batched previews
def preview_jobs(count: int = 256, seed: int = 0, max_side: int = 1024):
    """Seeded preview jobs: resolution log-uniform 128^2..max_side^2, spp U{4..32},
    depth U{4..8}, a scene of 1k..200k triangles (log-uniform) from the small
    configuration's generator (spheres + ground grid), scene seed = job index.
    Returns [(Scene, spp, depth), ...]."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(count):
        side = int(round(math.exp(rng.uniform(math.log(128), math.log(max_side)))))
        aspect = rng.choice([1.0, 4 / 3, 16 / 9])
        w = max(16, int(round(side * math.sqrt(aspect))))
        h = max(16, int(round(side / math.sqrt(aspect))))
        spp = int(rng.integers(4, 33))
        depth = int(rng.integers(4, 9))
        tris = math.exp(rng.uniform(math.log(1000), math.log(200000)))
        cells = 8 if tris < 20000 else 64
        n_spheres = max(1, int(round((tris - 2 * cells * cells) / 960)))
        sc = spheres_scene(num_spheres=n_spheres, seed=j, width=w, height=h, grid_cells=cells)
        jobs.append((sc, spp, depth))
    return jobs
