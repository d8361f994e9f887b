"""Synthetic scenes and ray batches for the workloads the backend is measured on.

All inputs are generated from seeds (no datasets exist for this path). Geometry is an FP32
triangle soup (n, 9): v0.xyz v1.xyz v2.xyz; triangle ids are soup indices.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import types as T


@dataclass
class Scene:
    verts: np.ndarray                      # (n, 9) float32
    tri_material: np.ndarray               # (n,) uint32
    materials: list = field(default_factory=list)   # dicts: type, rgb, roughness, eta, k
    lights: list = field(default_factory=list)      # dicts: type, tri, radiance, radius, center
    camera: dict | None = None             # position, look_at, up, vfov, width, height
    uvs: np.ndarray | None = None          # (n, 6) float32: (u, v) of each triangle's vertices
    images: list = field(default_factory=list)      # (H, W, 3) uint8 arrays, rows from the top

    @property
    def n_tri(self) -> int:
        return int(self.verts.shape[0])

    def materials_array(self):
        arr = (T.fl_material * max(1, len(self.materials)))()
        for i, m in enumerate(self.materials):
            arr[i].type = m.get("type", T.FL_MAT_LAMBERT)
            arr[i].rgb[:] = list(m.get("rgb", (0.5, 0.5, 0.5)))
            arr[i].roughness = m.get("roughness", 0.0)
            arr[i].eta = m.get("eta", 1.5)
            arr[i].k = m.get("k", 0.0)
            arr[i].standard = -1
            arr[i].texture = m.get("texture", -1) + 1
        # StandardSurfaceMaterial parameters: materials with "standard" get consecutive indices
        k = 0
        for i, m in enumerate(self.materials):
            if "standard" in m:
                arr[i].type = T.FL_MAT_STANDARD
                arr[i].standard = k
                k += 1
        return arr

    def standard_array(self):
        """fl_standard_surface records of the materials that carry a "standard" dict"""
        stds = [m["standard"] for m in self.materials if "standard" in m]
        arr = (T.fl_standard_surface * max(1, len(stds)))()
        for i, p in enumerate(stds):
            for name, _ in T.fl_standard_surface._fields_:
                if name in p:
                    v = p[name]
                    if isinstance(v, (tuple, list)):
                        getattr(arr[i], name)[:] = list(v)
                    else:
                        setattr(arr[i], name, v)
            arr[i].kd_texture = p.get("kd_texture", -1) + 1
            arr[i].bump_texture = p.get("bump_texture", -1) + 1
        return arr, len(stds)

    def images_array(self):
        """fl_image records of self.images plus the contiguous pixel buffers they point to"""
        pix = [np.ascontiguousarray(im, np.uint8) for im in self.images]
        arr = (T.fl_image * max(1, len(pix)))()
        for i, p in enumerate(pix):
            assert p.ndim == 3 and p.shape[2] == 3
            arr[i].height, arr[i].width = p.shape[0], p.shape[1]
            arr[i].rgb = p.ctypes.data_as(C.POINTER(C.c_uint8))
        return arr, pix

    def lights_array(self):
        arr = (T.fl_light * max(1, len(self.lights)))()
        for i, l in enumerate(self.lights):
            arr[i].type = l["type"]
            arr[i].tri = l.get("tri", 0)
            arr[i].radiance = l["radiance"]
            arr[i].radius = l.get("radius", 0.0)
            arr[i].center[:] = list(l.get("center", (0.0, 0.0, 0.0)))
            arr[i].direction[:] = list(l.get("direction", (0.0, -1.0, 0.0)))
            arr[i].cone_angle = l.get("cone_angle", 0.0)
            arr[i].penumbra_angle = l.get("penumbra_angle", 0.0)
        return arr

    def desc(self):
        """fl_scene_desc plus the buffers it points to (keep the tuple alive while used)."""
        verts = np.ascontiguousarray(self.verts, dtype=np.float32)
        tm = np.ascontiguousarray(self.tri_material, dtype=np.uint32)
        mats = self.materials_array()
        lights = self.lights_array()
        d = T.fl_scene_desc()
        d.verts = verts.ctypes.data_as(C.POINTER(C.c_float))
        d.n_tri = verts.shape[0]
        d.tri_material = tm.ctypes.data_as(C.POINTER(C.c_uint32))
        d.materials = C.cast(mats, C.POINTER(T.fl_material))
        d.n_materials = len(self.materials)
        d.lights = C.cast(lights, C.POINTER(T.fl_light))
        d.n_lights = len(self.lights)
        stds, n_std = self.standard_array()
        d.standard_surfaces = C.cast(stds, C.POINTER(T.fl_standard_surface))
        d.n_standard_surfaces = n_std
        uvs = None
        if self.uvs is not None:
            uvs = np.ascontiguousarray(self.uvs, np.float32).reshape(self.n_tri, 6)
            d.uvs = uvs.ctypes.data_as(C.POINTER(C.c_float))
        imgs, pix = self.images_array()
        d.images = C.cast(imgs, C.POINTER(T.fl_image))
        d.n_images = len(self.images)
        return d, (verts, tm, mats, lights, stds, uvs, imgs, pix)

    def camera_struct(self, width=None, height=None):
        c = self.camera
        cam = T.fl_camera()
        cam.position[:] = list(c["position"])
        cam.look_at[:] = list(c["look_at"])
        cam.up[:] = list(c.get("up", (0.0, 1.0, 0.0)))
        cam.vfov_deg = c["vfov"]
        cam.width = width or c["width"]
        cam.height = height or c["height"]
        cam.aperture = c.get("aperture", 0.0)
        return cam


def render_params(spp, max_depth, mode=T.FL_SPECTRAL_HERO4, rr=1.0, wave_paths=0, sample_offset=0, flags=0,
                  depths=None):
    """fl_render_params; depths=(diffuse, reflection, transmission) sets RenderParams' three
    depths (FL_RENDER_LOBE_DEPTHS) in place of max_depth for all three."""
    p = T.fl_render_params()
    p.flags = flags
    p.spp = spp
    p.max_depth = max_depth
    if depths is not None:
        p.flags |= T.FL_RENDER_LOBE_DEPTHS
        p.diffuse_depth, p.reflection_depth, p.transmission_depth = (int(d) for d in depths)
    p.rr_threshold = rr
    p.spectral_mode = mode
    p.wave_paths = wave_paths
    p.sample_offset = sample_offset
    return p


# ----------------------------------------------------------------------------- geometry helpers

def _quad(p0, p1, p2, p3):
    """two triangles (p0,p1,p2), (p0,p2,p3); normal = (p1-p0) x (p2-p0)"""
    return [list(p0) + list(p1) + list(p2), list(p0) + list(p2) + list(p3)]


def _box(cx, cz, sx, sy, sz, angle_deg, outward=False):
    """axis box of size (sx, sy, sz) standing on y = 0, centred at (cx, cz), rotated about y.
    The faces' geometric normals (Triangle::intersect's cross(v1 - v3, v2 - v3)) point into
    the box; outward=True reverses the winding so that they point out."""
    a = math.radians(angle_deg)
    ca, sa = math.cos(a), math.sin(a)

    def P(x, y, z):
        dx, dz = x - cx, z - cz
        return (cx + dx * ca + dz * sa, y, cz - dx * sa + dz * ca)

    x0, x1 = cx - sx / 2, cx + sx / 2
    z0, z1 = cz - sz / 2, cz + sz / 2
    y0, y1 = 0.0, sy
    c = [P(x0, y0, z0), P(x1, y0, z0), P(x1, y0, z1), P(x0, y0, z1),
         P(x0, y1, z0), P(x1, y1, z0), P(x1, y1, z1), P(x0, y1, z1)]
    faces = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (2, 3, 7, 6), (1, 2, 6, 5), (3, 0, 4, 7)]
    tris = []
    for f in faces:
        tris += _quad(*(c[i] for i in (f[::-1] if outward else f)))
    return tris


def cornell(width=256, height=256, variant="lambert") -> Scene:
    """Cornell-style box of 36 triangles (unit-cube room open at z = 0, two rotated boxes,
    0.25 x 0.25 ceiling light at y = 0.999 facing down with constant spectral radiance 10).
    variant "lambert": every surface Lambertian; "standard" / "standard2" / "standard3": the boxes are
    StandardSurface materials (see below); "materials": short box GGX conductor
    (roughness 0.3, eta 0.2, k 3.9), tall box rough dielectric (roughness 0.25, IOR 1.5);
    "glass": short box conductor (roughness 0.05), tall box smooth glass (IOR 1.5)."""
    tris, mats = [], []
    WHITE, RED, GREEN = 0, 1, 2
    SHORT, TALL = (3, 4) if variant != "lambert" else (WHITE, WHITE)
    # floor, ceiling, back wall (white)
    tris += _quad((0, 0, 0), (0, 0, 1), (1, 0, 1), (1, 0, 0)); mats += [WHITE] * 2
    tris += _quad((0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1)); mats += [WHITE] * 2
    tris += _quad((0, 0, 1), (0, 1, 1), (1, 1, 1), (1, 0, 1)); mats += [WHITE] * 2
    # image-left wall (x = 0, red), image-right wall (x = 1, green)
    tris += _quad((0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1)); mats += [RED] * 2
    tris += _quad((1, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0)); mats += [GREEN] * 2
    # short box (front, image right), tall box (back, image left)
    # ("standard3": outward normals, so that the thin film and the thin walls see their
    # outside from the room)
    out = variant == "standard3"
    tris += _box(0.66, 0.37, 0.3, 0.3, 0.3, -17.0, out); mats += [SHORT] * 12
    tris += _box(0.33, 0.67, 0.3, 0.6, 0.3, 17.0, out); mats += [TALL] * 12
    # light quad, normal (0, -1, 0)
    h, lo, hi = 0.999, 0.375, 0.625
    light_first = len(tris)
    tris += _quad((lo, h, lo), (hi, h, lo), (hi, h, hi), (lo, h, hi)); mats += [WHITE] * 2
    verts = np.asarray(tris, dtype=np.float32)
    materials = [
        {"type": T.FL_MAT_LAMBERT, "rgb": (0.725, 0.725, 0.725)},
        {"type": T.FL_MAT_LAMBERT, "rgb": (0.63, 0.065, 0.05)},
        {"type": T.FL_MAT_LAMBERT, "rgb": (0.14, 0.45, 0.091)},
    ]
    if variant == "materials":
        materials += [{"type": T.FL_MAT_CONDUCTOR, "roughness": 0.3, "eta": 0.2, "k": 3.9},
                      {"type": T.FL_MAT_ROUGH_DIELECTRIC, "roughness": 0.25, "eta": 1.5}]
    elif variant == "glass":
        materials += [{"type": T.FL_MAT_CONDUCTOR, "roughness": 0.05, "eta": 0.2, "k": 3.9},
                      {"type": T.FL_MAT_SMOOTH_DIELECTRIC, "eta": 1.5}]
    elif variant == "standard":
        # StandardSurface: Oren-Nayar diffuse with sheen; Fresnel-blended anisotropic GGX with a clear coat
        materials += [{"standard": {"kd": (0.8, 0.6, 0.3), "kd_weight": 1.0, "kd_roughness": 0.5,
                                    "sheen_color": (0.9, 0.9, 1.0), "sheen_weight": 0.8, "sheen_roughness": 0.4}},
                      {"standard": {"kd": (0.2, 0.4, 0.8), "kd_weight": 0.9, "kd_roughness": 0.3,
                                    "ks": (0.9, 0.9, 0.9), "ks_weight": 0.8, "ks_roughness": 0.35,
                                    "ks_anisotropic": 0.4, "ks_ior": 1.5, "fresnel_type": T.FL_FRESNEL_DIELECTRIC,
                                    "coat_color": (1.0, 1.0, 1.0), "coat_weight": 0.6, "coat_ior": 1.5,
                                    "coat_gloss": 0.7}}]
    elif variant == "standard2":
        # StandardSurface: Schlick-metallic blended lobe; glass-like specular transmission (R = ks, T = kt)
        materials += [{"standard": {"kd": (0.5, 0.5, 0.5), "kd_weight": 0.5, "kd_roughness": 0.2,
                                    "ks": (0.95, 0.7, 0.3), "ks_weight": 1.0, "ks_roughness": 0.25, "ks_ior": 1.5,
                                    "fresnel_type": T.FL_FRESNEL_METALLIC}},
                      {"standard": {"ks": (1.0, 1.0, 1.0), "ks_weight": 1.0, "ks_ior": 1.5, "ks_roughness": 0.2,
                                    "kt": (0.9, 0.95, 1.0), "kt_weight": 1.0, "sheen_color": (1.0, 0.8, 0.8),
                                    "sheen_weight": 0.3, "sheen_roughness": 0.5}}]
    elif variant == "standard3":
        # StandardSurface: thin-walled diffuse transmission with sheen; measured copper (Oren-Nayar
        # diffuse, anisotropic GGX conductor) under a thin film and a clear coat
        materials += [{"standard": {"kd": (0.3, 0.7, 0.4), "kd_weight": 1.0, "kd_roughness": 0.6, "thin_walled": 1,
                                    "sheen_color": (0.8, 0.8, 1.0), "sheen_weight": 0.5, "sheen_roughness": 0.3}},
                      {"standard": {"kd": (0.5, 0.5, 0.5), "kd_weight": 0.4, "kd_roughness": 0.5,
                                    "ks": (1.0, 1.0, 1.0), "ks_weight": 0.9, "ks_roughness": 0.3,
                                    "ks_anisotropic": 0.2, "ks_ior": 1.8,
                                    "fresnel_type": T.FL_FRESNEL_MEASURED_METAL, "metal_type": 1,
                                    "thin_film_thickness": 350.0, "thin_film_ior": 1.33,
                                    "coat_color": (1.0, 1.0, 1.0), "coat_weight": 0.3, "coat_ior": 1.5,
                                    "coat_gloss": 0.8}}]
    lights = [{"type": T.FL_LIGHT_TRIANGLE, "tri": light_first + k, "radiance": 10.0} for k in range(2)]
    cam = {"position": (0.5, 0.5, -1.4), "look_at": (0.5, 0.5, 0.0), "up": (0.0, 1.0, 0.0), "vfov": 40.0,
           "width": width, "height": height}
    return Scene(verts, np.asarray(mats, dtype=np.uint32), materials, lights, cam)


# ----------------------------------------------------------------------------- ray-cast microbenchmark

def triangle_soup(n_tri: int, seed: int = 1, sigma: float = 0.002) -> np.ndarray:
    """n_tri triangles: centroids uniform in [0,1]^3, vertex = centroid + N(0, sigma^2) per component."""
    rng = np.random.default_rng(seed)
    c = rng.random((n_tri, 1, 3), dtype=np.float32)
    e = rng.standard_normal((n_tri, 3, 3), dtype=np.float32) * np.float32(sigma)
    return (c + e).reshape(n_tri, 9).astype(np.float32)


def incoherent_rays(n: int, seed: int = 2, lo: float = -0.1, hi: float = 1.1):
    """origins uniform in [lo, hi]^3, directions uniform on the sphere, tmin 0, tmax +inf."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    d = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1).astype(np.float32)
    org = np.empty((n, 4), np.float32)
    dirs = np.empty((n, 4), np.float32)
    org[:, :3] = o
    org[:, 3] = 0.0
    dirs[:, :3] = d
    dirs[:, 3] = np.inf
    return org, dirs


def coherent_rays(width: int, height: int, position=(0.5, 0.5, -1.0), look_at=(0.5, 0.5, 0.5), vfov=60.0):
    """pinhole primary rays through pixel centres, row 0 at the top."""
    pos = np.asarray(position, np.float64)
    w = pos - np.asarray(look_at, np.float64)
    w /= np.linalg.norm(w)
    u = np.cross([0.0, 1.0, 0.0], w)
    u /= np.linalg.norm(u)
    v = np.cross(w, u)
    hh = math.tan(math.radians(vfov) / 2)
    hw = hh * width / height
    xs = (np.arange(width) + 0.5) / width
    ys = 1.0 - (np.arange(height) + 0.5) / height
    X, Y = np.meshgrid(xs, ys)
    d = (-w[None, None, :] + (2 * X[..., None] - 1) * hw * u[None, None, :] + (2 * Y[..., None] - 1) * hh * v[None, None, :])
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    n = width * height
    org = np.empty((n, 4), np.float32)
    dirs = np.empty((n, 4), np.float32)
    org[:, :3] = pos.astype(np.float32)
    org[:, 3] = 0.0
    dirs[:, :3] = d.reshape(n, 3).astype(np.float32)
    dirs[:, 3] = np.inf
    return org, dirs


# ----------------------------------------------------------------------------- procedural spheres

def uv_sphere(slices: int, stacks: int) -> np.ndarray:
    """unit UV sphere with fan poles: 2 * slices * (stacks - 1) triangles, outward winding
    (stacks bands between the poles; slices=128, stacks=65 gives 16,384 triangles)."""
    th = np.linspace(0.0, math.pi, stacks + 1)[1:-1]          # interior rings
    ph = np.linspace(0.0, 2.0 * math.pi, slices + 1)[:-1]
    st, ct = np.sin(th), np.cos(th)
    ring = np.stack([st[:, None] * np.cos(ph)[None, :], np.broadcast_to(ct[:, None], (th.size, ph.size)),
                     st[:, None] * np.sin(ph)[None, :]], -1)    # (rings, slices, 3)
    top, bot = np.array([0.0, 1.0, 0.0]), np.array([0.0, -1.0, 0.0])
    j = np.arange(slices)
    jn = (j + 1) % slices
    tris = []
    r0 = ring[0]
    tris.append(np.concatenate([np.broadcast_to(top, (slices, 3)), r0[jn], r0[j]], -1))
    for k in range(ring.shape[0] - 1):
        a, b = ring[k], ring[k + 1]
        tris.append(np.concatenate([a[j], a[jn], b[jn]], -1))
        tris.append(np.concatenate([a[j], b[jn], b[j]], -1))
    rl = ring[-1]
    tris.append(np.concatenate([np.broadcast_to(bot, (slices, 3)), rl[j], rl[jn]], -1))
    return np.concatenate(tris, 0)


def value_noise(p: np.ndarray, seed: int, freq: float = 3.0) -> np.ndarray:
    """seeded 3D value noise in [-1, 1]: random lattice values, smoothstep-trilinear blend."""
    rng = np.random.default_rng(seed)
    table = rng.uniform(-1.0, 1.0, 4096)
    perm = rng.permutation(4096)
    q = p * freq
    i0 = np.floor(q).astype(np.int64)
    f = q - i0
    w = f * f * (3.0 - 2.0 * f)

    def lat(ix, iy, iz):
        h = perm[(ix * 73856093 ^ iy * 19349663 ^ iz * 83492791) & 4095]
        return table[h]

    out = 0.0
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                wx = w[:, 0] if dx else 1 - w[:, 0]
                wy = w[:, 1] if dy else 1 - w[:, 1]
                wz = w[:, 2] if dz else 1 - w[:, 2]
                out = out + wx * wy * wz * lat(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz)
    return out


def procedural_spheres(n_spheres=64, slices=128, stacks=65, width=1920, height=1080, seed=7, extent=10.0,
                       sphere_light=(0.0, 6.0, 0.0, 0.5, 40.0), env=0.5) -> Scene:
    """Spheres of `2 * slices * (stacks - 1)` triangles radially displaced by value noise of
    amplitude 0.05 r, radii U[0.2, 1], centres U[-extent, extent]^2 resting on a 2-triangle
    ground plane; 40% Lambert (albedo U[0.1, 0.9]), 40% GGX conductor (roughness U[0.05, 0.8],
    eta 0.2, k 3.9), 20% rough dielectric (IOR 1.5, roughness U[0, 0.3]); constant environment
    radiance plus one sphere light (x, y, z, radius, radiance). The default is the
    1,048,578-triangle scene at 1920x1080."""
    rng = np.random.default_rng(seed)
    unit = uv_sphere(slices, stacks).reshape(-1, 3, 3)
    flat = unit.reshape(-1, 3)
    tris, mats, materials = [], [], []
    g = 2.0 * extent
    ground = np.array([[-g, 0, -g, -g, 0, g, g, 0, g], [-g, 0, -g, g, 0, g, g, 0, -g]], np.float32)
    tris.append(ground)
    materials.append({"type": 0, "rgb": (0.5, 0.5, 0.5)})
    mats.append(np.zeros(2, np.uint32))
    for s in range(n_spheres):
        r = rng.uniform(0.2, 1.0)
        cx, cz = rng.uniform(-extent, extent, 2)
        disp = 1.0 + 0.05 * value_noise(flat, seed * 1000 + s)
        v = (flat * (r * disp)[:, None] + np.array([cx, r, cz])).reshape(-1, 9)
        tris.append(v.astype(np.float32))
        u = rng.uniform()
        if u < 0.4:
            a = rng.uniform(0.1, 0.9)
            materials.append({"type": 0, "rgb": (a, a, a)})
        elif u < 0.8:
            materials.append({"type": 1, "roughness": rng.uniform(0.05, 0.8), "eta": 0.2, "k": 3.9})
        else:
            materials.append({"type": 2, "roughness": rng.uniform(0.0, 0.3), "eta": 1.5})
        mats.append(np.full(v.shape[0], len(materials) - 1, np.uint32))
    verts = np.concatenate(tris, 0).astype(np.float32)
    lx, ly, lz, lr, le = sphere_light
    lights = [{"type": 1, "radiance": le, "radius": lr, "center": (lx, ly, lz)}, {"type": 2, "radiance": env}]
    cam = {"position": (0.0, 0.7 * extent, -2.1 * extent), "look_at": (0.0, 0.5, 0.0), "up": (0.0, 1.0, 0.0),
           "vfov": 40.0, "width": width, "height": height}
    return Scene(verts, np.concatenate(mats), materials, lights, cam)


def sphere_library(slices: int, stacks: int, n: int = 8, seed: int = 3) -> np.ndarray:
    """n unit UV spheres (2 * slices * (stacks - 1) triangles each), each radially displaced by
    its own value noise of amplitude 0.05: (n, triangles, 9) float32, to be scaled and placed."""
    flat = uv_sphere(slices, stacks).reshape(-1, 3)
    out = []
    for k in range(n):
        disp = 1.0 + 0.05 * value_noise(flat, seed * 1000 + k)
        out.append((flat * disp[:, None]).reshape(-1, 9).astype(np.float32))
    return np.stack(out)


def request_scene(n_tri_target: float, seed: int, width: int, height: int, libraries: dict) -> Scene:
    """A procedural scene of the procedural_spheres kind with about n_tri_target triangles, fast
    enough to make per request: spheres of 16,384 triangles (1,024 below 131,072 triangles)
    taken from a library of pre-displaced unit spheres (`libraries[(slices, stacks)]`, from
    sphere_library), radii U[0.2, 1], centres U[-e, e]^2 with e growing as the square root of
    the sphere count, the same material mix, a ground plane, an environment and a sphere light."""
    rng = np.random.default_rng(seed)
    key = (128, 65) if n_tri_target >= 16384 * 8 else (32, 17)
    lib = libraries[key]
    per = lib.shape[1]
    n_sph = max(1, int(round(n_tri_target / per)))
    extent = max(3.0, 10.0 * (n_sph / 64) ** 0.5)
    pick = rng.integers(0, lib.shape[0], n_sph)
    r = rng.uniform(0.2, 1.0, n_sph).astype(np.float32)
    c = np.zeros((n_sph, 3), np.float32)
    c[:, 0] = rng.uniform(-extent, extent, n_sph)
    c[:, 1] = r
    c[:, 2] = rng.uniform(-extent, extent, n_sph)
    sph = (lib[pick].reshape(n_sph, per, 3, 3) * r[:, None, None, None] + c[:, None, None, :]).reshape(-1, 9)
    g = 2.0 * extent
    ground = np.array([[-g, 0, -g, -g, 0, g, g, 0, g], [-g, 0, -g, g, 0, g, g, 0, -g]], np.float32)
    verts = np.concatenate([ground, sph]).astype(np.float32)
    materials = [{"type": 0, "rgb": (0.5, 0.5, 0.5)}]
    u = rng.uniform(size=n_sph)
    for k in range(n_sph):
        if u[k] < 0.4:
            a = rng.uniform(0.1, 0.9)
            materials.append({"type": 0, "rgb": (a, a, a)})
        elif u[k] < 0.8:
            materials.append({"type": 1, "roughness": rng.uniform(0.05, 0.8), "eta": 0.2, "k": 3.9})
        else:
            materials.append({"type": 2, "roughness": rng.uniform(0.0, 0.3), "eta": 1.5})
    mats = np.concatenate([np.zeros(2, np.uint32), np.repeat(np.arange(1, n_sph + 1, dtype=np.uint32), per)])
    lights = [{"type": 1, "radiance": 40.0, "radius": 0.5, "center": (0.0, 6.0, 0.0)}, {"type": 2, "radiance": 0.5}]
    cam = {"position": (0.0, 0.7 * extent, -2.1 * extent), "look_at": (0.0, 0.5, 0.0), "up": (0.0, 1.0, 0.0),
           "vfov": 40.0, "width": width, "height": height}
    return Scene(verts, mats, materials, lights, cam)


def delta_lights():
    """A point light, a spot light (30 degree cone, 20 degree full-intensity core, tilted down
    the box) and a directional light entering through the open side of the Cornell box."""
    return [
        {"type": T.FL_LIGHT_POINT, "radiance": 1.5, "center": (0.5, 0.8, 0.5)},
        {"type": T.FL_LIGHT_SPOT, "radiance": 3.0, "center": (0.3, 0.95, 0.6), "direction": (0.1, -1.0, 0.2),
         "cone_angle": float(np.radians(30.0)), "penumbra_angle": float(np.radians(20.0))},
        {"type": T.FL_LIGHT_DIRECTIONAL, "radiance": 2.0, "direction": (0.2, -0.3, 1.0)},
    ]


def cornell_delta(width=64, height=64, variant="lambert") -> Scene:
    """The Cornell box with the point, spot and directional lights of delta_lights() added to
    its ceiling light."""
    sc = cornell(width, height, variant)
    return Scene(sc.verts, sc.tri_material, sc.materials, list(sc.lights) + delta_lights(), sc.camera)


def caustic(width=1024, height=1024, slices=256, stacks=129) -> Scene:
    """Lambertian room of 12 triangles (albedo 0.7), a sphere light of radius 0.02 and
    radiance 5e3, and a smooth glass sphere (IOR 1.5, radius 1, 2*slices*(stacks-1) =
    65,536 triangles by default) above the floor."""
    tris = []
    lo, hi = -3.0, 3.0
    c = [(lo, 0, lo), (hi, 0, lo), (hi, 0, hi), (lo, 0, hi), (lo, 6, lo), (hi, 6, lo), (hi, 6, hi), (lo, 6, hi)]
    for f in [(0, 1, 2, 3), (7, 6, 5, 4), (0, 4, 5, 1), (2, 6, 7, 3), (1, 5, 6, 2), (3, 7, 4, 0)]:
        tris += _quad(*(c[i] for i in f))
    room = np.asarray(tris, np.float32)
    glass = (uv_sphere(slices, stacks).reshape(-1, 3) * 1.0 + np.array([0.0, 1.6, 0.0])).reshape(-1, 9)
    verts = np.concatenate([room, glass.astype(np.float32)], 0)
    mats = np.concatenate([np.zeros(room.shape[0], np.uint32), np.ones(glass.shape[0], np.uint32)])
    materials = [{"type": 0, "rgb": (0.7, 0.7, 0.7)}, {"type": 3, "eta": 1.5}]
    lights = [{"type": 1, "radiance": 5e3, "radius": 0.02, "center": (0.3, 4.2, 0.2)}]
    cam = {"position": (0.0, 3.0, -2.9), "look_at": (0.0, 1.0, 0.5), "up": (0.0, 1.0, 0.0), "vfov": 60.0,
           "width": width, "height": height}
    return Scene(verts, mats, materials, lights, cam)


def texture_images(seed=11):
    """two seeded RGB images: a 48 x 32 checkerboard of random colours (6 x 4 cells) and a
    37 x 29 image of smooth colour ramps with noise (odd sizes exercise the texel rule)"""
    rng = np.random.default_rng(seed)
    cells = rng.integers(20, 236, size=(4, 6, 3))
    checker = np.repeat(np.repeat(cells, 8, axis=0), 8, axis=1).astype(np.uint8)
    y, x = np.mgrid[0:29, 0:37]
    ramp = np.stack([x * 255 / 36, y * 255 / 28, (x + y) * 255 / 64], axis=-1)
    ramp = np.clip(ramp + rng.normal(0, 12, ramp.shape), 0, 255).astype(np.uint8)
    return [checker, ramp]


def quad_uvs(n_tri):
    """uvs of the _quad triangles (p0, p1, p2), (p0, p2, p3): the quad maps onto [0, 1]^2"""
    one = np.array([[0, 0, 1, 0, 1, 1], [0, 0, 1, 1, 0, 1]], np.float32)
    return np.tile(one, (n_tri // 2, 1))


def cornell_textured(width=64, height=64, bump=False) -> Scene:
    """The Cornell box with image textures (ImageMapTexture): the back wall and the tall box
    are Lambert with the checkerboard, the floor Lambert with the ramp image, the short box a
    StandardSurface (Oren-Nayar diffuse + sheen) whose kd is the ramp image. Every quad maps
    onto [0, 1]^2; on the box faces u runs over [-0.15, 1.15] and v over [0, 1.15], so that
    the texel rule's clamps are reached. (v < 0 would send the reference past its image:
    for a row past the last it resets the column instead of the row.) bump: the short box
    also takes the ramp image's red channel as its bump map, and the tall box becomes a
    bumped StandardSurface over the checkerboard (Fresnel-blended GGX)."""
    sc = cornell(width, height, "lambert")
    CHECKER, RAMP, STD = len(sc.materials), len(sc.materials) + 1, len(sc.materials) + 2
    mats = list(sc.materials) + [
        {"type": T.FL_MAT_LAMBERT, "texture": 0},
        {"type": T.FL_MAT_LAMBERT, "texture": 1},
        {"standard": {"kd_texture": 1, "kd_weight": 1.0, "kd_roughness": 0.4,
                      "sheen_color": (0.9, 0.9, 1.0), "sheen_weight": 0.4, "sheen_roughness": 0.3}},
    ]
    tm = np.array(sc.tri_material, np.uint32)
    tm[0:2] = RAMP       # floor
    tm[4:6] = CHECKER    # back wall
    tm[10:22] = STD      # short box
    tm[22:34] = CHECKER  # tall box
    if bump:
        mats[STD] = {"standard": dict(mats[STD]["standard"], bump_texture=1)}
        mats.append({"standard": {"kd_texture": 0, "kd_weight": 0.8, "kd_roughness": 0.2, "ks": (0.9, 0.9, 0.9),
                                  "ks_weight": 0.7, "ks_roughness": 0.3, "ks_ior": 1.5, "bump_texture": 0}})
        tm[22:34] = len(mats) - 1
    uvs = quad_uvs(sc.n_tri)
    uvs[10:34, 0::2] = uvs[10:34, 0::2] * 1.3 - 0.15   # u in [-0.15, 1.15]
    uvs[10:34, 1::2] = uvs[10:34, 1::2] * 1.15          # v in [0, 1.15]
    return Scene(sc.verts, tm, mats, sc.lights, sc.camera, uvs=uvs, images=texture_images())
