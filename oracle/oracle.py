"""ctypes wrapper of liboracle.so and oracle/_ref/ref_render.

ORACLE — test infrastructure only: imported by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py, as the checker or as the timed CPU baseline. The product path
(filianore_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "filianore-core_b200"))
from filianore_b200 import types as T  # noqa: E402  (struct layouts only)

LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "ref_render")

_lib = None


def build(ref: bool = False, ref_dir: str | None = None) -> None:
    """liboracle.so; with ref, also _ref/ref_render from the reference tree ref_dir (default:
    $FL_REFERENCE_DIR)."""
    targets = ["all"] + (["ref"] if ref else []) + ([f"REF={ref_dir}"] if ref and ref_dir else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.orc_bvh_build.restype = C.c_void_p
        L.orc_bvh_build.argtypes = [P(C.c_float), C.c_uint32]
        L.orc_bvh_free.argtypes = [C.c_void_p]
        L.orc_bvh_node_count.restype = C.c_uint32
        L.orc_bvh_node_count.argtypes = [C.c_void_p]
        L.orc_trace_closest.argtypes = [C.c_void_p, P(C.c_float), P(C.c_float), C.c_uint32, C.c_void_p, C.c_int,
                                        P(C.c_uint64), P(C.c_uint64)]
        L.orc_trace_brute.argtypes = [P(C.c_float), C.c_uint32, P(C.c_float), P(C.c_float), C.c_uint32, C.c_void_p]
        L.orc_pcg32_sequence.argtypes = [C.c_uint64, C.c_uint64, C.c_int64, C.c_uint32, P(C.c_uint32)]
        L.orc_tables_init.argtypes = [C.c_void_p, P(T.fl_spectral_tables)]
        L.orc_tables_init.restype = C.c_int
        L.orc_tables_binned.argtypes = [C.c_void_p, P(C.c_float)]
        L.orc_average_spectrum_samples.restype = C.c_float
        L.orc_average_spectrum_samples.argtypes = [P(C.c_float), P(C.c_float), C.c_int, C.c_float, C.c_float]
        L.orc_reflectance.argtypes = [C.c_void_p, P(C.c_float), C.c_int, P(C.c_float), P(C.c_float)]
        L.orc_render.argtypes = [P(T.fl_scene_desc), C.c_void_p, P(T.fl_camera), P(T.fl_render_params), C.c_void_p,
                                 P(C.c_double), C.c_void_p]
        L.orc_render.restype = C.c_int
        L.orc_camera_rays.argtypes = [P(T.fl_camera), P(C.c_uint32), C.c_uint32, C.c_uint32, P(C.c_float),
                                      P(C.c_float), P(C.c_uint64), P(C.c_float)]
        L.orc_li.argtypes = [P(T.fl_scene_desc), C.c_void_p, P(T.fl_render_params), C.c_uint32, P(C.c_float),
                             P(C.c_float), P(C.c_uint64), P(C.c_float), P(C.c_float), P(C.c_uint64), P(C.c_double)]
        L.orc_li.restype = C.c_int
        L.orc_guide_eval.argtypes = [P(C.c_float), P(C.c_float), C.c_uint32, P(C.c_float), P(C.c_float), P(C.c_float)]
        L.orc_guide_gradient.argtypes = [P(C.c_float), P(C.c_float), C.c_uint32, P(C.c_float), P(C.c_float),
                                         P(C.c_float), C.c_int]
        L.orc_guide_gradient.restype = C.c_float
        L.orc_guide_set_exact.argtypes = [C.c_int]
        L.orc_bsdf_fcos.argtypes = [P(T.fl_material), P(C.c_float), C.c_uint32, P(C.c_float), C.c_int, P(C.c_float)]
        L.orc_image_texels.argtypes = [P(T.fl_image), P(C.c_float), C.c_uint32, P(C.c_float)]
        _lib = L
    return _lib


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


# ----------------------------------------------------------------------------- tracing

class CpuBVH:
    def __init__(self, tris: np.ndarray):
        self.tris = np.ascontiguousarray(tris, dtype=np.float32)
        self.h = lib().orc_bvh_build(_fp(self.tris), self.tris.shape[0])

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_bvh_free(self.h)
            self.h = None

    @property
    def node_count(self):
        return lib().orc_bvh_node_count(self.h)

    def trace(self, org, dirs, nthreads=None, counts=False):
        org = np.ascontiguousarray(org, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        n = org.shape[0]
        hits = np.zeros(n, dtype=T.HIT_DTYPE)
        nv, nt = C.c_uint64(0), C.c_uint64(0)
        lib().orc_trace_closest(self.h, _fp(org), _fp(dirs), n, hits.ctypes.data, nthreads or os.cpu_count() or 1,
                                C.byref(nv), C.byref(nt))
        return (hits, nv.value, nt.value) if counts else hits


def trace_brute(tris, org, dirs):
    tris = np.ascontiguousarray(tris, np.float32)
    org = np.ascontiguousarray(org, np.float32)
    dirs = np.ascontiguousarray(dirs, np.float32)
    hits = np.zeros(org.shape[0], dtype=T.HIT_DTYPE)
    lib().orc_trace_brute(_fp(tris), tris.shape[0], _fp(org), _fp(dirs), org.shape[0], hits.ctypes.data)
    return hits


def pcg32_sequence(initstate, initseq=1, advance=0, n=16):
    out = np.zeros(n, np.uint32)
    lib().orc_pcg32_sequence(initstate, initseq, advance, n, out.ctypes.data_as(C.POINTER(C.c_uint32)))
    return out


# ----------------------------------------------------------------------------- spectra

ORC_TABLES_SIZE = 1 << 16  # >= sizeof(orc_tables)


class Tables:
    """orc_tables initialised from a spectral-tables dict (see spectral_tables_struct)."""

    def __init__(self, tables: dict):
        self.raw = tables
        self.struct, self._keep = spectral_tables_struct(tables)
        self.buf = C.create_string_buffer(ORC_TABLES_SIZE)
        rc = lib().orc_tables_init(self.buf, C.byref(self.struct))
        assert rc == 0, "orc_tables_init failed"

    def binned(self):
        out = np.zeros(17 * 60, np.float32)
        lib().orc_tables_binned(self.buf, _fp(out))
        return out.reshape(17, 60)

    def metals(self):
        out = np.zeros(9 * 2 * 60, np.float32)
        lib().orc_tables_metals(self.buf, _fp(out))
        return out.reshape(9, 2, 60)

    def reflectance(self, rgb, mode=T.FL_SPECTRAL_BINS60, lambdas=None):
        rgb = np.asarray(rgb, np.float32)
        lam = np.asarray(lambdas if lambdas is not None else np.zeros(4), np.float32)
        out = np.zeros(60, np.float32)
        lib().orc_reflectance(self.buf, _fp(rgb), mode, _fp(lam), _fp(out))
        return out if mode == T.FL_SPECTRAL_BINS60 else out[:4]


def spectral_tables_struct(t: dict):
    keep = {k: np.ascontiguousarray(v, np.float32) for k, v in t.items() if isinstance(v, np.ndarray)}
    s = T.fl_spectral_tables()
    s.cie_lambda = _fp(keep["cie_lambda"])
    s.cie_x = _fp(keep["cie_x"])
    s.cie_y = _fp(keep["cie_y"])
    s.cie_z = _fp(keep["cie_z"])
    s.n_cie = keep["cie_lambda"].shape[0]
    s.cie_y_integral = float(t["cie_y_integral"])
    s.rgb2spec_lambda = _fp(keep["rgb_lambda"])
    s.n_rgb2spec = keep["rgb_lambda"].shape[0]
    rows_r = [np.ascontiguousarray(r) for r in keep["refl"]]
    rows_i = [np.ascontiguousarray(r) for r in keep["illum"]]
    for b in range(7):
        s.refl[b] = _fp(rows_r[b])
        s.illum[b] = _fp(rows_i[b])
    metals = T.set_metal_tables(s, t, _fp)
    return s, (keep, rows_r, rows_i, metals)


# ----------------------------------------------------------------------------- render

def render(scene, tables: Tables, params, nthreads=None, pixels=None, width=None, height=None):
    """returns (film_xyz_sums (H, W, 3) float64, counts dict)"""
    desc, keep = scene.desc()
    cam = scene.camera_struct(width, height)
    W, H = cam.width, cam.height
    film = np.zeros((H * W * 3,), np.float64)

    class Opts(C.Structure):
        _fields_ = [("nthreads", C.c_int), ("pixels", C.POINTER(C.c_uint32)), ("n_pixels", C.c_uint32)]

    class Counts(C.Structure):
        _fields_ = [("paths", C.c_uint64), ("rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("bounces", C.c_uint64)]

    opts = Opts()
    opts.nthreads = nthreads or os.cpu_count() or 1
    px = None
    if pixels is not None:
        px = np.ascontiguousarray(pixels, np.uint32)
        opts.pixels = px.ctypes.data_as(C.POINTER(C.c_uint32))
        opts.n_pixels = px.shape[0]
    cnt = Counts()
    rc = lib().orc_render(C.byref(desc), tables.buf, C.byref(cam), C.byref(params), C.byref(opts),
                          film.ctypes.data_as(C.POINTER(C.c_double)), C.byref(cnt))
    assert rc == 0, "orc_render failed"
    return film.reshape(H, W, 3), {"paths": cnt.paths, "rays": cnt.rays, "shadow_rays": cnt.shadow_rays,
                                   "bounces": cnt.bounces}


def camera_rays(scene, pixels, sample=0, width=None, height=None):
    """the render loop's camera rays of `sample` for the given pixels: (org_tmin (n, 4),
    dir_tmax (n, 4), generator state after the camera's draws (n,) uint64, hero wavelength (n,))"""
    cam = scene.camera_struct(width, height)
    px = np.ascontiguousarray(pixels, np.uint32)
    n = px.shape[0]
    org = np.zeros((n, 4), np.float32)
    dirs = np.zeros((n, 4), np.float32)
    rng = np.zeros(n, np.uint64)
    lam = np.zeros(n, np.float32)
    lib().orc_camera_rays(C.byref(cam), px.ctypes.data_as(C.POINTER(C.c_uint32)), n, sample, _fp(org), _fp(dirs),
                          rng.ctypes.data_as(C.POINTER(C.c_uint64)), _fp(lam))
    return org, dirs, rng, lam


def li(scene, tables: Tables, params, org, dirs, rng_state, lambda0):
    """PathIntegrator::Li of the oracle for n given rays: (radiance (n, NL), generator
    state after each path (n,), XYZ (n, 3))"""
    desc, keep = scene.desc()
    n = org.shape[0]
    nl = 60 if params.spectral_mode == T.FL_SPECTRAL_BINS60 else 4
    org = np.ascontiguousarray(org, np.float32)
    dirs = np.ascontiguousarray(dirs, np.float32)
    rng = np.ascontiguousarray(rng_state, np.uint64)
    lam = np.ascontiguousarray(lambda0, np.float32)
    L = np.zeros((n, nl), np.float32)
    rng_out = np.zeros(n, np.uint64)
    xyz = np.zeros((n, 3), np.float64)
    rc = lib().orc_li(C.byref(desc), tables.buf, C.byref(params), n, _fp(org), _fp(dirs),
                      rng.ctypes.data_as(C.POINTER(C.c_uint64)), _fp(lam), _fp(L),
                      rng_out.ctypes.data_as(C.POINTER(C.c_uint64)), xyz.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 0, "orc_li failed"
    return L, rng_out, xyz


# ----------------------------------------------------------------------------- reference binary

SCENE_MAGIC = b"FLSCENE2"


def write_scene_file(path, scene, params, nthreads=0, pixels=None, width=None, height=None):
    """scene file read by oracle/_ref/ref_render (layout: ref_harness.cpp SceneFileHeader)."""
    cam = scene.camera_struct(width, height)
    px = np.ascontiguousarray(pixels if pixels is not None else np.zeros(0), np.uint32)
    hdr = bytearray(SCENE_MAGIC)
    if params.flags & T.FL_RENDER_LOBE_DEPTHS:
        depths = [params.diffuse_depth, params.reflection_depth, params.transmission_depth]
    else:
        depths = [params.max_depth] * 3
    hdr += np.array([scene.n_tri, len(scene.materials), len(scene.lights), params.spp, params.max_depth,
                     params.spectral_mode, params.sample_offset, nthreads, px.shape[0]] + depths,
                    np.uint32).tobytes()
    hdr += np.array([params.rr_threshold], np.float32).tobytes()
    hdr += bytes(cam)
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(np.ascontiguousarray(scene.verts, np.float32).tobytes())
        f.write(np.ascontiguousarray(scene.tri_material, np.uint32).tobytes())
        f.write(bytes(scene.materials_array())[: C.sizeof(T.fl_material) * len(scene.materials)])
        f.write(bytes(scene.lights_array())[: C.sizeof(T.fl_light) * len(scene.lights)])
        f.write(px.tobytes())
        stds, n_std = scene.standard_array()
        f.write(np.uint32(n_std).tobytes())
        f.write(bytes(stds)[: C.sizeof(T.fl_standard_surface) * n_std])
        # texture coordinates and images
        f.write(np.uint32(0 if scene.uvs is None else 1).tobytes())
        if scene.uvs is not None:
            f.write(np.ascontiguousarray(scene.uvs, np.float32).reshape(scene.n_tri, 6).tobytes())
        f.write(np.uint32(len(scene.images)).tobytes())
        for im in scene.images:
            im = np.ascontiguousarray(im, np.uint8)
            f.write(np.array([im.shape[1], im.shape[0]], np.int32).tobytes())
            f.write(im.tobytes())


def run_reference(scene_path, out_path, W, H, forge=False):
    """runs the compiled reference integrator; returns (film (H, W, 3) float64, info dict).
    forge: call InitializeForge first (the reference itself never does)."""
    import json
    r = subprocess.run([REF_BIN, scene_path, out_path] + (["--forge"] if forge else []), check=True,
                       capture_output=True, text=True)
    info = json.loads(r.stdout.strip().splitlines()[-1])
    film = np.fromfile(out_path, dtype=np.float64).reshape(H, W, 3)
    return film, info


def load_metals_dump(path):
    """parses `ref_render --metals` output: per metal m (GetMetalCoefficientsFromForge order)
    lambda_m, eta_m, k_m (the raw curves) and the binned eta60 / k60 (9 x 60)."""
    raw = np.fromfile(path, dtype=np.uint8)
    n = np.frombuffer(raw[:36], np.int32).copy()
    f = np.frombuffer(raw[36:], np.float32)
    out, o = {"n": n}, 0
    for m in range(9):
        for key in ("lambda", "eta", "k"):
            out[f"{key}_{m}"] = f[o:o + n[m]].copy()
            o += n[m]
    binned = f[o:o + 1080].reshape(9, 2, 60)  # per metal: eta, then k
    out["eta60"] = binned[:, 0].copy()
    out["k60"] = binned[:, 1].copy()
    return out


def load_tables_dump(path):
    """parses `ref_render --tables` output into a tables dict (+ binned and KAT arrays)."""
    raw = np.fromfile(path, dtype=np.uint8)
    n_cie, n_rgb = np.frombuffer(raw[:8], np.int32)
    f = np.frombuffer(raw[8:], np.float32)
    o = 0

    def take(k):
        nonlocal o
        a = f[o:o + k].copy()
        o += k
        return a

    t = {"cie_y_integral": np.float32(take(1)[0])}
    t["cie_lambda"] = take(n_cie)
    t["cie_x"] = take(n_cie)
    t["cie_y"] = take(n_cie)
    t["cie_z"] = take(n_cie)
    t["rgb_lambda"] = take(n_rgb)
    t["refl"] = take(7 * n_rgb).reshape(7, n_rgb)
    t["illum"] = take(7 * n_rgb).reshape(7, n_rgb)
    t["binned60"] = take(17 * 60).reshape(17, 60)
    t["refl60_kat"] = take(4 * 60).reshape(4, 60)
    t["xyz_of_one"] = take(3)
    return t


# ----------------------------------------------------------------------------- guiding

def guide_eval(weights, records, bmin, bmax):
    """mixture parameters (n, 41) of the guide network for the records' points: pi[8], mu[8][3],
    kappa[8], the selection probability c"""
    w = np.ascontiguousarray(weights, dtype=np.float32)
    r = np.ascontiguousarray(records, dtype=np.float32)
    out = np.zeros((r.shape[0], 41), np.float32)
    lib().orc_guide_eval(_fp(w), _fp(r), r.shape[0], _fp(np.asarray(bmin, np.float32)),
                         _fp(np.asarray(bmax, np.float32)), _fp(out))
    return out


def guide_set_exact(on: bool):
    """evaluate the guide without FP16 roundings (finite-difference checks)"""
    lib().orc_guide_set_exact(1 if on else 0)


def guide_gradient(weights, records, bmin, bmax, learned=False):
    """(gradient, mean loss) of the weighted training loss (learned: the one-sample MIS
    mixture loss that also fits the selection probability)"""
    w = np.ascontiguousarray(weights, dtype=np.float32)
    r = np.ascontiguousarray(records, dtype=np.float32)
    g = np.zeros(w.shape[0], np.float32)
    loss = lib().orc_guide_gradient(_fp(w), _fp(r), r.shape[0], _fp(np.asarray(bmin, np.float32)),
                                    _fp(np.asarray(bmax, np.float32)), _fp(g), 1 if learned else 0)
    return g, float(loss)


def bsdf_fcos(material, wo, wi, corrected=False):
    """f(wo, wi) |cos theta_i| of a non-Lambert fl_material in its local frame (normal +z)"""
    w = np.ascontiguousarray(wi, np.float32)
    o = np.ascontiguousarray(wo, np.float32)
    out = np.zeros(w.shape[0], np.float32)
    lib().orc_bsdf_fcos(C.byref(material), _fp(o), w.shape[0], _fp(w), 1 if corrected else 0, _fp(out))
    return out



def image_texels(image, uv):
    """the oracle's ImageMapTexture texel (RGB / 255) at each (u, v) row of uv"""
    im = np.ascontiguousarray(image, np.uint8)
    uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    rec = T.fl_image(im.shape[1], im.shape[0], im.ctypes.data_as(C.POINTER(C.c_uint8)))
    out = np.zeros((uv.shape[0], 3), np.float32)
    lib().orc_image_texels(C.byref(rec), _fp(uv), uv.shape[0], _fp(out))
    return out
