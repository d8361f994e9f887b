"""Python binding of the filianore B200 backend (ctypes over lib/libfilianore_b200.so).

The library is the product: a C ABI (include/filianore_gpu.h) over hand-written sm_100a
kernels. This module only marshals arguments; it has no compute path of its own, and it
raises if the shared library is missing or fails to load.
"""
from __future__ import annotations

import atexit
import ctypes as C
import os
import weakref

import numpy as np

from . import types as T
from .types import *  # noqa: F401,F403

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("FILIANORE_B200_LIB", os.path.join(PKG_DIR, "lib", "libfilianore_b200.so"))
ROOT = os.path.dirname(PKG_DIR)
TABLES_PATH = os.path.join(ROOT, "tests", "golden", "spectral_tables.npz")
METALS_PATH = os.path.join(ROOT, "tests", "golden", "metal_tables.npz")

EXPORTED = [
    "fl_context_create", "fl_context_destroy", "fl_status_string", "fl_last_error", "fl_context_binned_tables",
    "fl_scene_create", "fl_scene_destroy", "fl_scene_get_info", "fl_trace_closest", "fl_trace_occluded",
    "fl_trace_count", "fl_render", "fl_li", "fl_render_noalloc", "fl_server_create", "fl_server_destroy",
    "fl_server_add_scene", "fl_server_remove_scene", "fl_server_submit", "fl_server_poll", "fl_server_wait", "fl_server_get_stats",
    "fl_guide_create", "fl_guide_destroy", "fl_guide_render", "fl_guide_render_timed", "fl_guide_get_weights",
    "fl_guide_set_weights", "fl_guide_get_info", "fl_guide_gradient", "fl_guide_eval", "fl_guide_get_records",
]

_lib = None


class FlError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{msg} ({status})")
        self.status = status


def build() -> None:
    import subprocess
    subprocess.run(["make", "-s", "-C", PKG_DIR], check=True)


def lib():
    """Loads the shared library (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FlError(-8, f"{LIB_PATH} is not built; run `make -C {PKG_DIR}`")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        vp = C.c_void_p
        L.fl_status_string.restype = C.c_char_p
        L.fl_status_string.argtypes = [C.c_int32]
        L.fl_last_error.argtypes = [vp, C.c_char_p, C.c_size_t]
        L.fl_context_create.argtypes = [C.c_int32, P(T.fl_spectral_tables), P(vp)]
        L.fl_context_destroy.argtypes = [vp]
        L.fl_context_binned_tables.argtypes = [vp, P(C.c_float), C.c_size_t]
        L.fl_scene_create.argtypes = [vp, P(T.fl_scene_desc), P(vp)]
        L.fl_scene_destroy.argtypes = [vp]
        L.fl_scene_get_info.argtypes = [vp, P(T.fl_scene_info)]
        L.fl_trace_closest.argtypes = [vp, vp, vp, C.c_uint32, vp, C.c_int32, vp]
        L.fl_trace_occluded.argtypes = [vp, vp, vp, C.c_uint32, vp, C.c_int32, vp]
        L.fl_trace_count.argtypes = [vp, vp, vp, C.c_uint32, C.c_int32, P(C.c_uint64), P(C.c_uint64)]
        L.fl_render.argtypes = [vp, P(T.fl_camera), P(T.fl_render_params), vp, vp, C.c_int32, P(T.fl_render_stats)]
        L.fl_render_noalloc.argtypes = [vp, P(T.fl_camera), P(T.fl_render_params), vp, vp, P(T.fl_render_stats)]
        L.fl_li.argtypes = [vp, P(T.fl_render_params), vp, vp, vp, vp, C.c_uint32, vp, vp, vp, C.c_int32]
        L.fl_server_create.argtypes = [vp, P(T.fl_server_config), P(vp)]
        L.fl_server_destroy.argtypes = [vp]
        L.fl_server_add_scene.argtypes = [vp, P(T.fl_scene_desc), P(C.c_uint64)]
        L.fl_server_remove_scene.argtypes = [vp, C.c_uint64]
        L.fl_server_submit.argtypes = [vp, P(T.fl_job_desc), P(C.c_uint64)]
        L.fl_server_poll.argtypes = [vp, C.c_uint64, vp, vp, P(T.fl_job_stats)]
        L.fl_server_wait.argtypes = [vp, C.c_uint64, C.c_int32, vp, vp, P(T.fl_job_stats)]
        L.fl_server_get_stats.argtypes = [vp, P(T.fl_server_stats)]
        L.fl_guide_create.argtypes = [vp, P(T.fl_guide_config), P(vp)]
        L.fl_guide_destroy.argtypes = [vp]
        L.fl_guide_render.argtypes = [vp, vp, P(T.fl_camera), P(T.fl_render_params), C.c_int32, vp, vp, C.c_int32,
                                      P(T.fl_render_stats)]
        L.fl_guide_render_timed.argtypes = [vp, vp, P(T.fl_camera), P(T.fl_render_params), C.c_double, C.c_double,
                                            vp, vp, C.c_int32, P(T.fl_render_stats)]
        L.fl_guide_get_weights.argtypes = [vp, P(C.c_float)]
        L.fl_guide_set_weights.argtypes = [vp, P(C.c_float)]
        L.fl_guide_get_info.argtypes = [vp, P(C.c_int64), P(C.c_float)]
        L.fl_guide_gradient.argtypes = [vp, P(C.c_float), C.c_uint32, P(C.c_float), P(C.c_float), P(C.c_float),
                                        P(C.c_float)]
        L.fl_guide_eval.argtypes = [vp, P(C.c_float), C.c_uint32, P(C.c_float), P(C.c_float), P(C.c_float)]
        L.fl_guide_get_records.argtypes = [vp, P(C.c_float), C.c_uint32, P(C.c_uint32)]
        for name in EXPORTED:
            if name not in ("fl_status_string",):
                getattr(L, name).restype = C.c_int32
        _lib = L
    return _lib


def check(status, ctx=None):
    if status != 0:
        buf = C.create_string_buffer(1024)
        lib().fl_last_error(ctx, buf, 1024)
        raise FlError(status, f"{lib().fl_status_string(status).decode()}: {buf.value.decode()}")


def reference_tables(path: str = TABLES_PATH, measured_metals: bool = False) -> dict:
    """The reference's spectral data (color/cie.h) as stored by tests/golden/make_golden.py.
    measured_metals adds the metal eta / k curves of color/metallurgy.h ("metal_lambda_m",
    "metal_eta_m", "metal_k_m" for the nine metals). Without them the measured-metal Fresnel
    sees eta = k = 0, as the reference does (it never calls InitializeForge)."""
    t = dict(np.load(path))
    if measured_metals:
        m = np.load(METALS_PATH)
        for i in range(9):
            for key in ("lambda", "eta", "k"):
                t[f"metal_{key}_{i}"] = m[f"{key}_{i}"]
    return t


def _tables_struct(t: dict):
    keep = {k: np.ascontiguousarray(t[k], np.float32) for k in ("cie_lambda", "cie_x", "cie_y", "cie_z", "rgb_lambda")}
    refl = [np.ascontiguousarray(r, np.float32) for r in t["refl"]]
    illum = [np.ascontiguousarray(r, np.float32) for r in t["illum"]]
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    s = T.fl_spectral_tables()
    s.cie_lambda, s.cie_x, s.cie_y, s.cie_z = (fp(keep[k]) for k in ("cie_lambda", "cie_x", "cie_y", "cie_z"))
    s.n_cie = keep["cie_lambda"].shape[0]
    s.cie_y_integral = float(t["cie_y_integral"])
    s.rgb2spec_lambda = fp(keep["rgb_lambda"])
    s.n_rgb2spec = keep["rgb_lambda"].shape[0]
    for b in range(7):
        s.refl[b] = fp(refl[b])
        s.illum[b] = fp(illum[b])
    metals = T.set_metal_tables(s, t, fp)
    return s, (keep, refl, illum, metals)


# Handles still open at interpreter exit are closed children first (guides and servers,
# then scenes, then contexts) while the CUDA runtime is still up.
_open = (weakref.WeakSet(), weakref.WeakSet(), weakref.WeakSet())


@atexit.register
def _close_all():
    for group in _open:
        for obj in list(group):
            try:
                obj.close()
            except Exception:
                pass


def _ptr(x):
    """device pointer of a torch tensor, or host pointer of a numpy array"""
    if hasattr(x, "data_ptr"):
        return C.c_void_p(x.data_ptr())
    return C.c_void_p(x.ctypes.data)


def _is_device(x):
    return hasattr(x, "is_cuda") and x.is_cuda


class Context:
    def __init__(self, device: int = 0, tables: dict | None = None):
        self.h = None
        s, self._keep = _tables_struct(tables if tables is not None else reference_tables())
        h = C.c_void_p()
        check(lib().fl_context_create(device, C.byref(s), C.byref(h)))
        self.h = h
        self.children = weakref.WeakSet()  # scenes, guides and servers made from this context
        _open[2].add(self)

    def close(self):
        """closes the context's scenes, guides and servers first, then the context"""
        if self.h:
            for c in list(self.children):
                c.close()
            lib().fl_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def binned_tables(self):
        out = np.zeros(17 * 60, np.float32)
        check(lib().fl_context_binned_tables(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size), self.h)
        return out.reshape(17, 60)

    def binned_metals(self):
        """the measured metals' 60-bin eta and k: (9, 2, 60)"""
        out = np.zeros(17 * 60 + 9 * 120, np.float32)
        check(lib().fl_context_binned_tables(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size), self.h)
        return out[17 * 60:].reshape(9, 2, 60)

    def scene(self, scene_obj):
        return SceneHandle(self, scene_obj)


class SceneHandle:
    def __init__(self, ctx: Context, sc):
        self.ctx = ctx
        self.h = None
        self.src = sc
        desc, keep = sc.desc()
        h = C.c_void_p()
        check(lib().fl_scene_create(ctx.h, C.byref(desc), C.byref(h)), ctx.h)
        self.h = h
        _open[1].add(self)
        ctx.children.add(self)

    def close(self):
        if self.h:
            lib().fl_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        i = T.fl_scene_info()
        check(lib().fl_scene_get_info(self.h, C.byref(i)), self.ctx.h)
        return {k: getattr(i, k) for k, _ in T.fl_scene_info._fields_}

    # ------------------------------------------------------------------ queries
    def trace_closest(self, org, dirs, out=None, stream=None):
        """org, dirs: (n, 4) float32 numpy (host) or torch CUDA tensors (device).
        Returns a structured numpy array (host) or fills/returns an (n, 4) int32 torch tensor."""
        n = org.shape[0]
        if _is_device(org):
            import torch
            if out is None:
                out = torch.empty((n, 4), dtype=torch.int32, device=org.device)
            check(lib().fl_trace_closest(self.h, _ptr(org), _ptr(dirs), n, _ptr(out), T.FL_MEM_DEVICE,
                                         C.c_void_p(stream)), self.ctx.h)
            return out
        org = np.ascontiguousarray(org, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        hits = out if out is not None else np.zeros(n, dtype=T.HIT_DTYPE)
        check(lib().fl_trace_closest(self.h, _ptr(org), _ptr(dirs), n, _ptr(hits), T.FL_MEM_HOST, None), self.ctx.h)
        return hits

    def trace_occluded(self, org, dirs):
        n = org.shape[0]
        if _is_device(org):
            import torch
            out = torch.empty(n, dtype=torch.uint8, device=org.device)
            check(lib().fl_trace_occluded(self.h, _ptr(org), _ptr(dirs), n, _ptr(out), T.FL_MEM_DEVICE, None),
                  self.ctx.h)
            return out
        org = np.ascontiguousarray(org, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        occ = np.zeros(n, np.uint8)
        check(lib().fl_trace_occluded(self.h, _ptr(org), _ptr(dirs), n, _ptr(occ), T.FL_MEM_HOST, None), self.ctx.h)
        return occ

    def trace_count(self, org, dirs):
        n = org.shape[0]
        mem = T.FL_MEM_DEVICE if _is_device(org) else T.FL_MEM_HOST
        if mem == T.FL_MEM_HOST:
            org = np.ascontiguousarray(org, np.float32)
            dirs = np.ascontiguousarray(dirs, np.float32)
        nv, nt = C.c_uint64(0), C.c_uint64(0)
        check(lib().fl_trace_count(self.h, _ptr(org), _ptr(dirs), n, mem, C.byref(nv), C.byref(nt)), self.ctx.h)
        return nv.value, nt.value

    def render(self, params, camera=None, film_rgb=None, film_xyz64=None, memory=None):
        """Renders self.src's camera (or `camera`, an fl_camera). Host numpy films by default."""
        cam = camera if camera is not None else self.src.camera_struct()
        W, H = cam.width, cam.height
        if film_rgb is None:
            film_rgb = np.zeros((H, W, 3), np.float32)
        mem = memory if memory is not None else (T.FL_MEM_DEVICE if _is_device(film_rgb) else T.FL_MEM_HOST)
        stats = T.fl_render_stats()
        xyz = _ptr(film_xyz64) if film_xyz64 is not None else None
        check(lib().fl_render(self.h, C.byref(cam), C.byref(params), _ptr(film_rgb), xyz, mem, C.byref(stats)),
              self.ctx.h)
        return film_rgb, {k: getattr(stats, k) for k, _ in T.fl_render_stats._fields_}


def li(scene: "SceneHandle", params, org, dirs, rng_state, lambda0=None):
    """Integrator::Li for a batch of host rays (fl_li): returns (radiance (n, NL) float32,
    generator states after the paths (n,) uint64, XYZ (n, 3) float64)."""
    n = org.shape[0]
    nl = 60 if params.spectral_mode == T.FL_SPECTRAL_BINS60 else 4
    org = np.ascontiguousarray(org, np.float32)
    dirs = np.ascontiguousarray(dirs, np.float32)
    rng = np.ascontiguousarray(rng_state, np.uint64)
    lam = None if lambda0 is None else np.ascontiguousarray(lambda0, np.float32)
    L = np.zeros((n, nl), np.float32)
    rng_out = np.zeros(n, np.uint64)
    xyz = np.zeros((n, 3), np.float64)
    check(lib().fl_li(scene.h, C.byref(params), _ptr(org), _ptr(dirs), _ptr(rng), _ptr(lam) if lam is not None else None,
                      n, _ptr(L), _ptr(rng_out), _ptr(xyz), T.FL_MEM_HOST), scene.ctx.h)
    return L, rng_out, xyz


class Guide:
    """Learned path guide (fl_guide_*): an MLP proposal for continuation directions at Lambert
    vertices, trained online on the renderer's own samples."""

    def __init__(self, ctx: Context, seed: int = 1, learning_rate: float = 1e-3, select_prob: float = 0.5,
                 batch: int = 32768, max_records: int = 1 << 20, steps_per_wave: int = 16,
                 position_scale: float = 1.0 / 16, weight_average: float = 0.99, learn_select: bool = False,
                 train_kernel: int = 0):
        self.ctx = ctx
        self.h = None
        cfg = T.fl_guide_config(seed, learning_rate, select_prob, batch, max_records, steps_per_wave, position_scale,
                                weight_average, int(learn_select), int(train_kernel))
        h = C.c_void_p()
        check(lib().fl_guide_create(ctx.h, C.byref(cfg), C.byref(h)), ctx.h)
        self.h = h
        _open[0].add(self)
        ctx.children.add(self)

    def close(self):
        if self.h:
            lib().fl_guide_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, scene: "SceneHandle", params, flags, camera=None, film_rgb=None, film_xyz64=None, memory=None):
        cam = camera if camera is not None else scene.src.camera_struct()
        if film_rgb is None:
            film_rgb = np.zeros((cam.height, cam.width, 3), np.float32)
        mem = memory if memory is not None else (T.FL_MEM_DEVICE if _is_device(film_rgb) else T.FL_MEM_HOST)
        st = T.fl_render_stats()
        xyz = _ptr(film_xyz64) if film_xyz64 is not None else None
        check(lib().fl_guide_render(self.h, scene.h, C.byref(cam), C.byref(params), flags, _ptr(film_rgb), xyz, mem,
                                    C.byref(st)), self.ctx.h)
        return film_rgb, {k: getattr(st, k) for k, _ in T.fl_render_stats._fields_}

    def render_timed(self, scene: "SceneHandle", params, budget_ms: float, train_fraction: float = 0.25, camera=None,
                     film_rgb=None, film_xyz64=None, memory=None):
        cam = camera if camera is not None else scene.src.camera_struct()
        if film_rgb is None:
            film_rgb = np.zeros((cam.height, cam.width, 3), np.float32)
        mem = memory if memory is not None else (T.FL_MEM_DEVICE if _is_device(film_rgb) else T.FL_MEM_HOST)
        st = T.fl_render_stats()
        xyz = _ptr(film_xyz64) if film_xyz64 is not None else None
        check(lib().fl_guide_render_timed(self.h, scene.h, C.byref(cam), C.byref(params), budget_ms, train_fraction,
                                          _ptr(film_rgb), xyz, mem, C.byref(st)), self.ctx.h)
        return film_rgb, {k: getattr(st, k) for k, _ in T.fl_render_stats._fields_}

    def weights(self):
        w = np.zeros(T.FL_GUIDE_PARAMS, np.float32)
        check(lib().fl_guide_get_weights(self.h, w.ctypes.data_as(C.POINTER(C.c_float))), self.ctx.h)
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        check(lib().fl_guide_set_weights(self.h, w.ctypes.data_as(C.POINTER(C.c_float))), self.ctx.h)

    def info(self):
        steps, loss = C.c_int64(), C.c_float()
        check(lib().fl_guide_get_info(self.h, C.byref(steps), C.byref(loss)), self.ctx.h)
        return {"adam_steps": steps.value, "last_loss": loss.value}

    def gradient(self, records, bmin, bmax):
        r = np.ascontiguousarray(records, np.float32)
        g = np.zeros(T.FL_GUIDE_PARAMS, np.float32)
        loss = C.c_float()
        bn = np.asarray(bmin, np.float32)
        bx = np.asarray(bmax, np.float32)
        check(lib().fl_guide_gradient(self.h, r.ctypes.data_as(C.POINTER(C.c_float)), r.shape[0],
                                      bn.ctypes.data_as(C.POINTER(C.c_float)), bx.ctypes.data_as(C.POINTER(C.c_float)),
                                      g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)), self.ctx.h)
        return g, loss.value

    def records(self, max_n: int = 1 << 20):
        """training records of the last trained wave, (n, 20)"""
        out = np.zeros((max_n, T.FL_GUIDE_RECORD_FLOATS), np.float32)
        n = C.c_uint32()
        check(lib().fl_guide_get_records(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), max_n, C.byref(n)),
              self.ctx.h)
        return out[:n.value]

    def eval(self, records, bmin, bmax):
        r = np.ascontiguousarray(records, np.float32)
        out = np.zeros((r.shape[0], 41), np.float32)  # pi[8], mu[8][3], kappa[8], c
        bn = np.asarray(bmin, np.float32)
        bx = np.asarray(bmax, np.float32)
        check(lib().fl_guide_eval(self.h, r.ctypes.data_as(C.POINTER(C.c_float)), r.shape[0],
                                  bn.ctypes.data_as(C.POINTER(C.c_float)), bx.ctypes.data_as(C.POINTER(C.c_float)),
                                  out.ctypes.data_as(C.POINTER(C.c_float))), self.ctx.h)
        return out


class Server:
    """Continuous-batching render server (fl_server_*): scenes stay resident under a memory
    budget, running jobs share every wave."""

    def __init__(self, ctx: Context, budget_bytes: int, max_depth: int = 16, max_jobs: int = 32, max_lights: int = 8,
                 wave_paths: int = 0, policy: int = 0):
        self.ctx = ctx
        self.h = None
        cfg = T.fl_server_config(budget_bytes, wave_paths, max_depth, max_jobs, max_lights, policy)
        h = C.c_void_p()
        check(lib().fl_server_create(ctx.h, C.byref(cfg), C.byref(h)), ctx.h)
        self.h = h
        _open[0].add(self)
        ctx.children.add(self)
        self.shapes = {}

    def close(self):
        if self.h:
            lib().fl_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, sc) -> int:
        desc, keep = sc.desc()
        sid = C.c_uint64()
        check(lib().fl_server_add_scene(self.h, C.byref(desc), C.byref(sid)), self.ctx.h)
        return sid.value

    def remove_scene(self, scene_id: int) -> None:
        """no more jobs for the scene; its memory is released once no submitted job uses it"""
        check(lib().fl_server_remove_scene(self.h, scene_id), self.ctx.h)

    def submit(self, scene_id: int, camera, params) -> int:
        job = T.fl_job_desc(scene_id, camera, params)
        jid = C.c_uint64()
        check(lib().fl_server_submit(self.h, C.byref(job), C.byref(jid)), self.ctx.h)
        self.shapes[jid.value] = (camera.height, camera.width)
        return jid.value

    def wait(self, job_id: int, timeout_ms: int = -1, want_xyz: bool = False):
        H, W = self.shapes.pop(job_id)
        rgb = np.zeros((H, W, 3), np.float32)
        xyz = np.zeros((H, W, 3), np.float64) if want_xyz else None
        st = T.fl_job_stats()
        rc = lib().fl_server_wait(self.h, job_id, timeout_ms, _ptr(rgb), _ptr(xyz) if xyz is not None else None,
                                  C.byref(st))
        if rc != 0:
            self.shapes[job_id] = (H, W)
        check(rc, self.ctx.h)
        return rgb, xyz, {k: getattr(st, k) for k, _ in T.fl_job_stats._fields_}

    def stats(self):
        st = T.fl_server_stats()
        lib().fl_server_get_stats(self.h, C.byref(st))
        return {k: getattr(st, k) for k, _ in T.fl_server_stats._fields_}


from . import scenes  # noqa: E402,F401  (scene generators: fb.scenes.cornell, ...)
