"""The C++ host adapter (include/filianore_gpu.hpp), which mirrors the reference's
SceneGeometry / BVH / Scene / PathIntegrator: it compiles and links against the library
(CPU), and on the GPU its render and its per-ray and batch intersections equal the C ABI's
(fl_render, fl_trace_closest) on the Cornell box, with RenderParams' three depths unequal;
and PathIntegrator::Li on its camera rays (PhysicalCamera::awaken_ray, a PCG32Sampler seeded
per pixel) equals the per-pixel film of a 1-spp render."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import filianore_b200 as fb
from filianore_b200 import scenes

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "cpp", "adapter_cornell.cpp")


def build(tmp):
    exe = os.path.join(tmp, "adapter_cornell")
    libdir = os.path.dirname(fb.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-o", exe, SRC, "-I", os.path.join(ROOT, "include"),
                    "-L", libdir, "-lfilianore_b200", f"-Wl,-rpath,{libdir}"], check=True)
    return exe


def test_adapter_compiles_and_links(tmp_path):
    exe = build(str(tmp_path))
    assert os.path.exists(exe)


def write_input(path, sc, params, org, dirs):
    t = fb.reference_tables()
    desc, keep = sc.desc()
    with open(path, "wb") as f:
        f.write(np.int32(t["cie_lambda"].shape[0]).tobytes())
        f.write(np.float32(t["cie_y_integral"]).tobytes())
        for k in ("cie_lambda", "cie_x", "cie_y", "cie_z"):
            f.write(np.ascontiguousarray(t[k], np.float32).tobytes())
        f.write(np.int32(t["rgb_lambda"].shape[0]).tobytes())
        f.write(np.ascontiguousarray(t["rgb_lambda"], np.float32).tobytes())
        f.write(np.ascontiguousarray(t["refl"], np.float32).tobytes())
        f.write(np.ascontiguousarray(t["illum"], np.float32).tobytes())
        f.write(np.uint32(sc.n_tri).tobytes())
        f.write(np.ascontiguousarray(sc.verts, np.float32).tobytes())
        f.write(np.ascontiguousarray(sc.tri_material, np.uint32).tobytes())
        mats, lights = sc.materials_array(), sc.lights_array()
        f.write(np.uint32(len(sc.materials)).tobytes())
        f.write(bytes(mats)[: len(sc.materials) * C.sizeof(fb.fl_material)])
        f.write(np.uint32(len(sc.lights)).tobytes())
        f.write(bytes(lights)[: len(sc.lights) * C.sizeof(fb.fl_light)])
        f.write(bytes(sc.camera_struct()))
        if params.flags & fb.FL_RENDER_LOBE_DEPTHS:
            depths = [params.diffuse_depth, params.reflection_depth, params.transmission_depth]
        else:
            depths = [params.max_depth] * 3
        f.write(np.array([params.spp] + depths + [params.spectral_mode], np.int32).tobytes())
        f.write(np.uint32(org.shape[0]).tobytes())
        f.write(np.ascontiguousarray(org, np.float32).tobytes())
        f.write(np.ascontiguousarray(dirs, np.float32).tobytes())
        stds, n_std = sc.standard_array()
        f.write(np.uint32(n_std).tobytes())
        f.write(bytes(stds)[: n_std * C.sizeof(fb.fl_standard_surface)])
        uvs = np.zeros((sc.n_tri, 6), np.float32) if sc.uvs is None else sc.uvs
        f.write(np.ascontiguousarray(uvs, np.float32).tobytes())
        f.write(np.uint32(len(sc.images)).tobytes())
        for im in sc.images:
            im = np.ascontiguousarray(im, np.uint8)
            f.write(np.array([im.shape[1], im.shape[0]], np.int32).tobytes())
            f.write(im.tobytes())


@pytest.mark.gpu
def test_adapter_matches_c_abi(tmp_path):
    exe = build(str(tmp_path))
    # area, point, spot and directional lights; image textures, a bump-mapped StandardSurface
    tex = scenes.cornell_textured(48, 48, bump=True)
    sc = scenes.Scene(tex.verts, tex.tri_material, tex.materials, list(tex.lights) + scenes.delta_lights(),
                      tex.camera, uvs=tex.uvs, images=tex.images)
    # RenderParams with a different depth per lobe kind
    params = scenes.render_params(4, 8, fb.FL_SPECTRAL_BINS60, depths=(3, 6, 5))
    rng = np.random.default_rng(3)
    n = 4096
    org = np.zeros((n, 4), np.float32)
    org[:, :3] = rng.uniform(0.05, 0.95, (n, 3))
    d = rng.normal(size=(n, 3))
    dirs = np.zeros((n, 4), np.float32)
    dirs[:, :3] = d / np.linalg.norm(d, axis=1, keepdims=True)
    dirs[:, 3] = np.where(rng.random(n) < 0.5, np.inf, 0.3)   # half the rays end at t = 0.3 (some miss)
    inp, out = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    write_input(inp, sc, params, org, dirs)
    subprocess.run([exe, inp, out], check=True)
    raw = np.fromfile(out, np.uint8)
    f32 = raw[: (48 * 48 * 3 + n * 6) * 4].view(np.float32)
    rgb_cpp = f32[: 48 * 48 * 3].reshape(48, 48, 3)
    rec = f32[48 * 48 * 3:].reshape(n, 6)
    tail = raw[(48 * 48 * 3 + n * 6) * 4:]
    li_xyz = tail[: 48 * 48 * 24].view(np.float64).reshape(48, 48, 3)
    singles = tail[48 * 48 * 24:].reshape(16, 40)
    one_xyz = singles[:, :24].copy().view(np.float64).reshape(16, 3)
    one_rec = singles[:, 24:].copy().view(np.uint64).reshape(16, 2)
    ctx = fb.Context(0)
    s = ctx.scene(sc)
    rgb, _ = s.render(params)
    hits = s.trace_closest(org, dirs)
    # the 1-spp film of the same depths: what Li's camera rays must add up to
    film1 = np.zeros((48, 48, 3), np.float64)
    p1 = scenes.render_params(1, 8, fb.FL_SPECTRAL_BINS60, depths=(3, 6, 5))
    s.render(p1, film_xyz64=film1)
    # the sampler after a single-ray Li equals the generator state fl_li returns for the same
    # camera rays (made here by the oracle's restatement of the render loop's camera)
    import oracle
    o, d, r0, _ = oracle.camera_rays(sc, np.arange(16))
    _, rng_after, _ = fb.li(s, p1, o, d, r0)
    s.close()
    ctx.close()
    assert np.array_equal(rgb_cpp, rgb)
    # PathIntegrator::Li on PhysicalCamera::awaken_ray's rays equals the per-pixel film of a
    # 1-spp render (one sample per pixel, so the film's FP64 sums are the samples themselves)
    assert np.array_equal(li_xyz, film1)
    assert np.array_equal(one_xyz, li_xyz.reshape(-1, 3)[:16])
    assert np.all(one_rec[:, 1] == 1)  # single-ray spectra equal the batch's bit for bit
    assert np.array_equal(one_rec[:, 0], rng_after)
    ids = hits["id"]
    hit = ids >= 0
    assert hit.any() and (~hit).any()
    # BVH::intersect: bool, primitive, t, and ray.tMax shrunk to t on a hit
    assert np.array_equal(rec[:, 0].astype(bool), hit)
    assert np.array_equal(rec[hit, 1].astype(np.int64), ids[hit])
    assert np.array_equal(rec[hit, 2], hits["t"][hit])
    assert np.array_equal(rec[hit, 3], hits["t"][hit])
    assert np.array_equal(rec[~hit, 3], dirs[~hit, 3])
    # BVH::trace (batch)
    assert np.array_equal(rec[:, 4].astype(np.int64), ids)
    assert np.array_equal(rec[hit, 5], hits["t"][hit])
