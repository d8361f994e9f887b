"""Generates the committed fixtures under tests/golden/ from the reference itself.

Runs only where the reference tree is present (it builds oracle/_ref/ref_render from the
reference sources with oracle/Makefile). Outputs:
  spectral_tables.npz   the reference's spectral data (color/cie.h: CIE 1931 observer,
                        RGB->spectrum bases) as the reference binary reads them, plus the
                        60-bin tables InitializeSpectrals builds and from_reflectance_rgb /
                        to_xyz known answers
  pcg32_kat.npz         pcg32 sequences from the vendored src/ext/pcg32.h
  cornell_ref.npz       the reference integrator's XYZ film sums for the 36-triangle Cornell
                        box: 64x64 at 4 spp (float64) and 256x256 at 16 spp (float32)
  cornell_materials_ref.npz  the same with GGX conductor + rough dielectric boxes
                        ("materials") and conductor + smooth glass boxes ("glass"):
                        64x64 at 4 spp (float64) and 128x128 at 16 spp (float32)
  cornell_depths_ref.npz  RenderParams with unequal depths per lobe kind: the "materials"
                        box at (diffuse, reflection, transmission) = (3, 6, 5) and the "glass"
                        box at (5, 3, 6), 64x64 at 4 spp (float64)
  cornell_delta_ref.npz the Cornell box ("lambert" and "materials") with the reference's
                        point, spot and directional lights added: 64x64 at 4 spp (float64)
  cornell_standard_ref.npz  the Cornell box with StandardSurfaceMaterial boxes ("standard":
                        Oren-Nayar + sheen, Fresnel-blended anisotropic GGX + clear coat;
                        "standard2": Schlick-metallic blend, specular R/T glass + sheen;
                        "standard3": thin-walled diffuse transmission + sheen, measured copper
                        with Oren-Nayar diffuse + thin film + clear coat), 64x64 at 4 spp
                        (float64); "standard3" twice: as the reference renders it (no
                        InitializeForge: zero metal spectra) and after InitializeForge
  metal_tables.npz      the measured metal curves of color/metallurgy.h (wavelengths, eta, k
                        per metal) and the 60-bin spectra InitializeForge makes of them
  cornell_textured_ref.npz  the Cornell box with ImageMapTexture materials (Lambert and a
                        StandardSurface kd) at 64x64 x 4 spp (float64): with texture
                        coordinates ("uv") and without (every hit at uv (0, 0), as the
                        reference's BVH::intersect leaves it: "nouv"); the same with bump
                        maps ("bump", "bump_nouv")
Usage: python tests/golden/make_golden.py [part ...]   (parts: tables pcg cornell materials
       depths delta metals standard textures; default all)
Scratch files go to oracle/_ref/tmp.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "filianore-core_b200"))

import oracle  # noqa: E402
from filianore_b200 import scenes, types as T  # noqa: E402


def tables(tmp):
    import subprocess
    tpath = os.path.join(tmp, "tables.bin")
    subprocess.run([oracle.REF_BIN, "--tables", tpath], check=True)
    t = oracle.load_tables_dump(tpath)
    np.savez_compressed(os.path.join(HERE, "spectral_tables.npz"), **t)


def pcg(tmp):
    import subprocess
    ppath = os.path.join(tmp, "pcg.bin")
    subprocess.run([oracle.REF_BIN, "--pcg", ppath], check=True)
    raw = np.fromfile(ppath, np.uint8)
    seq = np.frombuffer(raw[: 5 * 16 * 4], np.uint32).reshape(5, 16)
    adv = np.frombuffer(raw[5 * 16 * 4: 5 * 16 * 4 + 3 * 8 * 4], np.uint32).reshape(3, 8)
    flt = np.frombuffer(raw[5 * 16 * 4 + 3 * 8 * 4:], np.float32)
    np.savez_compressed(os.path.join(HERE, "pcg32_kat.npz"),
                        seeds=np.array([[0, 1], [1, 1], [12345, 1], [42, 54], [65535, 1]], np.uint64),
                        seq=seq, adv_deltas=np.array([1, 1 << 16, 5 << 16], np.int64), adv=adv,
                        float_seed=np.array([3, 1], np.uint64), floats=flt)


def cornell(tmp):
    """Cornell box renders by the reference integrator"""
    out = {}
    for (W, H, spp, key, dt) in [(64, 64, 4, "small", np.float64), (256, 256, 16, "full", np.float32)]:
        sc = scenes.cornell(W, H)
        p = scenes.render_params(spp, 8, T.FL_SPECTRAL_BINS60)
        spath = os.path.join(tmp, f"cornell_{key}.scene")
        fpath = os.path.join(tmp, f"cornell_{key}.film")
        oracle.write_scene_file(spath, sc, p)
        film, info = oracle.run_reference(spath, fpath, W, H)
        out[f"{key}_xyz"] = film.astype(dt)
        out[f"{key}_spp"] = np.int32(spp)
        print(key, info)
    np.savez_compressed(os.path.join(HERE, "cornell_ref.npz"), **out)


def materials(tmp):
    """the same box with the GGX conductor / rough dielectric / smooth glass materials"""
    out = {}
    for variant in ("materials", "glass"):
        for (W, spp, key, dt) in [(64, 4, "small", np.float64), (128, 16, "full", np.float32)]:
            sc = scenes.cornell(W, W, variant)
            p = scenes.render_params(spp, 8, T.FL_SPECTRAL_BINS60)
            spath = os.path.join(tmp, f"{variant}_{key}.scene")
            fpath = os.path.join(tmp, f"{variant}_{key}.film")
            oracle.write_scene_file(spath, sc, p)
            film, info = oracle.run_reference(spath, fpath, W, W)
            out[f"{variant}_{key}_xyz"] = film.astype(dt)
            print(variant, key, info)
    np.savez_compressed(os.path.join(HERE, "cornell_materials_ref.npz"), **out)


def depths(tmp):
    """RenderParams with three different depths (diffuse, reflection, transmission): the
    materials box at (3, 6, 5), the glass box at (5, 3, 6), and the StandardSurface boxes
    "standard2" at (5, 3, 6) and "standard3" at (3, 6, 5), 64x64 at 4 spp. (The materials
    box's GGX lobes are seen from below their normals, where the reference's sampler fails,
    so there only the diffuse depth matters; the glass and StandardSurface boxes exercise the
    specular, glossy and transmission depths.)"""
    out = {}
    for variant, ds in (("materials", (3, 6, 5)), ("glass", (5, 3, 6)), ("standard2", (5, 3, 6)),
                        ("standard3", (3, 6, 5))):
        sc = scenes.cornell(64, 64, variant)
        p = scenes.render_params(4, 8, T.FL_SPECTRAL_BINS60, depths=ds)
        spath = os.path.join(tmp, f"depths_{variant}.scene")
        fpath = os.path.join(tmp, f"depths_{variant}.film")
        oracle.write_scene_file(spath, sc, p)
        film, info = oracle.run_reference(spath, fpath, 64, 64)
        out[f"{variant}_xyz"] = film.astype(np.float64)
        out[f"{variant}_depths"] = np.array(ds, np.int32)
        print("depths", variant, ds, info)
    np.savez_compressed(os.path.join(HERE, "cornell_depths_ref.npz"), **out)


def delta(tmp):
    """the box with the reference's point, spot and directional lights added"""
    out = {}
    for variant in ("lambert", "materials"):
        sc = scenes.cornell_delta(64, 64, variant)
        p = scenes.render_params(4, 8, T.FL_SPECTRAL_BINS60)
        spath = os.path.join(tmp, f"delta_{variant}.scene")
        fpath = os.path.join(tmp, f"delta_{variant}.film")
        oracle.write_scene_file(spath, sc, p)
        film, info = oracle.run_reference(spath, fpath, 64, 64)
        out[f"{variant}_xyz"] = film.astype(np.float64)
        print("delta", variant, info)
    np.savez_compressed(os.path.join(HERE, "cornell_delta_ref.npz"), **out)


def metals(tmp):
    """the measured metal curves and InitializeForge's 60-bin spectra"""
    import subprocess
    path = os.path.join(tmp, "metals.bin")
    subprocess.run([oracle.REF_BIN, "--metals", path], check=True)
    np.savez_compressed(os.path.join(HERE, "metal_tables.npz"), **oracle.load_metals_dump(path))


def standard(tmp):
    """the box with StandardSurfaceMaterial boxes"""
    out = {}
    for variant, forge in (("standard", False), ("standard2", False), ("standard3", False), ("standard3", True)):
        sc = scenes.cornell(64, 64, variant)
        p = scenes.render_params(4, 8, T.FL_SPECTRAL_BINS60)
        key = variant + ("_forge" if forge else "")
        spath = os.path.join(tmp, f"{key}.scene")
        fpath = os.path.join(tmp, f"{key}.film")
        oracle.write_scene_file(spath, sc, p)
        film, info = oracle.run_reference(spath, fpath, 64, 64, forge=forge)
        out[f"{key}_xyz"] = film.astype(np.float64)
        print(key, info)
    np.savez_compressed(os.path.join(HERE, "cornell_standard_ref.npz"), **out)


def textures(tmp):
    """the box with image textures, with and without texture coordinates"""
    out = {}
    for key in ("uv", "nouv", "bump", "bump_nouv"):
        sc = scenes.cornell_textured(64, 64, bump=key.startswith("bump"))
        if key.endswith("nouv"):
            sc.uvs = None
        p = scenes.render_params(4, 8, T.FL_SPECTRAL_BINS60)
        spath = os.path.join(tmp, f"tex_{key}.scene")
        fpath = os.path.join(tmp, f"tex_{key}.film")
        oracle.write_scene_file(spath, sc, p)
        film, info = oracle.run_reference(spath, fpath, 64, 64)
        out[f"{key}_xyz"] = film.astype(np.float64)
        print("textured", key, info)
    np.savez_compressed(os.path.join(HERE, "cornell_textured_ref.npz"), **out)


PARTS = {"tables": tables, "pcg": pcg, "cornell": cornell, "materials": materials, "depths": depths, "delta": delta,
         "metals": metals, "standard": standard, "textures": textures}


def main(parts):
    sys.path.insert(0, ROOT)
    from __graft_entry__ import reference_dir
    if reference_dir() is None:
        sys.exit("the reference source tree is needed: set FL_REFERENCE_DIR")
    oracle.build(ref=True, ref_dir=reference_dir())
    scratch = os.path.join(ROOT, "oracle", "_ref", "tmp")
    os.makedirs(scratch, exist_ok=True)
    tmp = tempfile.mkdtemp(dir=scratch)
    for name in parts or list(PARTS):
        PARTS[name](tmp)


if __name__ == "__main__":
    main(sys.argv[1:])
