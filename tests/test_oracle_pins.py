"""Pins the CPU oracle against the reference's own outputs (fixtures made by
tests/golden/make_golden.py from the reference compiled in place)."""
import os

import numpy as np

import filianore_b200 as fb
import oracle
from filianore_b200 import scenes, types as T

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_pcg32_matches_vendored_pcg32():
    g = np.load(os.path.join(GOLDEN, "pcg32_kat.npz"))
    for (s, q), seq in zip(g["seeds"], g["seq"]):
        assert np.array_equal(oracle.pcg32_sequence(int(s), int(q), 0, 16), seq)
    for delta, seq in zip(g["adv_deltas"], g["adv"]):
        assert np.array_equal(oracle.pcg32_sequence(7, 1, int(delta), 8), seq)


def test_binned_tables_bit_exact(orc_tables, ref_tables):
    # InitializeSpectrals (color/spectruminits.cpp:6-64) restated
    assert np.array_equal(orc_tables.binned(), ref_tables["binned60"])


def test_from_reflectance_rgb_bit_exact(orc_tables, ref_tables):
    rgbs = [(0.725, 0.725, 0.725), (0.63, 0.065, 0.05), (0.14, 0.45, 0.091), (0.2, 0.9, 0.5)]
    for rgb, want in zip(rgbs, ref_tables["refl60_kat"]):
        assert np.array_equal(orc_tables.reflectance(rgb), want)


def test_to_xyz_of_constant_spectrum(ref_tables):
    # to_xyz(1) of the reference: Y of a unit constant spectrum is ~1 by construction
    x = ref_tables["xyz_of_one"]
    assert abs(float(x[1]) - 1.0) < 2e-3


def test_oracle_render_equals_reference_integrator(orc_tables):
    """60-bin restatement vs the reference's PathIntegrator on the Cornell box, same
    per-pixel PCG streams: bit-exact at 64x64, 4 spp."""
    g = np.load(os.path.join(GOLDEN, "cornell_ref.npz"))
    sc = scenes.cornell(64, 64)
    film, cnt = oracle.render(sc, orc_tables, scenes.render_params(4, 8, T.FL_SPECTRAL_BINS60))
    assert cnt["paths"] == 64 * 64 * 4
    assert np.array_equal(film, g["small_xyz"])


def test_oracle_render_full_cornell_matches_reference(orc_tables):
    """256x256, 16 spp, depth 8 (the CPU-runnable Cornell configuration); the fixture is
    stored as float32, so the bound is float32 rounding."""
    g = np.load(os.path.join(GOLDEN, "cornell_ref.npz"))
    sc = scenes.cornell(256, 256)
    film, _ = oracle.render(sc, orc_tables, scenes.render_params(16, 8, T.FL_SPECTRAL_BINS60))
    ref = g["full_xyz"].astype(np.float64)
    np.testing.assert_allclose(film, ref, rtol=2e-7, atol=1e-12)


def test_oracle_materials_equal_reference_bxdfs(orc_tables):
    """GGX conductor, rough dielectric (Walter transmission + microfacet reflection) and
    smooth glass, composed from the reference's own BxDF classes in the reference build,
    against the restatement: bit-exact at 64x64 x 4 spp, float32 rounding at 128x128 x 16."""
    g = np.load(os.path.join(GOLDEN, "cornell_materials_ref.npz"))
    for variant in ("materials", "glass"):
        sc = scenes.cornell(64, 64, variant)
        film, _ = oracle.render(sc, orc_tables, scenes.render_params(4, 8, T.FL_SPECTRAL_BINS60))
        assert np.array_equal(film, g[f"{variant}_small_xyz"]), variant
        sc = scenes.cornell(128, 128, variant)
        film, _ = oracle.render(sc, orc_tables, scenes.render_params(16, 8, T.FL_SPECTRAL_BINS60))
        np.testing.assert_allclose(film, g[f"{variant}_full_xyz"].astype(np.float64), rtol=2e-7, atol=1e-12)


def test_oracle_lobe_depths_equal_reference(orc_tables):
    """RenderParams with a different depth per lobe kind (pathintegrator.cpp:55-65: each an
    exact == test on the sampled lobe's kind, so paths run past the deepest one until
    Russian roulette ends them): bit-exact against the reference integrator at 64x64 x 4 spp,
    and different from the equal-depth render."""
    g = np.load(os.path.join(GOLDEN, "cornell_depths_ref.npz"))
    for variant in ("materials", "glass", "standard2", "standard3"):
        ds = tuple(int(d) for d in g[f"{variant}_depths"])
        sc = scenes.cornell(64, 64, variant)
        film, _ = oracle.render(sc, orc_tables, scenes.render_params(4, 8, T.FL_SPECTRAL_BINS60, depths=ds))
        assert np.array_equal(film, g[f"{variant}_xyz"]), variant
        deepest, _ = oracle.render(sc, orc_tables, scenes.render_params(4, max(ds), T.FL_SPECTRAL_BINS60))
        assert not np.array_equal(deepest, film)
        if variant != "materials":  # the materials box's GGX lobes never sample (seen from below)
            shallow, _ = oracle.render(sc, orc_tables, scenes.render_params(4, ds[0], T.FL_SPECTRAL_BINS60))
            assert not np.array_equal(shallow, film), variant


def test_oracle_delta_lights_equal_reference(orc_tables):
    """The reference's PointIlluminant, SpotIlluminant and DirectionalIlluminant (unweighted
    NEE, no BSDF-sampled MIS ray, d^2 decay) in the Cornell box beside its area light,
    Lambert and GGX materials: the restatement is bit-exact at 64x64 x 4 spp."""
    g = np.load(os.path.join(GOLDEN, "cornell_delta_ref.npz"))
    for variant in ("lambert", "materials"):
        sc = scenes.cornell_delta(64, 64, variant)
        film, _ = oracle.render(sc, orc_tables, scenes.render_params(4, 8, T.FL_SPECTRAL_BINS60))
        assert np.array_equal(film, g[f"{variant}_xyz"]), (variant, np.abs(film - g[f"{variant}_xyz"]).max())
        assert film.mean() > 0


def test_oracle_standard_surface_equal_reference(orc_tables):
    """StandardSurfaceMaterial built by the reference's own compute_scattering_functions
    (Oren-Nayar, Fresnel-blended diffuse/specular with Schlick dielectric and metallic
    Fresnel, Estevez sheen, GTR1 clear coat, specular R/T glass) in the Cornell box: the
    restatement is bit-exact at 64x64 x 4 spp."""
    g = np.load(os.path.join(GOLDEN, "cornell_standard_ref.npz"))
    for variant in ("standard", "standard2", "standard3"):
        sc = scenes.cornell(64, 64, variant)
        film, _ = oracle.render(sc, orc_tables, scenes.render_params(4, 8, T.FL_SPECTRAL_BINS60))
        assert np.array_equal(film, g[f"{variant}_xyz"]), (variant, np.abs(film - g[f"{variant}_xyz"]).max())
        assert film.mean() > 0


def test_oracle_measured_metals_equal_reference():
    """Measured-metal eta / k binned from the curves of color/metallurgy.h as InitializeForge
    does, bit-exact against the reference's own binning; without curves every metal is zero
    (the reference never calls InitializeForge). The "standard3" box (thin-walled diffuse
    transmission, measured copper with a thin film and a clear coat) after InitializeForge
    is bit-exact against the reference run with InitializeForge."""
    m = np.load(os.path.join(GOLDEN, "metal_tables.npz"))
    tab = oracle.Tables(fb.reference_tables(measured_metals=True))
    got = tab.metals()
    assert np.array_equal(got[:, 0], m["eta60"]) and np.array_equal(got[:, 1], m["k60"])
    assert (m["eta60"] > 0).all() and (m["k60"] > 0).all()
    assert not oracle.Tables(fb.reference_tables()).metals().any()
    g = np.load(os.path.join(GOLDEN, "cornell_standard_ref.npz"))
    film, _ = oracle.render(scenes.cornell(64, 64, "standard3"), tab, scenes.render_params(4, 8, T.FL_SPECTRAL_BINS60))
    assert np.array_equal(film, g["standard3_forge_xyz"])
    assert not np.array_equal(film, g["standard3_xyz"])


def test_oracle_image_textures_equal_reference(orc_tables):
    """ImageMapTexture (the reference's own class, reading the images through stbi_load) on
    Lambert materials and a StandardSurface kd: bit-exact with texture coordinates (u over
    [-0.15, 1.15] on the boxes, so the texel clamps are reached) and without them (every hit
    at uv (0, 0), as the reference's BVH::intersect leaves it); and with bump maps, which run
    the reference's own Material::bump_evaluate and set_shading_geometry."""
    g = np.load(os.path.join(GOLDEN, "cornell_textured_ref.npz"))
    for key in ("uv", "nouv", "bump", "bump_nouv"):
        sc = scenes.cornell_textured(64, 64, bump=key.startswith("bump"))
        if key.endswith("nouv"):
            sc.uvs = None
        film, _ = oracle.render(sc, orc_tables, scenes.render_params(4, 8, T.FL_SPECTRAL_BINS60))
        assert np.array_equal(film, g[f"{key}_xyz"]), (key, np.abs(film - g[f"{key}_xyz"]).max())
    assert not np.array_equal(g["uv_xyz"], g["nouv_xyz"])


def test_texel_rule_edges():
    """ImageMapTexture's nearest-texel rule (shading/textures/imagemap.cpp:36-62) on a 5 x 3
    image whose texels encode their column and row: i = int(u * width) and j = int((1 - v) *
    height - 0.001), truncated toward zero and clamped to the image. For a row past the last
    (v < 0) the reference sets i = height - 1 and reads outside the image; the oracle (like
    the library) clamps j as well and returns the texel (min(height - 1, width - 1), last row)."""
    W, H = 5, 3
    img = np.zeros((H, W, 3), np.uint8)
    for j in range(H):
        for i in range(W):
            img[j, i] = (10 * i, 10 * j, 7)
    cases = [((0.0, 0.0), (0, 2)), ((0.99, 0.99), (4, 0)), ((0.5, 0.5), (2, 1)), ((-0.3, 0.5), (0, 1)),
             ((1.7, 0.5), (4, 1)), ((0.5, 1.8), (2, 0)), ((0.2, 2 / 3), (1, 0)), ((0.2, 0.3333), (1, 1)),
             ((0.9, -0.2), (2, 2)), ((0.1, -5.0), (2, 2))]
    got = oracle.image_texels(img, np.array([c[0] for c in cases], np.float32))
    for (uv, (i, j)), rgb in zip(cases, got):
        assert np.array_equal(rgb, img[j, i] / np.float32(255.0)), (uv, i, j, rgb * 255)


def test_oracle_li_on_camera_rays_equals_render(orc_tables):
    """The oracle's per-ray PathIntegrator::Li (orc_li) on the render loop's camera rays of
    sample 0 adds up to the 1-spp film of orc_render exactly, in both spectral modes and with
    unequal lobe depths: the per-ray entry point and the image loop are the same estimator."""
    sc = scenes.cornell(24, 16, "glass")
    o, d, r, lam = oracle.camera_rays(sc, np.arange(24 * 16))
    for mode in (T.FL_SPECTRAL_BINS60, T.FL_SPECTRAL_HERO4):
        p = scenes.render_params(1, 8, mode, depths=(5, 3, 6))
        film, _ = oracle.render(sc, orc_tables, p)
        _, r_out, xyz = oracle.li(sc, orc_tables, p, o, d, r, lam)
        assert np.array_equal(xyz.reshape(16, 24, 3), film)
        assert np.any(r_out != r)  # paths that hit draw numbers (misses draw none)
