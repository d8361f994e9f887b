"""ctypes mirrors of the structs in include/filianore_gpu.h (the C ABI)."""
import ctypes as C

import numpy as np

FL_OK = 0
FL_ERR_INVALID = -1
FL_ERR_OOM = -2
FL_ERR_CUDA = -3
FL_ERR_TIMEOUT = -4
FL_ERR_TRAVERSAL = -5
FL_ERR_NOT_READY = -6
FL_ERR_CAPACITY = -7
FL_ERR_NO_DEVICE = -8

FL_MEM_HOST = 0
FL_MEM_DEVICE = 1

FL_MAT_LAMBERT = 0
FL_MAT_CONDUCTOR = 1
FL_MAT_ROUGH_DIELECTRIC = 2
FL_MAT_SMOOTH_DIELECTRIC = 3

FL_LIGHT_TRIANGLE = 0
FL_LIGHT_SPHERE = 1
FL_LIGHT_ENV = 2
FL_LIGHT_POINT = 3
FL_LIGHT_SPOT = 4
FL_LIGHT_DIRECTIONAL = 5

FL_SPECTRAL_HERO4 = 0
FL_SPECTRAL_BINS60 = 1

FL_RENDER_PROFILE = 1
FL_RENDER_COUNT = 2
FL_RENDER_CORRECTED_GGX = 4
FL_RENDER_LOBE_DEPTHS = 8
FL_MAX_BOUNCES = 250
FL_MAT_STANDARD = 4
FL_FRESNEL_DIELECTRIC = 0
FL_FRESNEL_METALLIC = 1
FL_FRESNEL_MEASURED_METAL = 2
METALS = ("gold", "copper", "silver", "aluminium", "beryllium", "chromium", "mercury", "iridium", "lithium")

FL_SERVE_SHORTEST_FIRST = 0
FL_SERVE_FIRST_COME = 1
FL_SERVE_FAIR_SHARE = 2
FL_SERVE_SHORTEST_FIRST_AGED = 3
FL_SERVE_RESPONSE_RATIO = 4
FL_SERVE_DEADLINE = 5
FL_SERVE_FIRST_COME_LANE = 6
FL_GUIDE_TRAIN_MMA_SYNC = 0
FL_GUIDE_TRAIN_TCGEN05 = 1


class fl_spectral_tables(C.Structure):
    _fields_ = [
        ("cie_lambda", C.POINTER(C.c_float)),
        ("cie_x", C.POINTER(C.c_float)),
        ("cie_y", C.POINTER(C.c_float)),
        ("cie_z", C.POINTER(C.c_float)),
        ("n_cie", C.c_int32),
        ("cie_y_integral", C.c_float),
        ("rgb2spec_lambda", C.POINTER(C.c_float)),
        ("n_rgb2spec", C.c_int32),
        ("refl", C.POINTER(C.c_float) * 7),
        ("illum", C.POINTER(C.c_float) * 7),
        ("n_metals", C.c_int32),
        ("metal_n", C.c_int32 * 9),
        ("metal_lambda", C.POINTER(C.c_float) * 9),
        ("metal_eta", C.POINTER(C.c_float) * 9),
        ("metal_k", C.POINTER(C.c_float) * 9),
    ]


class fl_material(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("rgb", C.c_float * 3),
        ("roughness", C.c_float),
        ("eta", C.c_float),
        ("k", C.c_float),
        ("standard", C.c_int32),
        ("texture", C.c_int32),
    ]


class fl_image(C.Structure):
    _fields_ = [
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("rgb", C.POINTER(C.c_uint8)),
    ]


class fl_light(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("tri", C.c_uint32),
        ("radiance", C.c_float),
        ("radius", C.c_float),
        ("center", C.c_float * 3),
        ("direction", C.c_float * 3),
        ("cone_angle", C.c_float),
        ("penumbra_angle", C.c_float),
    ]


class fl_standard_surface(C.Structure):
    _fields_ = [
        ("kd", C.c_float * 3), ("kd_weight", C.c_float), ("kd_roughness", C.c_float),
        ("ks", C.c_float * 3), ("ks_weight", C.c_float), ("ks_roughness", C.c_float), ("ks_anisotropic", C.c_float),
        ("ks_ior", C.c_float), ("fresnel_type", C.c_int32), ("metal_type", C.c_int32),
        ("kt", C.c_float * 3), ("kt_weight", C.c_float),
        ("sheen_color", C.c_float * 3), ("sheen_weight", C.c_float), ("sheen_roughness", C.c_float),
        ("coat_color", C.c_float * 3), ("coat_weight", C.c_float), ("coat_ior", C.c_float), ("coat_gloss", C.c_float),
        ("thin_film_thickness", C.c_float), ("thin_film_ior", C.c_float), ("thin_walled", C.c_int32),
        ("kd_texture", C.c_int32),
        ("bump_texture", C.c_int32),
    ]


class fl_scene_desc(C.Structure):
    _fields_ = [
        ("verts", C.POINTER(C.c_float)),
        ("n_tri", C.c_uint32),
        ("tri_material", C.POINTER(C.c_uint32)),
        ("materials", C.POINTER(fl_material)),
        ("n_materials", C.c_uint32),
        ("lights", C.POINTER(fl_light)),
        ("n_lights", C.c_uint32),
        ("standard_surfaces", C.POINTER(fl_standard_surface)),
        ("n_standard_surfaces", C.c_uint32),
        ("uvs", C.POINTER(C.c_float)),
        ("images", C.POINTER(fl_image)),
        ("n_images", C.c_uint32),
    ]


class fl_scene_info(C.Structure):
    _fields_ = [
        ("n_tri", C.c_uint32),
        ("n_nodes", C.c_uint32),
        ("n_leaves", C.c_uint32),
        ("max_depth", C.c_uint32),
        ("bvh_bytes", C.c_uint64),
        ("build_ms", C.c_double),
    ]


class fl_hit(C.Structure):
    _fields_ = [("id", C.c_int32), ("t", C.c_float), ("u", C.c_float), ("v", C.c_float)]


class fl_camera(C.Structure):
    _fields_ = [
        ("position", C.c_float * 3),
        ("look_at", C.c_float * 3),
        ("up", C.c_float * 3),
        ("vfov_deg", C.c_float),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("aperture", C.c_float),
    ]


class fl_render_params(C.Structure):
    _fields_ = [
        ("spp", C.c_int32),
        ("max_depth", C.c_int32),
        ("rr_threshold", C.c_float),
        ("spectral_mode", C.c_int32),
        ("wave_paths", C.c_int32),
        ("sample_offset", C.c_uint32),
        ("flags", C.c_int32),
        ("reserved", C.c_int32),
        ("diffuse_depth", C.c_int32),
        ("reflection_depth", C.c_int32),
        ("transmission_depth", C.c_int32),
        ("reserved2", C.c_int32),
    ]


class fl_render_stats(C.Structure):
    _fields_ = [
        ("paths", C.c_uint64),
        ("rays", C.c_uint64),
        ("shadow_rays", C.c_uint64),
        ("bounces", C.c_uint64),
        ("ms", C.c_double),
        ("traversal_errors", C.c_uint32),
        ("launches", C.c_uint32),
        ("ms_trace", C.c_double),
        ("ms_shade", C.c_double),
        ("ms_shadow", C.c_double),
        ("ms_continue", C.c_double),
        ("nodes_visited", C.c_uint64),
        ("tris_tested", C.c_uint64),
        ("paths_cut", C.c_uint64),
    ]


HIT_DTYPE = [("id", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")]


class fl_server_config(C.Structure):
    _fields_ = [
        ("memory_budget_bytes", C.c_uint64),
        ("wave_paths", C.c_int32),
        ("max_depth", C.c_int32),
        ("max_jobs", C.c_int32),
        ("max_lights", C.c_int32),
        ("policy", C.c_int32),
    ]


class fl_job_desc(C.Structure):
    _fields_ = [("scene_id", C.c_uint64), ("camera", fl_camera), ("params", fl_render_params)]


class fl_job_stats(C.Structure):
    _fields_ = [("submit_ms", C.c_double), ("start_ms", C.c_double), ("done_ms", C.c_double),
                ("samples", C.c_uint64)]


class fl_server_stats(C.Structure):
    _fields_ = [
        ("jobs_submitted", C.c_uint64), ("jobs_done", C.c_uint64), ("waves", C.c_uint64), ("paths", C.c_uint64),
        ("builds", C.c_uint64), ("evictions", C.c_uint64), ("resident_bytes", C.c_uint64),
        ("running", C.c_uint32), ("pending", C.c_uint32), ("busy_ms", C.c_double),
        ("wave_max_ms", C.c_double), ("build_ms", C.c_double), ("build_max_ms", C.c_double),
        ("finish_ms", C.c_double), ("idle_ms", C.c_double),
    ]


class fl_guide_config(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64),
        ("learning_rate", C.c_float),
        ("select_prob", C.c_float),
        ("batch", C.c_int32),
        ("max_records", C.c_int32),
        ("steps_per_wave", C.c_int32),
        ("position_scale", C.c_float),
        ("weight_average", C.c_float),
        ("learn_select", C.c_int32),
        ("train_kernel", C.c_int32),
    ]


FL_GUIDE_SAMPLE = 1
FL_GUIDE_TRAIN = 2
FL_GUIDE_PARAMS = 20032
FL_GUIDE_RECORD_FLOATS = 20


def set_metal_tables(s, t: dict, fp):
    """fills the metal fields of an fl_spectral_tables from a tables dict; returns the arrays
    the struct points to (keep them alive)"""
    if "metal_lambda_0" not in t:
        s.n_metals = 0
        return []
    keep = []
    s.n_metals = 9
    for i in range(9):
        arrs = [np.ascontiguousarray(t[f"metal_{key}_{i}"], np.float32) for key in ("lambda", "eta", "k")]
        keep += arrs
        s.metal_n[i] = arrs[0].shape[0]
        s.metal_lambda[i], s.metal_eta[i], s.metal_k[i] = (fp(a) for a in arrs)
    return keep
