"""ctypes mirror of the C ABI records declared in include/ratbite_b200.h and
include/ratbite_b200_kernels.h.

The field order and types must match the headers exactly; test_abi.py checks
the sizes against the compiled library.
"""
import ctypes as C

RB_ABI_VERSION = 4

RB_OK = 0
RB_ERR_INVALID = -1
RB_ERR_CUDA = -2
RB_ERR_UNSUPPORTED = -3
RB_ERR_NO_SCENE = -4
RB_ERR_DEVICE = -5
RB_ERR_OOM = -6
RB_ERR_TOO_LARGE = -7

RB_DEV_STACK_OVERFLOW = 1 << 0
RB_DEV_QUEUE_OVERFLOW = 1 << 1
RB_DEV_NAN_RADIANCE = 1 << 2
RB_DEV_ITERATION_LIMIT = 1 << 3
RB_DEV_BAD_INDEX = 1 << 4
RB_DEV_BAD_GEOMETRY = 1 << 5

RB_INDEX_U16 = 0
RB_INDEX_U32 = 1

RB_BXDF_PURE_CONDUCTOR = 0
RB_BXDF_PURE_DIELECTRIC = 1
RB_BXDF_COMPLEX_SURFACE = 2

RB_ATTR_NORMAL = 1 << 0
RB_ATTR_FRAME = 1 << 1
RB_ATTR_COLOR = 1 << 2
RB_ATTR_TEX_COORD_1 = 1 << 3
RB_ATTR_TEX_COORD_2 = 1 << 4

RB_FACTOR_BASE_COLOR = 1 << 0
RB_FACTOR_METALNESS = 1 << 1
RB_FACTOR_ROUGHNESS = 1 << 2
RB_FACTOR_TRANSMISSION = 1 << 3
RB_FACTOR_CUTOFF = 1 << 4
RB_FACTOR_BLEND = 1 << 5
RB_FACTOR_SHEEN_COLOR = 1 << 6
RB_FACTOR_SHEEN_ROUGH = 1 << 7
RB_FACTOR_EMISSION = 1 << 8
# texture slots of rb_material.textures / texture_index (TextureTypeBitfield)
RB_TEXTURE_BASE_COLOR = 0
RB_TEXTURE_NORMAL = 1
RB_TEXTURE_MET_ROUGH = 2
RB_TEXTURE_TRANSMISSION = 3
RB_TEXTURE_SHEEN_COLOR = 4
RB_TEXTURE_SHEEN_ROUGH = 5
RB_TEXTURE_EMISSION = 6
RB_TEXTURE_SLOTS = 7
RB_TEXFMT_R8 = 0
RB_TEXFMT_RGBA8 = 1
RB_TEXADDR_WRAP = 0
RB_TEXADDR_CLAMP = 1
RB_TEXADDR_MIRROR = 2
RB_TEXFILTER_NEAREST = 0
RB_TEXFILTER_LINEAR = 1
RB_ACCEL_FLAT = 0
RB_ACCEL_INSTANCED = 1

RB_SPECTRUM_BINS = 471
RB_LUT_SIZE = 32

# PathStateBitfield (src/kernels/pathtrace.cu:25-37)
PS_PREVIOUS_HIT_SPECULAR = 1 << 0
PS_CURRENT_HIT_SPECULAR = 1 << 1
PS_REGULARIZED = 1 << 2
PS_RAY_REFRACTED = 1 << 3
PS_PATH_TERMINATED = 1 << 4
PS_TRIANGULAR_GEOMETRY = 1 << 5
PS_RIGHT_HANDED_FRAME = 1 << 6
PS_REFRACTION_HAPPENED = 1 << 7
PS_FINISHED = 1 << 8

# QRNG::DimensionOffset (src/device/quasi_random.h:13-29)
DIM_FILTER = 0
DIM_LENS = 1
DIM_WAVELENGTH = 0
DIM_LIGHT = 1
DIM_SURFACE_BXDF_0 = 2
DIM_SURFACE_BXDF_1 = 3
DIM_ALPHA_BLEND = 7
DIM_ROULETTE = 8

# LightType (src/core/light_tree_types.h:10-18)
LIGHT_TRIANGLE = 0
LIGHT_SKY = 1
LIGHT_NONE = 2

F3 = C.c_float * 3
F4 = C.c_float * 4
F12 = C.c_float * 12


RB_CDF_FP64 = 0
RB_CDF_REFERENCE = 1


class rb_config(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_paths_in_flight", C.c_uint32),
                ("envmap_cdf_mode", C.c_uint32), ("failed_sample_mode", C.c_uint32),
                ("inject_queue_limit", C.c_uint32), ("inject_alloc_failure", C.c_uint32),
                ("inject_stack_limit", C.c_uint32), ("acceleration", C.c_uint32)]


RB_FAILED_DROP = 0
RB_FAILED_KEEP = 1


class rb_jobs_options(C.Structure):
    _fields_ = [("max_paths_in_flight", C.c_uint32), ("grid_percent", C.c_uint32), ("done_events", C.c_void_p)]


class rb_material(C.Structure):
    _fields_ = [
        ("bxdf", C.c_uint32), ("double_sided", C.c_uint32), ("sheen_present", C.c_uint32),
        ("index_type", C.c_uint32), ("attributes", C.c_uint32), ("attribute_stride", C.c_uint32),
        ("normal_offset", C.c_uint32), ("frame_offset", C.c_uint32), ("color_offset", C.c_uint32),
        ("texcoord1_offset", C.c_uint32), ("texcoord2_offset", C.c_uint32),
        ("ior_spectrum", C.c_uint32), ("absorp_spectrum", C.c_uint32), ("emission_spectrum", C.c_uint32),
        ("mf_roughness", C.c_float), ("ior", C.c_float), ("alpha_cutoff", C.c_float),
        ("textures", C.c_uint32), ("factors", C.c_uint32),
        ("base_color", F4), ("metalness", C.c_float), ("roughness", C.c_float),
        ("transmission", C.c_float), ("sheen_color", F3), ("sheen_roughness", C.c_float),
        ("emissive", F3),
        ("triangle_count", C.c_uint32), ("indices", C.c_void_p),
        ("vertex_count", C.c_uint32), ("attribute_data", C.c_void_p),
        ("texcoord_sets", C.c_uint32), ("texture_index", C.c_uint32 * RB_TEXTURE_SLOTS),
    ]


class rb_texture(C.Structure):
    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32), ("format", C.c_uint32), ("srgb", C.c_uint32),
        ("address_u", C.c_uint32), ("address_v", C.c_uint32), ("filter", C.c_uint32), ("reserved", C.c_uint32),
        ("data", C.c_void_p),
    ]


class rb_submesh(C.Structure):
    _fields_ = [
        ("material", C.c_uint32), ("index_type", C.c_uint32), ("triangle_count", C.c_uint32),
        ("indices", C.c_void_p), ("vertex_count", C.c_uint32), ("vertices", C.c_void_p),
        ("discarded_count", C.c_uint32), ("discarded", C.c_void_p),
    ]


class rb_mesh(C.Structure):
    _fields_ = [("submesh_count", C.c_uint32), ("submeshes", C.POINTER(rb_submesh))]


class rb_instance(C.Structure):
    _fields_ = [("mesh", C.c_uint32), ("transform", F12)]


class rb_emissive_subset(C.Structure):
    _fields_ = [("transform", F12), ("triangle_count", C.c_uint32), ("vertices", C.c_void_p)]


class rb_geometry(C.Structure):
    _fields_ = [
        ("mesh_count", C.c_uint32), ("meshes", C.POINTER(rb_mesh)),
        ("instance_count", C.c_uint32), ("instances", C.POINTER(rb_instance)),
        ("emissive_subset_count", C.c_uint32), ("emissive_subsets", C.POINTER(rb_emissive_subset)),
    ]


class rb_light_tree(C.Structure):
    _fields_ = [
        ("triangle_count", C.c_uint32), ("triangles", C.c_void_p),
        ("node_count", C.c_uint32), ("nodes", C.c_void_p),
        ("pointer_count", C.c_uint32), ("pointers", C.c_void_p),
        ("bitmasks", C.c_void_p),
    ]


class rb_launch(C.Structure):
    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32),
        ("inv_width", C.c_float), ("inv_height", C.c_float),
        ("perspective_scale_w", C.c_float), ("perspective_scale_h", C.c_float),
        ("max_path_depth", C.c_uint32), ("max_reflected_depth", C.c_uint32),
        ("max_transmitted_depth", C.c_uint32),
        ("cam_u", F3), ("cam_v", F3), ("cam_w", F3),
        ("dof_enabled", C.c_uint32), ("aperture", C.c_float), ("focus_distance", C.c_float),
    ]


class rb_device_status(C.Structure):
    _fields_ = [("flags", C.c_uint32), ("first_code_detail", C.c_uint32),
                ("paths_traced", C.c_uint64), ("rays_traced", C.c_uint64)]


RB_MODE_IMMEDIATE = 0
RB_MODE_GRADUAL = 1


class rb_progress(C.Structure):
    _fields_ = [("launched_offset", C.c_uint32), ("launched_count", C.c_uint32), ("processed", C.c_uint32),
                ("total", C.c_uint32), ("finished", C.c_uint32), ("reserved", C.c_uint32)]


RB_STATS_COUNT = 1
RB_STATS_TIME = 2


class rb_render_stats(C.Structure):
    _fields_ = [
        ("extend_rays", C.c_uint64), ("extend_nodes", C.c_uint64), ("extend_tris", C.c_uint64),
        ("shadow_rays", C.c_uint64), ("shadow_nodes", C.c_uint64), ("shadow_tris", C.c_uint64),
        ("waves", C.c_uint64),
        ("ms_generate", C.c_double), ("ms_extend", C.c_double), ("ms_shade", C.c_double),
        ("ms_shadow", C.c_double), ("ms_resolve", C.c_double),
        ("launches_generate", C.c_uint32), ("launches_extend", C.c_uint32), ("launches_shade", C.c_uint32),
        ("launches_shadow", C.c_uint32), ("launches_resolve", C.c_uint32), ("reserved", C.c_uint32),
        ("ms_surface", C.c_double), ("ms_nee", C.c_double), ("ms_bsdf", C.c_double),
        ("launches_nee", C.c_uint32), ("launches_bsdf", C.c_uint32),
        ("surface_records", C.c_uint64),
    ]


class rb_bxdf_case(C.Structure):
    _fields_ = [
        ("material", C.c_uint32), ("sample", C.c_uint32), ("hash", C.c_uint32), ("bounce", C.c_uint32),
        ("frame_t", F3), ("frame_b", F3), ("frame_n", F3),
        ("layers", C.c_uint32), ("base_color", F3), ("metalness", C.c_float), ("ior", C.c_float),
        ("roughness", C.c_float), ("transmission", C.c_float), ("sheen_color", F3),
        ("sheen_alpha", C.c_float),
        ("light_spectrum", F4), ("light_dir", F3), ("light_pdf", C.c_float), ("occluded", C.c_uint32),
        ("L", F4), ("lambda_", F4), ("lambda_pdf", F4), ("active_count", C.c_float),
        ("throughput", F4), ("bxdf_pdf", C.c_float), ("dir", F3), ("flags", C.c_uint32),
        ("refraction_scale", C.c_float),
    ]


class rb_light_case(C.Structure):
    _fields_ = [
        ("position", F3), ("normal", F3), ("rand", C.c_float),
        ("type", C.c_uint32), ("index", C.c_uint32), ("pdf", C.c_float),
        ("q_type", C.c_uint32), ("q_index", C.c_uint32), ("q_pdf", C.c_float),
    ]


# numpy dtypes of the reference's light-tree records (the byte layouts
# rb_set_lights takes): EmissiveTriangleLightData (68 B), PackedNode (32 B).
def emissive_triangle_dtype():
    import numpy as np
    return np.dtype([("vertices", "<f4", 9), ("uvs", "<f4", 6), ("material", "<u4"), ("prim", "<u4")])


def packed_node_dtype():
    import numpy as np
    return np.dtype([("mean", "<f4", 3), ("variance", "<f4"), ("direction", "<u4"),
                     ("sharpness", "<f4"), ("flux", "<f4"), ("core", "<u4")])


NRC_INPUTS = 10


class rb_nrc_config(C.Structure):
    _fields_ = [("device", C.c_int32), ("seed", C.c_uint32), ("learning_rate", C.c_float), ("beta1", C.c_float),
                ("beta2", C.c_float), ("epsilon", C.c_float), ("reserved", C.c_uint32 * 2)]


class rb_cache_params(C.Structure):
    _fields_ = [("spread_threshold", C.c_float), ("train_one_in", C.c_uint32), ("targets_per_sample", C.c_uint32),
                ("batch", C.c_uint32), ("frozen", C.c_uint32), ("samples_per_wave", C.c_uint32),
                ("scene_min", C.c_float * 3), ("scene_max", C.c_float * 3), ("min_roughness", C.c_float),
                ("reserved", C.c_uint32 * 3)]


class rb_cache_stats(C.Structure):
    _fields_ = [("queries", C.c_uint64), ("records", C.c_uint64), ("steps", C.c_uint64), ("last_loss", C.c_float),
                ("launches", C.c_uint32), ("ms_infer", C.c_double), ("ms_train", C.c_double),
                ("drop_bias", C.c_float), ("drop_bias_other", C.c_float), ("radiance_scale", C.c_float)]
