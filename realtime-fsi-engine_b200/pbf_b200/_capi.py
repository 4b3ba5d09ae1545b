"""ctypes binding of the engine's C ABI (include/pbf_b200.h).

This is the binding a Python caller of the reference's fluid path would add:
every function of the header is declared here with its exact signature.  The
shared library is the in-tree build ``realtime-fsi-engine_b200/lib/libpbf_b200.so``;
there is no fallback — a missing library raises ``ImportError``.
"""
import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("PBF_B200_LIB", os.path.join(PKG_DIR, "lib", "libpbf_b200.so"))

PBF_OK = 0
PBF_ERR_INVALID = -1
PBF_ERR_CUDA = -2
PBF_ERR_STATE = -3
PBF_ERR_ALLOC = -4
PBF_ERR_NUMERIC = -5
PBF_ERR_TIMEOUT = -6
PBF_ERR_NOT_BUILT = -7

STAGE_PREDICT, STAGE_SORT, STAGE_TABLE, STAGE_REORDER = 1, 2, 3, 4
STAGE_LAMBDA, STAGE_DELTAP, STAGE_INTEGRATE, STAGE_VORTICITY = 5, 6, 7, 8
BUF_KEYS, BUF_SORTED_KEYS, BUF_SORTED_IDS, BUF_TABLE = 1, 2, 3, 4
BUF_XSTAR, BUF_VPRED, BUF_RHO, BUF_OMEGA, BUF_POS, BUF_VEL, BUF_LOD = 5, 6, 7, 8, 9, 10, 11
NUM_PASS_SLOTS = 12
PASS_NAMES = {0: "step", 1: "predict_hash", 2: "radix_sort", 3: "cell_table", 4: "reorder", 5: "lambda",
              6: "deltap_apply", 7: "integrate", 8: "vorticity"}


class FluidConfig(C.Structure):
    """pbf_fluid_config == FluidConfig (include/core/config.h:9-63)."""

    _fields_ = [
        ("dt", C.c_float), ("gravity", C.c_float * 3), ("h", C.c_float), ("rho0", C.c_float),
        ("solver_iterations", C.c_uint32), ("substep_iterations", C.c_uint32), ("eps", C.c_float),
        ("particle_count", C.c_uint32), ("spawn_min", C.c_float * 3), ("spawn_max", C.c_float * 3),
        ("spawn_random", C.c_uint32), ("spacing", C.c_float), ("initial_velocity", C.c_float * 3),
        ("bounds_min", C.c_float * 3), ("bounds_max", C.c_float * 3), ("bound_damping", C.c_float),
        ("hash_size", C.c_uint32), ("enable_scorr", C.c_uint32), ("k_corr", C.c_float),
        ("n_corr", C.c_float), ("delta_q", C.c_float), ("cohesion_strength", C.c_float),
        ("enable_viscosity", C.c_uint32), ("viscosity", C.c_float), ("interaction_radius", C.c_float),
        ("interaction_strength", C.c_float), ("enable_vorticity", C.c_uint32),
        ("vorticity_epsilon", C.c_float), ("enable_apbf", C.c_uint32), ("min_lod", C.c_uint32),
        ("max_lod", C.c_uint32), ("lod_max_dist", C.c_float),
    ]


class DerivedParams(C.Structure):
    """pbf_derived_params == FluidConfigUBO (include/fluid/PBFluids.h:21-61)."""

    _fields_ = [
        ("bounds_min", C.c_float * 4), ("bounds_max", C.c_float * 4), ("gravity_dt", C.c_float * 4),
        ("h", C.c_float), ("rho0", C.c_float), ("eps", C.c_float), ("wq", C.c_float),
        ("k_corr", C.c_float), ("n_corr", C.c_float), ("viscosity", C.c_float), ("bound_damping", C.c_float),
        ("hash_size", C.c_uint32), ("particle_count", C.c_uint32), ("enable_scorr", C.c_uint32),
        ("enable_viscosity", C.c_uint32), ("cohesion_strength", C.c_float), ("interaction_radius", C.c_float),
        ("interaction_strength", C.c_float), ("w0_self", C.c_float), ("hash_mask", C.c_uint32),
        ("poly6_coeff", C.c_float), ("spiky_coeff", C.c_float), ("inv_rho0", C.c_float),
        ("min_lod", C.c_uint32), ("max_lod", C.c_uint32), ("lod_max_dist", C.c_float), ("enable_apbf", C.c_uint32),
    ]


class Particle(C.Structure):
    """pbf_particle == Particle (include/fluid/Particle.h:8-12), 48 bytes."""

    _fields_ = [("pos", C.c_float * 3), ("pad0", C.c_float), ("pred_pos", C.c_float * 3), ("pad1", C.c_float),
                ("vel", C.c_float * 3), ("pad2", C.c_float)]


class ContactCandidate(C.Structure):
    """pbf_contact_candidate == ContactCandidate (include/fluid/PBFluids.h:67-70)."""

    _fields_ = [("pos", C.c_float * 4), ("vel", C.c_float * 4)]


class SceneDesc(C.Structure):
    """pbf_scene_desc: one scene of a batch (particle count, hash size, walls)."""

    _fields_ = [("num_particles", C.c_uint32), ("hash_size", C.c_uint32), ("bounds_min", C.c_float * 3),
                ("bounds_max", C.c_float * 3)]


class BatchTuning(C.Structure):
    """pbf_batch_tuning: one autotuner candidate and its time per step."""

    _fields_ = [("block", C.c_int32), ("order", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("ms_per_step", C.c_float), ("neighbour_mode", C.c_int32)]


class DeformParams(C.Structure):
    """pbf_deform_params == SceneDeform's handle policy (include/core/Scene.h:17-27)."""

    _fields_ = [("stiffness", C.c_float), ("max_displacement", C.c_float), ("max_total_disp", C.c_float),
                ("restore_enabled", C.c_uint32), ("restore_strength", C.c_float),
                ("control_threshold", C.c_float), ("control_threshold_low", C.c_float)]


class ScenePreset(C.Structure):
    """pbf_scene_preset (include/core/Scene.h:29-67 as a C struct)."""

    _fields_ = [("name", C.c_char * 48), ("fluid", FluidConfig), ("cam_yaw", C.c_float), ("cam_pitch", C.c_float),
                ("cam_dist", C.c_float), ("point_size", C.c_float), ("mesh_file", C.c_char * 64),
                ("mesh_fit_size", C.c_float), ("sdf_cell", C.c_float), ("sdf_padding", C.c_float),
                ("sdf_container", C.c_uint32), ("mesh_translate", C.c_float * 3), ("mesh_rot_deg", C.c_float * 3),
                ("deform", DeformParams), ("local_kring", C.c_int32), ("contact_radius", C.c_float)]


BATCH_ALL = 0xFFFFFFFF
BOPT_BLOCK, BOPT_ORDER, BOPT_BLOCKS_PER_SM, BOPT_USE_GRAPH, BOPT_NEIGHBOUR_MODE = 1, 2, 3, 4, 5

assert C.sizeof(Particle) == 48 and C.sizeof(ContactCandidate) == 32
assert C.sizeof(DerivedParams) == 144
assert C.sizeof(SceneDesc) == 32 and C.sizeof(BatchTuning) == 20

vp = C.c_void_p
i32 = C.c_int32
u32 = C.c_uint32
P = C.POINTER

# (name, restype, argtypes) of every entry point in include/pbf_b200.h
SIGNATURES = [
    ("pbf_abi_version", C.c_int, []),
    ("pbf_last_error", C.c_char_p, []),
    ("pbf_default_config", C.c_int, [P(FluidConfig)]),
    ("pbf_derive_params", C.c_int, [P(FluidConfig), C.c_float, P(DerivedParams)]),
    ("pbf_create", C.c_int, [P(FluidConfig), C.c_int, P(vp)]),
    ("pbf_destroy", C.c_int, [vp]),
    ("pbf_set_params", C.c_int, [vp, P(FluidConfig)]),
    ("pbf_get_params", C.c_int, [vp, P(FluidConfig)]),
    ("pbf_get_derived", C.c_int, [vp, P(DerivedParams)]),
    ("pbf_set_bounds", C.c_int, [vp, P(C.c_float), P(C.c_float), C.c_float]),
    ("pbf_set_collision_padding", C.c_int, [vp, C.c_float]),
    ("pbf_set_camera_pos", C.c_int, [vp, P(C.c_float)]),
    ("pbf_set_interaction", C.c_int, [vp, C.c_int, P(C.c_float)]),
    ("pbf_set_particles", C.c_int, [vp, vp, u32]),
    ("pbf_upload_particles", C.c_int, [vp, vp, u32]),
    ("pbf_particle_count", C.c_int, [vp, P(u32)]),
    ("pbf_read_particles", C.c_int, [vp, vp, u32]),
    ("pbf_set_particles_device", C.c_int, [vp, vp, vp, u32]),
    ("pbf_read_particles_device", C.c_int, [vp, vp, vp, u32]),
    ("pbf_step", C.c_int, [vp]),
    ("pbf_sync", C.c_int, [vp]),
    ("pbf_get_stream", C.c_int, [vp, P(vp)]),
    ("pbf_set_sdf_grid", C.c_int, [vp, vp, P(i32), P(C.c_float), C.c_float]),
    ("pbf_clear_sdf", C.c_int, [vp]),
    ("pbf_attach_sdf", C.c_int, [vp, vp]),
    ("pbf_set_sdf_mode", C.c_int, [vp, C.c_float, C.c_int]),
    ("pbf_read_sdf_grid", C.c_int, [vp, vp, C.c_size_t]),
    ("pbf_sample_sdf", C.c_int, [vp, vp, u32, vp, vp]),
    ("pbf_set_sdf_mesh", C.c_int, [vp, vp, i32, vp, i32, C.c_double]),
    ("pbf_rebuild_mesh", C.c_int, [vp, vp, i32]),
    ("pbf_update_mesh_vertices", C.c_int, [vp, vp, i32]),
    ("pbf_sdf_grid_info", C.c_int, [vp, P(i32), P(C.c_double), P(C.c_double)]),
    ("pbf_closest_triangle", C.c_int, [vp, vp, u32, vp, vp]),
    ("pbf_filter_contacts", C.c_int, [vp, C.c_float]),
    ("pbf_read_contacts", C.c_int, [vp, vp, u32, P(u32)]),
    ("pbf_vertex_forces", C.c_int, [vp, C.c_float, C.c_int, vp, i32, P(i32)]),
    ("pbf_run_stage", C.c_int, [vp, C.c_int, u32]),
    ("pbf_read_buffer", C.c_int, [vp, C.c_int, vp, C.c_size_t]),
    ("pbf_buffer_device_ptr", C.c_int, [vp, C.c_int, P(vp), P(C.c_size_t)]),
    ("pbf_sort_keys", C.c_int, [vp, u32, u32, vp, vp]),
    ("pbf_build_table", C.c_int, [vp, u32, u32, vp]),
    ("pbf_sort_keys_noalloc", C.c_int, [vp, u32, u32, vp, vp, vp]),
    ("pbf_set_profiling", C.c_int, [vp, C.c_int]),
    ("pbf_read_pass_times", C.c_int, [vp, P(C.c_double), P(C.c_uint64)]),
    ("pbf_reset_pass_times", C.c_int, [vp]),
    ("pbf_kernel_launches", C.c_int, [vp, P(C.c_uint64)]),
    ("pbf_set_use_graph", C.c_int, [vp, C.c_int]),
    ("pbf_set_option", C.c_int, [vp, C.c_int, C.c_int]),
    ("pbf_list_stats", C.c_int, [vp, P(u32), P(u32), P(u32)]),
    ("pbf_check_finite", C.c_int, [vp, P(u32)]),
    # batched scenes
    ("pbf_batch_create", C.c_int, [P(FluidConfig), vp, u32, C.c_int, P(vp)]),
    ("pbf_batch_destroy", C.c_int, [vp]),
    ("pbf_batch_info", C.c_int, [vp, P(u32), P(u32)]),
    ("pbf_batch_scene_range", C.c_int, [vp, u32, P(u32), P(u32)]),
    ("pbf_batch_set_collision_padding", C.c_int, [vp, C.c_float]),
    ("pbf_batch_set_particles", C.c_int, [vp, u32, vp, u32]),
    ("pbf_batch_read_particles", C.c_int, [vp, u32, vp, u32]),
    ("pbf_batch_set_sdf_grid", C.c_int, [vp, u32, vp, P(i32), P(C.c_float), C.c_float]),
    ("pbf_batch_set_sdf_mode", C.c_int, [vp, u32, C.c_float, u32]),
    ("pbf_batch_clear_sdf", C.c_int, [vp, u32]),
    ("pbf_batch_step", C.c_int, [vp]),
    ("pbf_batch_sync", C.c_int, [vp]),
    ("pbf_batch_get_stream", C.c_int, [vp, P(vp)]),
    ("pbf_batch_device_ptrs", C.c_int, [vp, P(vp), P(vp)]),
    ("pbf_batch_kernel_launches", C.c_int, [vp, P(C.c_uint64)]),
    ("pbf_batch_set_option", C.c_int, [vp, C.c_int, C.c_int]),
    ("pbf_batch_get_option", C.c_int, [vp, C.c_int, P(C.c_int)]),
    ("pbf_batch_autotune", C.c_int, [vp, u32, vp, vp, u32, P(u32)]),
    # host deformation
    ("pbf_deform_default_params", C.c_int, [P(DeformParams)]),
    ("pbf_deform_create", C.c_int, [vp, i32, vp, i32, P(vp)]),
    ("pbf_deform_destroy", C.c_int, [vp]),
    ("pbf_deform_set_mode", C.c_int, [vp, i32, i32, i32]),
    ("pbf_deform_add_anchor", C.c_int, [vp, i32]),
    ("pbf_deform_set_control_points", C.c_int, [vp, vp, vp, i32]),
    ("pbf_deform_precompute", C.c_int, [vp]),
    ("pbf_deform_solve", C.c_int, [vp]),
    ("pbf_deform_vertices", C.c_int, [vp, vp, i32]),
    ("pbf_deform_set_vertices", C.c_int, [vp, vp, i32]),
    ("pbf_deform_step", C.c_int, [vp, vp, i32, C.c_float, P(DeformParams), P(i32), P(i32), P(i32)]),
    ("pbf_deform_patch_size", C.c_int, [vp, P(i32)]),
    ("pbf_deform_verify_incremental", C.c_int, [vp, P(C.c_double)]),
    # scene presets and headless set-up
    ("pbf_scene_count", C.c_int, []),
    ("pbf_scene_get", C.c_int, [i32, P(ScenePreset)]),
    ("pbf_off_load", C.c_int, [C.c_char_p, vp, i32, vp, i32, P(i32), P(i32)]),
    ("pbf_mesh_fit", C.c_int, [vp, i32, P(C.c_float), C.c_double]),
    ("pbf_mesh_fit_center", C.c_int, [P(FluidConfig), P(C.c_float)]),
    ("pbf_mesh_place", C.c_int, [vp, i32, P(C.c_float), P(C.c_float)]),
    ("pbf_spawn_particles", C.c_int, [P(FluidConfig), vp, u32, P(u32)]),
    # differentiable step
    ("pbf_batch_set_sdf_offset", C.c_int, [vp, u32, P(C.c_float)]),
    ("pbf_batch_set_state", C.c_int, [vp, vp, vp]),
    ("pbf_batch_get_state", C.c_int, [vp, vp, vp]),
    ("pbf_batch_forward_record", C.c_int, [vp]),
    ("pbf_batch_backward", C.c_int, [vp, vp, vp, vp, vp, P(C.c_float)]),
]

_lib = None


class PBFError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pbf error {code}: {msg}")
        self.code = code


def lib():
    """Load the in-tree libpbf_b200.so (raises ImportError when it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libpbf_b200.so not built at {LIB_PATH}; run __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != PBF_OK:
        raise PBFError(rc, lib().pbf_last_error().decode(errors="replace"))
    return rc


def fvec(vals):
    return (C.c_float * len(vals))(*[float(v) for v in vals])
