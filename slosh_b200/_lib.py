"""ctypes binding of ``libslosh_b200.so`` and numpy dtypes of its records.

The shared library is built in-tree (``slosh_b200/lib/libslosh_b200.so``) by
:func:`slosh_b200.build.build_library`.  Loading fails loudly when it is
missing: there is no CPU fallback for the substep.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libslosh_b200.so")

# Status codes (include/slosh_b200.h).
SLOSH_OK = 0
SLOSH_E_INVALID = -1
SLOSH_E_CUDA = -2
SLOSH_E_OVERFLOW = -3
SLOSH_E_CAPACITY = -4
SLOSH_E_NOMEM = -5
SLOSH_E_STATE = -6
SLOSH_E_MATERIAL = -7
SLOSH_E_TIMEOUT = -8

STATUS_NAMES = {
    SLOSH_E_INVALID: "SLOSH_E_INVALID",
    SLOSH_E_CUDA: "SLOSH_E_CUDA",
    SLOSH_E_OVERFLOW: "SLOSH_E_OVERFLOW",
    SLOSH_E_CAPACITY: "SLOSH_E_CAPACITY",
    SLOSH_E_NOMEM: "SLOSH_E_NOMEM",
    SLOSH_E_STATE: "SLOSH_E_STATE",
    SLOSH_E_MATERIAL: "SLOSH_E_MATERIAL",
    SLOSH_E_TIMEOUT: "SLOSH_E_TIMEOUT",
}

# Particle model tags (GpuParticleModel discriminants + the Tait fluid).
MODEL_ELASTIC_LINEAR = 0
MODEL_ELASTIC_NEO_HOOKEAN = 1
MODEL_SAND_LINEAR = 2
MODEL_SAND_NEO_HOOKEAN = 3
MODEL_FLUID_TAIT = 4

SHAPE_BALL = 0
SHAPE_CUBOID = 1
SHAPE_CAPSULE = 2
SHAPE_CONE = 3
SHAPE_CYLINDER = 4
SHAPE_TRIMESH = 6

COUPLING_ONE_WAY = 0
COUPLING_TWO_WAY = 1
BC_STICK = 0
BC_SLIP = 1
BC_SEPARATE = 2
BC_FRICTION_Z_UP = 3
BC_NON_REFLECTING = 4
BC_DISABLED = 5

# slosh_particle: 192 bytes.
PARTICLE_DTYPE = np.dtype(
    [
        ("position", "<f4", 3),
        ("velocity", "<f4", 3),
        ("def_grad", "<f4", 9),  # column-major
        ("affine", "<f4", 9),  # column-major
        ("force_dt", "<f4", 3),
        ("vel_grad_det", "<f4"),
        ("init_volume", "<f4"),
        ("init_radius", "<f4"),
        ("mass", "<f4"),
        ("damping", "<f4"),
        ("phase", "<f4"),
        ("enabled", "<u4"),
        ("fixed", "<u4"),
        ("model_tag", "<u4"),
        ("model", "<f4", 12),
    ]
)
assert PARTICLE_DTYPE.itemsize == 192

# slosh_body: 192 bytes.
BODY_DTYPE = np.dtype(
    [
        ("shape_a", "<f4", 4),
        ("shape_b", "<f4", 4),
        ("rotation", "<f4", 4),
        ("translation", "<f4", 4),
        ("linvel", "<f4", 4),
        ("angvel", "<f4", 4),
        ("inv_mass", "<f4", 4),
        ("local_com", "<f4", 4),
        ("inv_inertia", "<f4", 12),
        ("bc_type", "<u4"),
        ("bc_friction", "<f4"),
        ("coupling", "<u4"),
        ("pad", "<u4"),
    ]
)
assert BODY_DTYPE.itemsize == 192


class SloshConfig(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_uint32),
        ("cell_width", ctypes.c_float),
        ("grid_capacity", ctypes.c_uint32),
        ("max_particles", ctypes.c_uint32),
        ("device", ctypes.c_int32),
        ("flags", ctypes.c_uint32),
    ]


class SloshParams(ctypes.Structure):
    _fields_ = [("gravity", ctypes.c_float * 3), ("dt", ctypes.c_float)]


class SloshGridDump(ctypes.Structure):
    _fields_ = [
        ("n_blocks", ctypes.c_uint32),
        ("n_sorted", ctypes.c_uint32),
        ("nb_buckets", ctypes.c_uint32),
        ("n_neighbors", ctypes.c_uint32),
        ("keys", ctypes.c_void_p),
        ("first_particle", ctypes.c_void_p),
        ("num_particles", ctypes.c_void_p),
        ("num_particles_with_extras", ctypes.c_void_p),
        ("bucket_counts", ctypes.c_void_p),
        ("sorted_ids", ctypes.c_void_p),
        ("primary_first", ctypes.c_void_p),
        ("primary_perm", ctypes.c_void_p),
        ("neighbors", ctypes.c_void_p),
    ]


class SloshBatchConfig(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32),
        ("max_particles", ctypes.c_uint32),
        ("grid_capacity", ctypes.c_uint32),
        ("max_scenes", ctypes.c_uint32),
        ("max_bodies", ctypes.c_uint32),
        ("device", ctypes.c_int32),
        ("flags", ctypes.c_uint32),
    ]


class SloshSceneDesc(ctypes.Structure):
    _fields_ = [("cell_width", ctypes.c_float), ("params", SloshParams)]


class SloshTuning(ctypes.Structure):
    _fields_ = [
        ("p2g_ctas_per_sm", ctypes.c_uint32),
        ("g2p_threads", ctypes.c_uint32),
        ("g2p_ctas_per_sm", ctypes.c_uint32),
        ("p2g_stages", ctypes.c_uint32),
        ("fused", ctypes.c_uint32),
    ]


class SloshBatchStats(ctypes.Structure):
    _fields_ = [
        ("live_scenes", ctypes.c_uint32),
        ("n_particles", ctypes.c_uint32),
        ("n_blocks", ctypes.c_uint32),
        ("n_materials", ctypes.c_uint32),
        ("n_svd_fp64", ctypes.c_uint32),
        ("n_bodies", ctypes.c_uint32),
        ("fused_graph", ctypes.c_uint32),
        ("g2p_launches", ctypes.c_uint32),
        ("tuning", SloshTuning),
    ]


class SloshServerConfig(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("hbm_budget_bytes", ctypes.c_uint64),
        ("max_scenes", ctypes.c_uint32),
        ("max_bodies", ctypes.c_uint32),
        ("tick_substeps", ctypes.c_uint32),
        ("max_in_flight", ctypes.c_uint32),
        ("autotune", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
    ]


class SloshRequest(ctypes.Structure):
    _fields_ = [
        ("desc", SloshSceneDesc),
        ("n", ctypes.c_uint32),
        ("n_bodies", ctypes.c_uint32),
        ("substeps", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
        ("particles", ctypes.c_void_p),
        ("bodies", ctypes.c_void_p),
        ("out_positions", ctypes.c_void_p),
    ]


class SloshCompletion(ctypes.Structure):
    _fields_ = [
        ("id", ctypes.c_uint64),
        ("status", ctypes.c_int32),
        ("n", ctypes.c_uint32),
        ("substeps", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
        ("submit_s", ctypes.c_double),
        ("admit_s", ctypes.c_double),
        ("done_s", ctypes.c_double),
    ]


class SloshServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_uint64),
        ("admitted", ctypes.c_uint64),
        ("completed", ctypes.c_uint64),
        ("particle_substeps", ctypes.c_uint64),
        ("in_flight_bytes", ctypes.c_uint64),
        ("pool_bytes", ctypes.c_uint64),
        ("busy_s", ctypes.c_double),
        ("now_s", ctypes.c_double),
        ("in_flight", ctypes.c_uint32),
        ("queued", ctypes.c_uint32),
        ("max_in_flight_seen", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
        ("tuning", SloshTuning),
    ]


# Stage hooks (slosh's MpmPipelineHooks points).
HOOK_AFTER_PARTICLE_SORT = 0
HOOK_RUN_P2G = 1
HOOK_AFTER_P2G = 2
HOOK_AFTER_GRID_UPDATE = 3
HOOK_RUN_G2P = 4
HOOK_AFTER_G2P = 5
HOOK_AFTER_PARTICLES_UPDATE = 6
HOOK_NAMES = (
    "after_particle_sort",
    "run_p2g",
    "after_p2g",
    "after_grid_update",
    "run_g2p",
    "after_g2p",
    "after_particles_update",
)
HOOK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p)


class SloshDeviceView(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_uint32),
        ("n_particles", ctypes.c_uint32),
        ("capacity", ctypes.c_uint32),
        ("grid_capacity", ctypes.c_uint32),
        ("cell_width", ctypes.c_float),
        ("dt", ctypes.c_float),
        ("pad", ctypes.c_uint32 * 2),
        ("n_blocks", ctypes.c_void_p),
        ("block_keys", ctypes.c_void_p),
        ("block_first", ctypes.c_void_p),
        ("block_count", ctypes.c_void_p),
        ("perm", ctypes.c_void_p),
        ("x_mass", ctypes.c_void_p),
        ("vel", ctypes.c_void_p),
        ("affine", ctypes.c_void_p),
        ("def_grad", ctypes.c_void_p),
        ("flags", ctypes.c_void_p),
        ("plastic", ctypes.c_void_p),
        ("out_x_mass", ctypes.c_void_p),
        ("out_vel", ctypes.c_void_p),
        ("out_affine", ctypes.c_void_p),
        ("out_def_grad", ctypes.c_void_p),
        ("out_flags", ctypes.c_void_p),
        ("out_plastic", ctypes.c_void_p),
        ("nodes", ctypes.c_void_p),
    ]


# Every symbol include/slosh_b200.h declares, with its ctypes signature.
_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
SIGNATURES = {
    "slosh_ctx_create": (ctypes.c_int, [ctypes.POINTER(SloshConfig), ctypes.POINTER(_P)]),
    "slosh_ctx_destroy": (None, [_P]),
    "slosh_set_params": (ctypes.c_int, [_P, ctypes.POINTER(SloshParams)]),
    "slosh_upload_particles": (ctypes.c_int, [_P, _P, _U32, _P]),
    "slosh_append_particles": (ctypes.c_int, [_P, _P, _U32, _P]),
    "slosh_remove_particles": (ctypes.c_int, [_P, _U32, _U32, ctypes.POINTER(_U32), _P]),
    "slosh_download_particles": (ctypes.c_int, [_P, _P, _U32, _P]),
    "slosh_download_positions": (ctypes.c_int, [_P, _P, _U32, _P]),
    "slosh_set_bodies": (ctypes.c_int, [_P, _P, _U32]),
    "slosh_get_bodies": (ctypes.c_int, [_P, _P, _U32]),
    "slosh_add_trimesh": (ctypes.c_int, [_P, _P, _U32, _P, _U32, _P]),
    "slosh_step": (ctypes.c_int, [_P, _U32, _P]),
    "slosh_sync": (ctypes.c_int, [_P, _P]),
    "slosh_set_hook": (ctypes.c_int, [_P, _U32, HOOK_FN, _P]),
    "slosh_enqueue_builtin": (ctypes.c_int, [_P, _U32, _P]),
    "slosh_device_view_get": (ctypes.c_int, [_P, ctypes.POINTER(SloshDeviceView)]),
    "slosh_kernels_per_substep": (_U32, [_P]),
    "slosh_profile_substeps": (ctypes.c_int, [_P, _U32, _P, _P, _U32, ctypes.POINTER(_U32)]),
    "slosh_kernel_name": (ctypes.c_int, [_U32, ctypes.c_char_p, ctypes.c_size_t]),
    "slosh_get_stats": (ctypes.c_int, [_P, _P]),
    "slosh_grid_debug": (ctypes.c_int, [_P, ctypes.POINTER(SloshGridDump), _U32, _U32]),
    "slosh_debug_nodes": (ctypes.c_int, [_P, ctypes.c_int, _P, _U32, ctypes.POINTER(_U32)]),
    "slosh_prefix_sum": (ctypes.c_int, [_P, _P, _P, _U32]),
    "slosh_prefix_sum_noalloc": (ctypes.c_int, [_P, _P, _U32, _P]),
    "slosh_timestep_bound": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_float), _P]),
    "slosh_last_error": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_size_t]),
    "slosh_batch_create": (ctypes.c_int, [ctypes.POINTER(SloshBatchConfig), ctypes.POINTER(_P)]),
    "slosh_batch_destroy": (None, [_P]),
    "slosh_batch_add_scene": (
        ctypes.c_int,
        [_P, ctypes.POINTER(SloshSceneDesc), _P, _U32, _P, _U32, ctypes.POINTER(_U32), _P],
    ),
    "slosh_batch_remove_scene": (ctypes.c_int, [_P, _U32]),
    "slosh_batch_step": (ctypes.c_int, [_P, _U32, _P]),
    "slosh_batch_download_particles": (ctypes.c_int, [_P, _U32, _P, _U32, _P]),
    "slosh_batch_download_positions": (ctypes.c_int, [_P, _U32, _P, _U32, _P]),
    "slosh_batch_get_bodies": (ctypes.c_int, [_P, _U32, _P, _U32]),
    "slosh_batch_timestep_bound": (ctypes.c_int, [_P, _U32, ctypes.POINTER(ctypes.c_float), _P]),
    "slosh_batch_sync": (ctypes.c_int, [_P, _P]),
    "slosh_batch_get_stats": (ctypes.c_int, [_P, ctypes.POINTER(SloshBatchStats)]),
    "slosh_batch_autotune": (ctypes.c_int, [_P, _U32, _P]),
    "slosh_batch_set_tuning": (ctypes.c_int, [_P, ctypes.POINTER(SloshTuning)]),
    "slosh_batch_last_error": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_size_t]),
    "slosh_server_create": (ctypes.c_int, [ctypes.POINTER(SloshServerConfig), ctypes.POINTER(_P)]),
    "slosh_server_destroy": (None, [_P]),
    "slosh_server_submit": (ctypes.c_int, [_P, ctypes.POINTER(SloshRequest), ctypes.POINTER(ctypes.c_uint64)]),
    "slosh_server_poll": (ctypes.c_int, [_P, _P, _U32, ctypes.POINTER(_U32)]),
    "slosh_server_wait_idle": (ctypes.c_int, [_P, ctypes.c_double]),
    "slosh_server_get_stats": (ctypes.c_int, [_P, ctypes.POINTER(SloshServerStats)]),
    "slosh_server_last_error": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_size_t]),
}

_lib = None


def load() -> ctypes.CDLL:
    """Loads the CUDA library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with slosh_b200.build.build_library() "
            "(nvcc, sm_100a). The MPM substep has no CPU fallback."
        )
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class SloshError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


def ptr(a: np.ndarray | None) -> ctypes.c_void_p | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(a.ctypes.data)
