"""ctypes binding to libsdfo_cuda.so (the C ABI declared in include/sdfo.h).

The library is built in-tree (``sdf-contact-module_b200/lib``) by
``__graft_entry__.build()`` or ``python sdf-contact-module_b200/build.py``.
There is no CPU fallback: every entry point raises when the library is
missing or the call fails.
"""
from __future__ import annotations

import ctypes
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libsdfo_cuda.so")

SDFO_OK = 0
SDFO_ERR_IO = -8
FILE_ANY, FILE_DENSE, FILE_SPARSE = 0, 1, 2
FIRST_ORDER, SECOND_ORDER, TRILINEAR, TRICUBIC, CONTACT_AWARE = 0, 1, 2, 3, 4
LAYOUT_DENSE, LAYOUT_SPARSE = 1, 2
STORAGE_FP32, STORAGE_FP16 = 0, 1
BVH_REFERENCE, BVH_LBVH = 0, 1
BE_TANGENT_REFERENCE, BE_TANGENT_EXACT = 0, 1
SIGN_RAY_PARITY, SIGN_PSEUDONORMAL = 0, 1

MODE_NAMES = {"first_order": FIRST_ORDER, "second_order": SECOND_ORDER,
              "trilinear": TRILINEAR, "tricubic": TRICUBIC, "contact_aware": CONTACT_AWARE,
              "FirstOrder": FIRST_ORDER, "SecondOrder": SECOND_ORDER, "Trilinear": TRILINEAR,
              "Tricubic": TRICUBIC, "ContactAware": CONTACT_AWARE}

_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double


class GridInfo(ctypes.Structure):
    _fields_ = [("bmin", _D * 3), ("bmax", _D * 3), ("voxel", _D * 3), ("shape", _I32 * 3),
                ("layout", _I32), ("storage", _I32), ("has_hessian", _I32), ("block_dim", _I32),
                ("halo_voxels", _I32), ("block_count", _I32), ("candidate_stride", _I32),
                ("band_distance", _D)]


class BuildParams(ctypes.Structure):
    _fields_ = [("padding", _D), ("voxel_size", _D), ("target_resolution", _I32),
                ("max_resolution", _I32)]


class SparseBuildParams(ctypes.Structure):
    _fields_ = [("base", BuildParams), ("block_dim", _I32), ("halo_voxels", _I32),
                ("band_voxels", _I32), ("store_hessian", _I32), ("band_distance", _D)]


class ContactAwareParams(ctypes.Structure):
    _fields_ = [("base", BuildParams), ("max_candidates", _I32), ("tile_dim", _I32),
                ("use_tile_acceleration", _I32), ("store_hessian", _I32),
                ("feature_distance_tolerance", _D), ("normal_merge_angle_degrees", _D),
                ("sparse", _I32), ("block_dim", _I32), ("halo_voxels", _I32),
                ("band_voxels", _I32), ("band_distance", _D)]


class MeshDesc(ctypes.Structure):
    _fields_ = [("h_verts", _P), ("nv", _I64), ("h_tris", _P), ("nt", _I64),
                ("params", SparseBuildParams)]


class Pose(ctypes.Structure):
    _fields_ = [("R", _D * 9), ("t", _D * 3)]


class BodyState(ctypes.Structure):
    _fields_ = [("r", _D * 3), ("R", _D * 9), ("v", _D * 3), ("w", _D * 3)]


class ContactParams(ctypes.Structure):
    _fields_ = [("stiffness", _D), ("order", _D), ("damping", _D), ("friction", _D),
                ("regularizer", _D), ("activation_distance", _D)]


class BEParams(ctypes.Structure):
    _fields_ = [("max_iter", _I32), ("line_search", _I32), ("max_toi_bisect_iter", _I32),
                ("stable_steps", _I32), ("release_steps", _I32), ("tangent", _I32),
                ("tol", _D), ("pen_max", _D), ("dt_min", _D), ("dt_impact", _D),
                ("dt_contact", _D), ("dt_max_contact", _D), ("dt_normal", _D), ("dt_growth", _D)]


class RigidBody(ctypes.Structure):
    _fields_ = [("mass", _D), ("inertia", _D * 9), ("gravity", _D * 3)]


class BuildStats(ctypes.Structure):
    _fields_ = [("setup_ms", _D), ("bvh_ms", _D), ("fill_ms", _D), ("hessian_ms", _D),
                ("total_ms", _D), ("voxels_filled", _I64), ("candidate_blocks", _I64),
                ("triangles", _I32), ("bvh_nodes", _I32)]


class TraversalStats(ctypes.Structure):
    _fields_ = [("voxels", _I64), ("nearest_nodes", _I64), ("nearest_triangles", _I64),
                ("ray_nodes", _I64), ("ray_triangles", _I64), ("nearest_triangles_exact", _I64)]


class Tuning(ctypes.Structure):
    _fields_ = [("host_chunk_queries", _I32), ("fill_ctas_per_sm", _I32), ("fill_tile_log2_x", _I32),
                ("fill_tile_log2_y", _I32), ("lbvh_traversal", _I32), ("host_chunk_growth_pct", _I32),
                ("host_io_mode", _I32), ("triangle_cull", _I32),
                ("sparse_pair_records", _I32), ("query_walk", _I32)]


class DeviceViews(ctypes.Structure):
    _fields_ = [("phin", _P), ("hessian6", _P), ("table", _P), ("block_ijk", _P),
                ("stored_voxels", _I64), ("table_dims", _I32 * 3), ("reserved0", _I32)]


# (name, restype, argtypes) of every exported function in include/sdfo.h
SIGNATURES = [
    ("sdfo_version", ctypes.c_char_p, []),
    ("sdfo_abi_version", ctypes.c_int, []),
    ("sdfo_last_error", ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    ("sdfo_device_check", ctypes.c_int, [ctypes.c_int]),
    ("sdfo_build_params_default", None, [ctypes.POINTER(BuildParams)]),
    ("sdfo_sparse_build_params_default", None, [ctypes.POINTER(SparseBuildParams)]),
    ("sdfo_contact_aware_params_default", None, [ctypes.POINTER(ContactAwareParams)]),
    ("sdfo_setup_grid", ctypes.c_int, [_P, _I64, ctypes.POINTER(BuildParams), ctypes.POINTER(GridInfo)]),
    ("sdfo_grid_build_dense", ctypes.c_int,
     [_P, _I64, _P, _I64, ctypes.POINTER(BuildParams), _P, ctypes.POINTER(_P)]),
    ("sdfo_grid_build_sparse", ctypes.c_int,
     [_P, _I64, _P, _I64, ctypes.POINTER(SparseBuildParams), _P, ctypes.POINTER(_P)]),
    ("sdfo_grid_build_contact_aware", ctypes.c_int,
     [_P, _I64, _P, _I64, _P, ctypes.POINTER(ContactAwareParams), _P, ctypes.POINTER(_P)]),
    ("sdfo_grid_build_sparse_batched", ctypes.c_int,
     [ctypes.POINTER(MeshDesc), _I32, _P, ctypes.POINTER(_P)]),
    ("sdfo_set_fill_ctas_per_sm", ctypes.c_int, [_I32]),
    ("sdfo_grid_build_stats", ctypes.c_int, [_P, ctypes.POINTER(BuildStats)]),
    ("sdfo_device_cache", ctypes.c_int, [_I64, _P]),
    ("sdfo_build_traversal_stats", ctypes.c_int,
     [_P, _I64, _P, _I64, _P, _P, ctypes.POINTER(TraversalStats)]),
    ("sdfo_set_bvh_mode", ctypes.c_int, [_I32]),
    ("sdfo_get_bvh_mode", ctypes.c_int, []),
    ("sdfo_set_sign_mode", ctypes.c_int, [_I32]),
    ("sdfo_get_sign_mode", ctypes.c_int, []),
    ("sdfo_grid_create_dense", ctypes.c_int,
     [ctypes.POINTER(GridInfo), _P, _P, _P, _P, _P, ctypes.POINTER(_P)]),
    ("sdfo_grid_create_sparse", ctypes.c_int,
     [ctypes.POINTER(GridInfo), _P, _P, _P, _P, _P, ctypes.POINTER(_P)]),
    ("sdfo_grid_to_fp16", ctypes.c_int, [_P, _P, ctypes.POINTER(_P)]),
    ("sdfo_grid_export_dense", ctypes.c_int, [_P, _P, _P, _P, _P]),
    ("sdfo_grid_export_sparse", ctypes.c_int, [_P, _P, _P, _P, _P]),
    ("sdfo_grid_copy_payload", ctypes.c_int, [_P, _P, _P]),
    ("sdfo_grid_export_candidates", ctypes.c_int, [_P, _P, _P, _P, _P]),
    ("sdfo_grid_attach_candidates", ctypes.c_int, [_P, _I32, _P, _P, _P, _P]),
    ("sdfo_grid_create_view", ctypes.c_int, [_P, _P, ctypes.POINTER(_P)]),
    ("sdfo_grid_get_info", ctypes.c_int, [_P, ctypes.POINTER(GridInfo)]),
    ("sdfo_grid_device_views", ctypes.c_int, [_P, ctypes.POINTER(DeviceViews)]),
    ("sdfo_grid_destroy", ctypes.c_int, [_P]),
    ("sdfo_file_probe", ctypes.c_int, [ctypes.c_char_p, _P, _P]),
    ("sdfo_device_status", ctypes.c_int, [_P, _I32]),
    ("sdfo_debug_wait_test", ctypes.c_int, [ctypes.c_uint32, _I32]),
    ("sdfo_set_tuning", ctypes.c_int, [ctypes.POINTER(Tuning)]),
    ("sdfo_get_tuning", ctypes.c_int, [ctypes.POINTER(Tuning)]),
    ("sdfo_contact_pair_create", ctypes.c_int, [_P, _P, _P, _I64, _I32, _D, _I32, _P]),
    ("sdfo_contact_pair_export_bvh", ctypes.c_int, [_P, _P, _P, _P, _P]),
    ("sdfo_contact_pair_eval", ctypes.c_int, [_P, _I32, _P, _I64, _P, _P, _P, _P, _P, _P]),
    ("sdfo_contact_pair_destroy", ctypes.c_int, [_P]),
    ("sdfo_be_params_default", None, [_P]),
    ("sdfo_be_scene_init", None, [_P, _P, _D, _P]),
    ("sdfo_be_stepper_create", ctypes.c_int, [_P, _P, _P, _P, _P, _I64, _P]),
    ("sdfo_be_stepper_step", ctypes.c_int, [_P, _P, _I64, _P, _P, _P]),
    ("sdfo_be_stepper_set_threads", ctypes.c_int, [_P, _I32]),
    ("sdfo_be_stepper_advance", ctypes.c_int, [_P, _P, _I64, _P, ctypes.c_double, _I32, _P, _P]),
    ("sdfo_be_stepper_integrate", ctypes.c_int,
     [_P, _P, _I64, _P, ctypes.c_double, _I32, _I64, _P, _P, _P]),
    ("sdfo_be_stepper_stats", ctypes.c_int, [_P, _P, _I32]),
    ("sdfo_be_stepper_destroy", ctypes.c_int, [_P]),
    ("sdfo_grid_load_file", ctypes.c_int, [ctypes.c_char_p, _I32, _P, _P]),
    ("sdfo_grid_save_file", ctypes.c_int, [_P, ctypes.c_char_p, _P]),
    ("sdfo_query", ctypes.c_int, [_P, _I32, _P, _I32, _I64, _P, _P, _P, _P, _P, _P, _P]),
    ("sdfo_query_host", ctypes.c_int, [_P, _I32, _P, _I32, _I64, _P, _P, _P, _P, _P, _P]),
    ("sdfo_query_host_static", ctypes.c_int, [_P, _I32, _P, _I32, _I64, _P, _P, _P, _P]),
    ("sdfo_query_backward", ctypes.c_int, [_P, _I32, _P, _I64, _P, _P, _P, _P, _P]),
    ("sdfo_query_candidates", ctypes.c_int,
     [_P, _I32, _P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    ("sdfo_query_candidates_host", ctypes.c_int,
     [_P, _I32, _P, _I32, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    ("sdfo_query_linearize", ctypes.c_int, [_P, _I32, _P, _I64, _P, _P, _P, _P, _P]),
    ("sdfo_query_backward_saved", ctypes.c_int,
     [_P, _I32, _P, _I64, _P, _P, _P, _P, _P, _P, _P, _P]),
    ("sdfo_query_batch_create", ctypes.c_int, [_P, _I32, _P, ctypes.POINTER(_P)]),
    ("sdfo_query_batch_run", ctypes.c_int, [_P, _I32, _P, _P, _P, _P, _P, _P]),
    ("sdfo_query_batch_set_threads", ctypes.c_int, [_P, _I32]),
    ("sdfo_query_batch_set_run", ctypes.c_int, [_P, _I32]),
    ("sdfo_query_batch_total", ctypes.c_int, [_P, ctypes.POINTER(_I64)]),
    ("sdfo_query_batch_destroy", ctypes.c_int, [_P]),
    ("sdfo_contact_eval", ctypes.c_int,
     [_P, _I32, _P, _P, _I64, _P, _I64, _P, ctypes.POINTER(ContactParams), _P, _P, _P]),
]

_lib = None


class SdfoError(RuntimeError):
    """A libsdfo_cuda call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[sdfo {code}] {msg}")
        self.code = code


def library_path() -> str:
    return LIB_PATH


def load(path: str | None = None):
    """Loads libsdfo_cuda.so (raises FileNotFoundError when it is not built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(
            f"libsdfo_cuda.so not found at {p}; build it with "
            "`python sdf-contact-module_b200/build.py` (no CPU fallback exists)")
    lib = ctypes.CDLL(p)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    load().sdfo_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(code: int) -> None:
    if code != SDFO_OK:
        raise SdfoError(code, last_error())


def get_tuning() -> dict:
    """The process-wide tuning knobs (sdfo_get_tuning) as a dict."""
    t = Tuning()
    check(load().sdfo_get_tuning(ctypes.byref(t)))
    return {name: int(getattr(t, name)) for name, _ in Tuning._fields_}


def set_tuning(**fields) -> dict:
    """Sets the named tuning knobs (others keep their values); returns the
    resulting settings."""
    cur = get_tuning()
    unknown = set(fields) - set(cur)
    if unknown:
        raise ValueError(f"unknown tuning fields {sorted(unknown)}")
    cur.update({k: int(v) for k, v in fields.items()})
    check(load().sdfo_set_tuning(ctypes.byref(Tuning(**cur))))
    return get_tuning()


def mode_id(mode) -> int:
    if isinstance(mode, str):
        if mode not in MODE_NAMES:
            raise ValueError(f"unknown query mode {mode!r}")
        return MODE_NAMES[mode]
    m = int(mode)
    if m < 0 or m > 4:
        raise ValueError(f"unknown query mode {mode!r}")
    return m
