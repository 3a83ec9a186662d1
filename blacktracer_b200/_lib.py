"""ctypes bindings of libblacktracer_b200.so (the C ABI in include/blacktracer.h).

The library is the only compute path: if it is missing or fails to load,
every entry point raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libblacktracer_b200.so")

BT_OK, BT_ERR_ARG, BT_ERR_CUDA, BT_ERR_NOMEM, BT_ERR_NUMERIC, BT_ERR_STATE = range(6)
RAY_ESCAPED, RAY_CAPTURED, RAY_MAXSTEP, RAY_NONCONVERGED = range(4)
PRECISION_PLAIN, PRECISION_MIXED, PRECISION_FAST = 0, 1, 2


class BtError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"blacktracer error {code}: {msg}")
        self.code = code


class bt_camera(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "theta", "phi", "r", "speed", "br", "btheta", "bphi",
        "alpha", "w", "wbar", "Delta", "ro")]


class bt_integ_opts(C.Structure):
    _fields_ = [("eps", C.c_double), ("h1", C.c_double), ("z_end", C.c_double),
                ("maxstp", C.c_int32), ("precision", C.c_int32),
                ("fp64_band", C.c_double)]


class bt_grid_info(C.Structure):
    _fields_ = [("N", C.c_int32), ("M", C.c_int32), ("maxlevel", C.c_int32),
                ("startlevel", C.c_int32), ("angle", C.c_int32),
                ("traced", C.c_int64), ("n_leaf_blocks", C.c_int64),
                ("flags", C.c_uint32),
                ("thphi", C.c_void_p), ("steps", C.c_void_p), ("exists", C.c_void_p),
                ("blevel", C.c_void_p), ("status", C.c_void_p),
                ("trace_ms", C.c_float), ("trace_launches", C.c_int32),
                ("launches", C.c_int32)]


class bt_grid_export_t(C.Structure):
    _fields_ = [("vi", C.c_void_p), ("vj", C.c_void_p), ("theta", C.c_void_p),
                ("phi", C.c_void_p), ("steps", C.c_void_p), ("cap_vertices", C.c_size_t),
                ("bi", C.c_void_p), ("bj", C.c_void_p), ("level", C.c_void_p),
                ("cap_blocks", C.c_size_t), ("n_vertices", C.c_size_t),
                ("n_blocks", C.c_size_t)]


class bt_trace_shape(C.Structure):
    _fields_ = [("threads", C.c_int32), ("blocks_per_sm", C.c_int32), ("refill", C.c_int32)]


class bt_tune_result(C.Structure):
    _fields_ = [("shape", bt_trace_shape), ("flow", C.c_int32), ("band_met", C.c_int32),
                ("fp64_band", C.c_double), ("band_p99_rad", C.c_double),
                ("best_ms", C.c_float), ("level_ms", C.c_float), ("flow_ms", C.c_float),
                ("candidates", C.c_int32)]


class bt_batch_info(C.Structure):
    _fields_ = [("count", C.c_int32), ("traced", C.c_int64), ("flags", C.c_uint32),
                ("trace_ms", C.c_float), ("trace_launches", C.c_int32),
                ("launches", C.c_int32), ("graph", C.c_int32), ("shape", bt_trace_shape)]


class bt_server_config(C.Structure):
    _fields_ = [("maxlevel", C.c_int32), ("startlevel", C.c_int32), ("angle", C.c_int32),
                ("precision", C.c_int32), ("grid_cache_bytes", C.c_size_t),
                ("render_bytes", C.c_size_t), ("max_inflight", C.c_int32),
                ("max_build_batch", C.c_int32), ("env", C.c_void_p), ("stars", C.c_void_p),
                ("step", C.c_int32), ("lr", C.c_int32)]


class bt_request(C.Structure):
    _fields_ = [("id", C.c_uint64), ("width", C.c_int32), ("height", C.c_int32),
                ("cam", bt_camera), ("a", C.c_double), ("out", C.c_void_p)]


class bt_completion(C.Structure):
    _fields_ = [("id", C.c_uint64), ("status", C.c_int32), ("grid_reused", C.c_int32),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double)]


class bt_server_stats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "submitted", "completed", "failed", "grid_hits", "grid_misses", "grids_built",
        "build_sets", "evictions", "grids_resident")] + [
        ("grid_cache_bytes_used", C.c_size_t), ("render_bytes_used", C.c_size_t)]


class bt_frame(C.Structure):
    _fields_ = [("grid", C.c_void_p), ("grid_rows", C.c_int32), ("grid_cols", C.c_int32),
                ("grid_level", C.c_int32), ("view", C.c_void_p), ("hor", C.c_float),
                ("ver", C.c_float), ("cam", C.c_float * 7), ("env", C.c_void_p),
                ("stars", C.c_void_p), ("map", C.c_int32), ("star", C.c_int32),
                ("lr", C.c_int32), ("step", C.c_int32), ("diffraction", C.c_int32),
                ("out", C.c_void_p), ("bb_table", C.c_int32), ("psf_scale", C.c_int32),
                ("grid2", C.c_void_p), ("alpha", C.c_float), ("cam2", C.c_float * 7),
                ("blend", C.c_void_p), ("trails", C.c_void_p)]


class bt_map_census_t(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("env_columns", "env_pixels", "star_pixels",
                                          "star_candidates_ref", "star_candidates",
                                          "star_hits", "heavy_candidates", "heavy_hits")]


class bt_trails_info(C.Structure):
    _fields_ = [("frame", C.c_int64), ("hits", C.c_uint32), ("dropped", C.c_uint32),
                ("walks_cut", C.c_uint32), ("trail", C.c_void_p)]


class bt_psh(C.Structure):
    _fields_ = [("hash_table", C.c_void_p), ("pos_tag", C.c_void_p),
                ("offset_table", C.c_void_p), ("cap_hash", C.c_size_t),
                ("cap_offset", C.c_size_t), ("hash_width", C.c_int32),
                ("offset_width", C.c_int32)]


class bt_map_buffers(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("thphi", "gap", "bh", "area", "light",
                                          "stars_img", "env_img", "light_diffracted")]


_vp = C.c_void_p
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_SIGS = {
    "bt_camera_static": (C.c_int, [C.c_double] * 5 + [C.POINTER(bt_camera)]),
    "bt_camera_orbit": (C.c_int, [C.c_double] * 7 + [C.POINTER(bt_camera)]),
    "bt_camera_params": (C.c_int, [C.POINTER(bt_camera), C.POINTER(C.c_float)]),
    "bt_integ_opts_default": (None, [C.POINTER(bt_integ_opts)]),
    "bt_integrate_rays": (C.c_int, [C.POINTER(bt_camera), C.c_double, _vp, _vp, C.c_size_t,
                                    _vp, _vp, _vp, _vp, C.POINTER(bt_integ_opts), _vp]),
    "bt_integrate_rays_host": (C.c_int, [C.POINTER(bt_camera), C.c_double, _vp, _vp,
                                         C.c_size_t, _vp, _vp, _vp, _vp,
                                         C.POINTER(bt_integ_opts), _vp]),
    "bt_integrate_rays_host_static": (C.c_int, [C.POINTER(bt_camera), C.c_double, _vp, _vp,
                                                C.c_size_t, _vp, _vp, _vp, _vp,
                                                C.POINTER(bt_integ_opts), _vp]),
    "bt_integrate_rays_host_static_capacity": (C.c_size_t, []),
    "bt_grid_dims": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "bt_grid_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(_vp)]),
    "bt_grid_destroy": (None, [_vp]),
    "bt_grid_build": (C.c_int, [_vp, C.POINTER(bt_camera), C.c_double, C.c_int,
                                C.POINTER(bt_integ_opts), _vp]),
    "bt_grid_query": (C.c_int, [_vp, C.POINTER(bt_grid_info), _vp]),
    "bt_grid_export_dense": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bt_grid_map_export": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32), C.POINTER(C.c_int32), _vp]),
    "bt_grid_export": (C.c_int, [_vp, C.POINTER(bt_grid_export_t), _vp]),
    "bt_grid_set_timing": (C.c_int, [_vp, C.c_int]),
    "bt_grid_set_graph": (C.c_int, [_vp, C.c_int]),
    "bt_grid_set_tfix_passes": (C.c_int, [_vp, C.c_int]),
    "bt_grid_set_tfix_launch": (C.c_int, [_vp, C.c_int]),
    "bt_grid_set_flow_drop": (C.c_int, [_vp]),
    "bt_grid_set_flow": (C.c_int, [_vp, C.c_int]),
    "bt_batch_set_flow": (C.c_int, [_vp, C.c_int]),
    "bt_batch_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(_vp)]),
    "bt_batch_destroy": (None, [_vp]),
    "bt_batch_build": (C.c_int, [_vp, C.POINTER(bt_camera), C.POINTER(C.c_double), C.c_int,
                                 C.POINTER(bt_integ_opts), _vp]),
    "bt_batch_grid": (_vp, [_vp, C.c_int]),
    "bt_batch_set_graph": (C.c_int, [_vp, C.c_int]),
    "bt_batch_set_timing": (C.c_int, [_vp, C.c_int]),
    "bt_batch_set_shape": (C.c_int, [_vp, C.POINTER(bt_trace_shape)]),
    "bt_batch_query": (C.c_int, [_vp, C.POINTER(bt_batch_info), _vp]),
    "bt_batch_autotune": (C.c_int, [_vp, C.POINTER(bt_camera), C.POINTER(C.c_double), C.c_int,
                                    C.POINTER(bt_integ_opts), C.c_int,
                                    C.POINTER(bt_trace_shape), C.POINTER(C.c_float), _vp]),
    "bt_batch_tune": (C.c_int, [_vp, C.POINTER(bt_camera), C.POINTER(C.c_double), C.c_int,
                                C.POINTER(bt_integ_opts), C.c_double, C.c_int,
                                C.POINTER(bt_tune_result), _vp]),
    "bt_grid_set_shape": (C.c_int, [_vp, C.POINTER(bt_trace_shape)]),
    "bt_grid_tune": (C.c_int, [_vp, C.POINTER(bt_integ_opts), C.c_double, C.c_int,
                               C.POINTER(bt_tune_result), _vp]),
    "bt_probe_fp64_tflops": (C.c_int, [C.POINTER(C.c_double), _vp]),
    "bt_view_sphere": (C.c_int, [_vp, C.c_int, C.c_int, _vp]),
    "bt_env_create": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.POINTER(_vp), _vp]),
    "bt_env_destroy": (None, [_vp]),
    "bt_env_sat": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "bt_stars_tree_size": (C.c_int, [C.c_int]),
    "bt_psf_airy": (C.c_int, [C.c_int, C.c_float, _vp]),
    "bt_psf_levels": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp, C.c_int,
                                C.POINTER(C.c_int)]),
    "bt_stars_blackbody": (C.c_int, [_vp, C.c_int, _vp, _vp, C.c_int, C.POINTER(C.c_int), _vp]),
    "bt_map_diffract": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "bt_map_set_star_capacity": (C.c_int, [_vp, C.c_size_t, C.c_size_t]),
    "bt_map_set_star_slab": (C.c_int, [_vp, C.c_int]),
    "bt_blend_create": (C.c_int, [C.POINTER(_vp)]),
    "bt_blend_destroy": (None, [_vp]),
    "bt_blend_prepare": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, _vp]),
    "bt_blend_info": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(C.c_int32),
                                C.POINTER(C.c_uint32)]),
    "bt_stars_build_tree": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_float,
                                      _vp, _vp, _vp, C.POINTER(C.c_int)]),
    "bt_stars_create": (C.c_int, [_vp, _vp, C.c_int, _vp, C.c_int, _vp, C.c_int,
                                  C.POINTER(_vp), _vp]),
    "bt_stars_destroy": (None, [_vp]),
    "bt_map_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(_vp)]),
    "bt_map_destroy": (None, [_vp]),
    "bt_map_render": (C.c_int, [_vp, C.POINTER(bt_frame), _vp]),
    "bt_map_scratch": (C.c_int, [_vp, C.POINTER(bt_map_buffers)]),
    "bt_batch_build_first": (C.c_int, [_vp, C.c_int, C.POINTER(bt_camera),
                                       C.POINTER(C.c_double), C.c_int,
                                       C.POINTER(bt_integ_opts), _vp]),
    "bt_server_config_default": (None, [C.POINTER(bt_server_config)]),
    "bt_server_create": (C.c_int, [C.POINTER(bt_server_config), C.POINTER(_vp)]),
    "bt_server_submit": (C.c_int, [_vp, C.POINTER(bt_request)]),
    "bt_server_poll": (C.c_int, [_vp, C.POINTER(bt_completion), C.c_int,
                                 C.POINTER(C.c_int), C.c_int]),
    "bt_server_stats_get": (C.c_int, [_vp, C.POINTER(bt_server_stats)]),
    "bt_server_destroy": (None, [_vp]),
    "bt_psh_build": (C.c_int, [_vp, _vp, C.c_size_t, C.POINTER(bt_psh)]),
    "bt_grid_map_from_psh": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                       _vp, C.c_int, _vp]),
    "bt_grid_file_write": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int,
                                     C.POINTER(bt_psh)]),
    "bt_grid_file_read": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                    C.POINTER(C.c_int32), C.POINTER(bt_psh)]),
    "bt_grid_save": (C.c_int, [_vp, C.c_char_p, _vp]),
    "bt_grid_file_map_shape": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32),
                                         C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                         C.POINTER(C.c_int32)]),
    "bt_grid_file_load_map": (C.c_int, [C.c_char_p, _vp, C.c_int, C.c_int, _vp]),
    "bt_stars_file_write": (C.c_int, [C.c_char_p, _vp, _vp, C.c_int, _vp, C.c_int]),
    "bt_stars_file_info": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "bt_stars_file_read": (C.c_int, [C.c_char_p, _vp, _vp, C.c_int, _vp, C.c_int]),
    "bt_view_camera": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                 _vp]),
    "bt_trails_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_size_t,
                                   C.POINTER(_vp)]),
    "bt_trails_destroy": (None, [_vp]),
    "bt_trails_reset": (C.c_int, [_vp]),
    "bt_trails_query": (C.c_int, [_vp, C.POINTER(bt_trails_info), _vp]),
    "bt_map_census": (C.c_int, [_vp, C.POINTER(bt_frame), C.POINTER(bt_map_census_t), _vp]),
    "bt_probe_fast_rcp": (C.c_int, [_vp, _vp, C.c_size_t, _vp]),
    "bt_last_error": (C.c_char_p, []),
    "bt_version": (C.c_char_p, []),
}

_lib = None


def lib():
    """Loads the CUDA library (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m blacktracer_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def check(rc: int) -> None:
    if rc != BT_OK:
        raise BtError(rc, lib().bt_last_error().decode(errors="replace"))
