"""ctypes binding of the C ABI in include/simtrack_b200.h.

The shared library is built in-tree (simtrack_b200/_lib/libsimtrack_b200.so,
see simtrack_b200/build.py).  There is no fallback: if the library is missing
or a CUDA call fails, the error surfaces as SimTrackError.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_long, c_ulonglong, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libsimtrack_b200.so"

STB_OK = 0
STB_EINVAL = -1
STB_ENOMEM = -2
STB_ECUDA = -3
STB_ETIMEOUT = -4
STB_EABORTED = -5
STB_EUNSUPPORTED = -6

_CODES = {STB_EINVAL: "EINVAL", STB_ENOMEM: "ENOMEM", STB_ECUDA: "ECUDA", STB_ETIMEOUT: "ETIMEOUT",
          STB_EABORTED: "EABORTED", STB_EUNSUPPORTED: "EUNSUPPORTED"}


class SimTrackError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_CODES.get(code, code)}: {msg}")
        self.code = code


# (name, restype, argtypes) for every exported entry point.
SIGNATURES = [
    ("stb_last_error", c_char_p, []),
    ("stb_version", c_int, []),
    ("stb_set_ref_energy", c_int, [c_double, c_double, c_double, c_double]),
    ("stb_set_spin_g", c_int, [c_double]),
    ("stb_set_flags", c_int, [c_int, c_int]),
    ("stb_set_radiation", c_int, [c_int, c_ulonglong]),
    ("stb_cal_srloss_u0rad", c_int, [c_void_p, c_int, POINTER(c_double)]),
    ("stb_cal_srloss_particle", c_int, [c_void_p, POINTER(c_double), POINTER(c_double), c_int]),
    ("stb_get_ref", c_int, [POINTER(c_double)]),
    ("stb_element_new", c_int, [c_char_p, c_char_p, POINTER(c_double), c_int, POINTER(c_void_p)]),
    ("stb_element_free", c_int, [c_void_p]),
    ("stb_element_setp", c_int, [c_void_p, c_char_p, c_double]),
    ("stb_element_getp", c_int, [c_void_p, c_char_p, POINTER(c_double)]),
    ("stb_element_set_misalign", c_int, [c_void_p] + [c_double] * 6),
    ("stb_element_set_aperture", c_int, [c_void_p, c_double, c_double]),
    ("stb_element_type", c_int, [c_void_p, c_char_p, c_int]),
    ("stb_line_new", c_int, [POINTER(c_void_p)]),
    ("stb_line_free", c_int, [c_void_p]),
    ("stb_line_append", c_int, [c_void_p, c_void_p]),
    ("stb_line_insert", c_int, [c_void_p, c_long, c_void_p]),
    ("stb_line_delete", c_int, [c_void_p, c_long]),
    ("stb_line_replace", c_int, [c_void_p, c_long, c_void_p]),
    ("stb_line_rewind", c_int, [c_void_p, c_long]),
    ("stb_line_invert", c_int, [c_void_p]),
    ("stb_line_ncell", c_long, [c_void_p]),
    ("stb_line_length", c_double, [c_void_p]),
    ("stb_line_cell", c_int, [c_void_p, c_long, POINTER(c_void_p)]),
    ("stb_table_create", c_int, [c_void_p, c_int, POINTER(c_void_p)]),
    ("stb_table_free", c_int, [c_void_p]),
    ("stb_table_info", c_int, [c_void_p, POINTER(c_double)]),
    ("stb_table_autotune", c_int, [c_void_p] + [c_void_p] * 6 + [c_long, c_int, c_double, POINTER(c_int),
                                                                  POINTER(c_double), c_int]),
    ("stb_table_set_variant", c_int, [c_void_p, c_int]),
    ("stb_track_variant_info", c_int, [c_int, c_char_p, c_int, POINTER(c_int), POINTER(c_int)]),
    ("stb_track_device", c_int, [c_void_p] + [c_void_p] * 6 + [c_long, c_int, c_int, c_double, c_void_p,
                                                                c_void_p, c_void_p]),
    ("stb_track_host", c_int, [c_void_p, POINTER(c_double), c_long, c_int, c_double, POINTER(c_int),
                               POINTER(c_int), POINTER(c_int)]),
    ("stb_scan_create", c_int, [POINTER(c_void_p), c_int, POINTER(c_double), POINTER(c_long), c_double, c_int,
                                POINTER(c_void_p)]),
    ("stb_scan_free", c_int, [c_void_p]),
    ("stb_scan_configure", c_int, [c_void_p, c_int, c_int]),
    ("stb_scan_run", c_int, [c_void_p, c_int, c_int, c_int]),
    ("stb_scan_results", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("stb_scan_stats", c_int, [c_void_p, POINTER(c_double)]),
    ("stb_scan_autotune", c_int, [c_void_p, c_int, POINTER(c_int), POINTER(c_double), c_int]),
    ("stb_scan_set_tbt", c_int, [c_void_p, c_void_p, c_int]),
    ("stb_table_create_spin", c_int, [c_void_p, c_int, POINTER(c_void_p)]),
    ("stb_element_name", c_int, [c_void_p, c_char_p, c_int]),
    ("stb_element_geometry", c_int, [c_void_p, POINTER(c_double)]),
    ("stb_line_read_madx", c_int, [c_void_p, c_char_p]),
    ("stb_line_read_bmad", c_int, [c_void_p, c_char_p]),
    ("stb_track_da_driver", c_int, [c_void_p, c_int, c_int, c_double, c_double, c_double, c_double, c_char_p,
                                    POINTER(c_double), POINTER(c_double), POINTER(c_long), c_int]),
    ("stb_cal_tunes_track", c_int, [c_void_p, POINTER(c_double), c_int, c_double, c_double, POINTER(c_double),
                                    POINTER(c_int), c_int]),
    ("stb_cal_tunes_track_orbit", c_int, [c_void_p, c_double, c_double, c_double, POINTER(c_double), c_int]),
    ("stb_cal_chrom_track", c_int, [c_void_p, c_double, c_double, POINTER(c_double), c_int]),
    ("stb_track_tbt", c_int, [c_void_p, POINTER(c_double), c_long, c_int, POINTER(c_double), POINTER(c_int),
                              POINTER(c_int), POINTER(c_int), c_int]),
    ("stb_track_tbt_bpm", c_int, [c_void_p, POINTER(c_double), c_long, c_int, POINTER(c_double), c_int, POINTER(c_int),
                                  POINTER(c_int), POINTER(c_int), c_int]),
    ("stb_cal_dz0", c_int, [c_void_p, POINTER(c_double), POINTER(c_double), c_int]),
    ("stb_track_wrt_onmom", c_int, [c_void_p, POINTER(c_double), c_long, POINTER(c_double), c_int, POINTER(c_int),
                                    POINTER(c_int), POINTER(c_int), c_int]),
    ("stb_track_tbt_spin_bpm", c_int, [c_void_p, POINTER(c_double), c_long, c_int, POINTER(c_double), c_int,
                                       POINTER(c_int), POINTER(c_int), POINTER(c_int), c_int]),
    ("stb_track_tbt_spin", c_int, [c_void_p, POINTER(c_double), c_long, c_int, POINTER(c_double), POINTER(c_int),
                                   POINTER(c_int), POINTER(c_int), c_int]),
    ("stb_track_tbt_fma", c_int, [c_void_p, c_double, c_double, c_double, c_double, c_double, c_char_p,
                                  POINTER(c_long), c_int]),
    ("stb_track_tbt_lyapunov", c_int, [c_void_p, c_double, c_double, c_double, c_char_p, POINTER(c_long), c_int]),
    ("stb_cal_orbit", c_int, [c_void_p, c_double, POINTER(c_double), c_int]),
    ("stb_track_da", c_int, [c_void_p, c_int, c_double, c_double, c_double, c_char_p, POINTER(c_double),
                             POINTER(c_double), c_int]),
    ("stb_track_radial_device", c_int, [c_void_p] + [c_void_p] * 6 + [c_long, c_int, c_int, c_double, c_void_p,
                                                                       c_void_p, c_void_p]),
    ("stb_track_radial_host", c_int, [c_void_p, POINTER(c_double), c_long, c_int, c_double, POINTER(c_int),
                                      POINTER(c_int), POINTER(c_int)]),
    ("stb_track_radial_probe", c_int, [c_void_p, POINTER(c_double), c_long, c_int, c_double, POINTER(c_double),
                                       POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    ("stb_track_spin_device", c_int, [c_void_p] + [c_void_p] * 9 + [c_long, c_int, c_int, c_double, c_void_p,
                                                                     c_void_p, c_void_p]),
    ("stb_track_spin_host", c_int, [c_void_p, POINTER(c_double), c_long, c_int, c_double, POINTER(c_int),
                                    POINTER(c_int), POINTER(c_int)]),
    ("stb_track_spin_probe", c_int, [c_void_p, POINTER(c_double), c_long, c_int, c_double, POINTER(c_double),
                                     POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    ("stb_fine_tune", c_int, [c_void_p, c_void_p, c_int, c_long, c_long, c_double, c_double, c_void_p, c_int,
                              c_void_p]),
    ("stb_tbt_features", c_int, [c_void_p, c_long, c_int, c_void_p, c_void_p, POINTER(c_double), c_void_p, c_int,
                                 c_void_p]),
    ("stb_scan_retire", c_int, [c_void_p, c_void_p]),
    ("stb_scan_set_abort", c_int, [c_void_p, c_int]),
    ("stb_scan_set_packing", c_int, [c_void_p, c_int]),
    ("stb_scan_packing", c_int, [c_void_p, POINTER(c_int)]),
    ("stb_table_set_contraction", c_int, [c_void_p, c_int]),
    ("stb_table_set_segment_bytes", c_int, [c_void_p, c_long]),
    ("stb_table_segments", c_int, [c_void_p, POINTER(c_int), POINTER(c_int)]),
    ("stb_table_autotune_spin", c_int, [c_void_p, POINTER(c_void_p), c_long, c_int, c_double, POINTER(c_int),
                                        POINTER(c_double), c_int]),
    ("stb_spin_variant_info", c_int, [c_int, ctypes.c_char_p, c_int, POINTER(c_int), POINTER(c_int)]),
    ("stb_scan_set_budget", c_int, [c_void_p, c_double]),
    ("stb_scan_checkpoint", c_int, [c_void_p, c_char_p]),
    ("stb_scan_restore", c_int, [c_void_p, c_char_p]),
    ("stb_track_seeds_static", c_int, [POINTER(c_void_p), c_int, POINTER(c_long)] + [c_void_p] * 8 +
     [c_int, c_int, c_double, c_void_p]),
    ("stb_mlp_create", c_int, [c_int, c_int, c_int, c_int, c_ulonglong, c_int, POINTER(c_void_p)]),
    ("stb_mlp_free", c_int, [c_void_p]),
    ("stb_mlp_param_count", c_long, [c_void_p]),
    ("stb_mlp_get_params", c_int, [c_void_p, POINTER(c_float), c_int]),
    ("stb_mlp_set_params", c_int, [c_void_p, POINTER(c_float)]),
    ("stb_mlp_set_adamw", c_int, [c_void_p, c_float, c_float, c_float, c_float, c_float]),
    ("stb_mlp_forward", c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    ("stb_mlp_gradients", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, POINTER(c_float)]),
    ("stb_mlp_train_step", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, POINTER(c_float)]),
    ("stb_mlp_gemm_test", c_int, [c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_int, c_int]),
    ("stb_fp64_peak", c_int, [c_int, POINTER(c_double)]),
    ("stb_check_drift_quotients", c_int, [c_long, c_ulonglong, c_int, POINTER(c_ulonglong)]),
    ("stb_check_sincos", c_int, [c_long, c_ulonglong, c_int, POINTER(c_ulonglong)]),
    ("stb_bb4d_soft_gaussian_device", c_int, [c_double, c_long, c_void_p, c_double, c_long, c_void_p, c_double,
                                              c_double, c_double, c_double, c_int, c_void_p]),
    ("stb_bb4d_soft_gaussian_host", c_int, [c_double, c_long, POINTER(c_double), c_double, c_long, POINTER(c_double),
                                            c_double, c_double, c_double, c_double, c_int]),
    ("stb_bb4d_pic_device", c_int, [c_double, c_long, c_void_p, c_double, c_long, c_void_p, c_double, c_double,
                                    c_double, c_double, c_int, c_void_p]),
    ("stb_bb4d_pic_host", c_int, [c_double, c_long, POINTER(c_double), c_double, c_long, POINTER(c_double), c_double,
                                  c_double, c_double, c_double, c_int]),
    ("stb_lumi_pic_4d_device", c_int, [c_double, c_long, c_double, c_long, c_void_p, c_void_p, c_int, c_double, c_int,
                                       c_void_p, POINTER(c_double)]),
    ("stb_lumi_pic_4d_host", c_int, [c_double, c_long, c_double, c_long, POINTER(c_double), POINTER(c_double), c_int,
                                     c_double, c_int, POINTER(c_double)]),
    ("stb_pic_green_function", c_int, [c_double, c_double, c_int, c_int, c_double, c_double, POINTER(c_double),
                                       POINTER(c_double), c_int]),
    ("stb_bb4d_pic_nonoffset_device", c_int, [c_double, c_long, c_void_p, c_double, c_long, c_void_p, c_double,
                                              c_double, c_double, c_double, c_int, c_int, c_double, c_double,
                                              c_void_p, c_void_p, c_int, c_void_p]),
    ("stb_bb4d_pic_nonoffset_host", c_int, [c_double, c_long, POINTER(c_double), c_double, c_long, POINTER(c_double),
                                            c_double, c_double, c_double, c_double, c_int, c_int, c_double, c_double,
                                            POINTER(c_double), POINTER(c_double), c_int]),
    ("stb_bb6d_pic_device", c_int, [c_double, c_long, c_void_p, c_double, c_long, c_void_p, c_double, c_double,
                                    c_double, c_double, c_int, c_int, c_int, c_void_p]),
    ("stb_bb6d_pic_host", c_int, [c_double, c_long, POINTER(c_double), c_double, c_long, POINTER(c_double), c_double,
                                  c_double, c_double, c_double, c_int, c_int, c_int]),
    ("stb_lumi_pic_6d_device", c_int, [c_double, c_long, c_double, c_long, c_int, c_int, c_void_p, c_void_p, c_double,
                                       c_double, c_double, c_double, c_int, c_double, c_int, c_void_p,
                                       POINTER(c_double)]),
    ("stb_lumi_pic_6d_host", c_int, [c_double, c_long, c_double, c_long, c_int, c_int, POINTER(c_double),
                                     POINTER(c_double), c_double, c_double, c_double, c_double, c_int, c_double, c_int,
                                     POINTER(c_double)]),
    ("stb_bb6d_pic_nonoffset_host", c_int, [c_double, c_long, POINTER(c_double), c_double, c_long, POINTER(c_double),
                                            c_double, c_double, c_double, c_double, c_int, c_int, POINTER(c_double),
                                            POINTER(c_double), c_int, c_int, c_double, c_double, POINTER(c_double),
                                            POINTER(c_double), c_int]),
    ("stb_lumi_pic_6d_angle_host", c_int, [c_double, c_long, c_double, c_long, c_double, c_int, c_int,
                                           POINTER(c_double), POINTER(c_double), c_double, c_double, c_double,
                                           c_double, c_int, c_double, c_int, POINTER(c_double)]),
    ("stb_bb6d_pic_interpolation_host", c_int, [c_double, c_long, POINTER(c_double), c_double, c_long,
                                                POINTER(c_double), c_double, c_double, c_double, c_double, c_int,
                                                c_int, POINTER(c_double), POINTER(c_double), c_int, c_int, c_double,
                                                c_double, POINTER(c_double), POINTER(c_double), c_int]),
    ("stb_bb6d_soft_gaussian_device", c_int, [c_double, c_long, c_void_p, c_double, c_long, c_void_p, c_double,
                                              c_double, c_double, c_double, c_int, c_int, c_int, c_void_p]),
    ("stb_bb6d_soft_gaussian_host", c_int, [c_double, c_long, POINTER(c_double), c_double, c_long, POINTER(c_double),
                                            c_double, c_double, c_double, c_double, c_int, c_int, c_int]),
    ("stb_bb6d_soft_gaussian_zb_host", c_int, [c_double, c_long, POINTER(c_double), c_double, c_long,
                                               POINTER(c_double), c_double, c_double, c_double, c_double, c_int, c_int,
                                               POINTER(c_double), POINTER(c_double), c_int]),
    ("stb_rad_normals", c_int, [c_ulonglong, c_ulonglong, c_ulonglong, c_long, POINTER(c_double), c_int]),
    ("stb_philox4x32_10", c_int, [POINTER(ctypes.c_uint), POINTER(ctypes.c_uint), POINTER(ctypes.c_uint)]),
    ("stb_math_eval", c_int, [c_int, POINTER(c_double), POINTER(c_double), c_long, c_int]),
    ("stb_track_probe", c_int, [c_void_p, POINTER(c_double), c_long, c_int, c_double, POINTER(c_double),
                                POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
]

_lib = None


def lib() -> ctypes.CDLL:
    """Loads the in-tree native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise SimTrackError(STB_EINVAL, f"native library not built: {LIB_PATH} "
                                            "(run python -m simtrack_b200.build)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != STB_OK:
        msg = lib().stb_last_error()
        raise SimTrackError(rc, msg.decode() if msg else "")
