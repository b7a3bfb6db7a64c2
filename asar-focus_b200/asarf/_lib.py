"""ctypes binding of the C ABI in include/asarf.h (libasarf.so)."""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libasarf.so"


class Osv(C.Structure):
    _fields_ = [("time_us", C.c_int64), ("pos", C.c_double * 3), ("vel", C.c_double * 3)]


class SceneC(C.Structure):
    _fields_ = [
        ("range_size", C.c_int32), ("azimuth_size", C.c_int32), ("samples_per_line", C.c_int32),
        ("raw_line_bytes", C.c_int32), ("total_raw_samples", C.c_int64),
        ("range_sampling_rate", C.c_double), ("chirp_kr", C.c_double), ("pulse_duration", C.c_double),
        ("chirp_samples", C.c_int32), ("apply_window", C.c_int32),
        ("prf", C.c_double), ("wavelength", C.c_double), ("carrier_frequency", C.c_double),
        ("range_spacing", C.c_double), ("slant_range_first", C.c_double), ("azimuth_spacing", C.c_double),
        ("az_bw_frac", C.c_double),
        ("vr_poly", C.c_double * 3), ("vr_poly_given", C.c_int32), ("vr_poly_init", C.c_double * 3),
        ("n_osv", C.c_int32), ("osv", C.POINTER(Osv)),
        ("first_line_time_us", C.c_int64), ("line_time_interval", C.c_double),
        ("center_point", C.c_double * 3), ("lines_before", C.c_int32), ("lines_after", C.c_int32),
        ("raw_format", C.c_int32), ("fbaq_i_lut", C.POINTER(C.c_float)), ("fbaq_q_lut", C.POINTER(C.c_float)),
    ]


RAW_ERS_BYTES = 0
RAW_ASAR_FBAQ4 = 1


class Options(C.Structure):
    _fields_ = [("rc_fft_len", C.c_int32), ("ref_compat_stats", C.c_int32), ("iq_padding_ref", C.c_int32),
                ("dc_poly_given", C.c_int32), ("dc_poly", C.c_double * 3), ("product", C.c_int32),
                ("record_header_bytes", C.c_int32), ("calibration", C.c_float), ("sq_stats", C.c_int32),
                ("precision", C.c_int32), ("absolute_phase", C.c_int32), ("az_n2", C.c_int32),
                ("az_tile_width", C.c_int32), ("strided_tile_width", C.c_int32), ("keep_slc", C.c_int32),
                ("compiled_schedules", C.c_int32)]


PRECISION_FP32 = 0
PRECISION_SPLIT = 1

PRODUCT_DETECTED = 0
PRODUCT_IMP_MDS = 1
PRODUCT_IMS_MDS = 2


class Dims(C.Structure):
    _fields_ = [
        ("nk", C.c_int32), ("rg_pad_ref", C.c_int32), ("az_pad", C.c_int32), ("rc_fft_len", C.c_int32),
        ("n1", C.c_int32), ("n2", C.c_int32), ("slc_cols", C.c_int32), ("out_rows", C.c_int32 * 2),
        ("out_cols", C.c_int32 * 2), ("out_rows_max", C.c_int32), ("out_cols_max", C.c_int32),
        ("max_aperture", C.c_int32), ("vr_poly", C.c_double * 3), ("device_bytes", C.c_size_t),
        ("out_bytes_max", C.c_int64), ("precision", C.c_int32), ("split_radix", C.c_int32), ("split_m", C.c_int32),
        ("az_tile_width", C.c_int32), ("strided_tile_width", C.c_int32), ("compiled_schedules", C.c_int32),
    ]


class Results(C.Structure):
    _fields_ = [
        ("dc_i", C.c_double), ("dc_q", C.c_double), ("iq_gain", C.c_double), ("phase_error", C.c_double),
        ("stddev_i", C.c_double), ("stddev_q", C.c_double), ("doppler_centroid_poly", C.c_double * 3),
        ("doppler_centroid_estimate", C.c_double * 3),
        ("vr_poly", C.c_double * 3), ("n_dc_blocks", C.c_int32), ("dc_block_hz", C.c_double * 80),
        ("variant", C.c_int32), ("first_line", C.c_int32), ("n_lines", C.c_int32), ("out_rows", C.c_int32),
        ("out_cols", C.c_int32), ("errors", C.c_uint32), ("records", C.c_int32), ("record_bytes", C.c_int32),
        ("sq_stats", C.c_double * 4),
    ]


class RawStats(C.Structure):
    _fields_ = [
        ("dc_i", C.c_double), ("dc_q", C.c_double), ("iq_gain", C.c_double), ("phase_error", C.c_double),
        ("stddev_i", C.c_double), ("stddev_q", C.c_double), ("doppler_centroid_poly", C.c_double * 3),
        ("n_dc_blocks", C.c_int32), ("reserved", C.c_int32), ("dc_block_hz", C.c_double * 80),
        ("applied_dc_i", C.c_float), ("applied_dc_q", C.c_float), ("applied_gain", C.c_float),
        ("applied_sin", C.c_float), ("applied_cos", C.c_float), ("errors", C.c_uint32),
    ]


class IqResults(C.Structure):
    _fields_ = [("dc_i", C.c_double), ("dc_q", C.c_double), ("iq_gain", C.c_double), ("phase_error", C.c_double),
                ("stddev_i", C.c_double), ("stddev_q", C.c_double)]


class RdaParams(C.Structure):
    _fields_ = [("prf", C.c_double), ("wavelength", C.c_double), ("range_spacing", C.c_double),
                ("slant_range_first", C.c_double), ("az_bw_frac", C.c_double), ("vr_poly", C.c_double * 3),
                ("dc_poly", C.c_double * 3)]


class StripDims(C.Structure):
    _fields_ = [("n_blocks", C.c_int32), ("block_lines", C.c_int32), ("overlap", C.c_int32),
                ("first_line", C.c_int32), ("slc_rows", C.c_int32), ("slc_cols", C.c_int32),
                ("slc_pitch", C.c_int32), ("out_rows", C.c_int32), ("out_cols", C.c_int32),
                ("max_aperture", C.c_int32), ("device_bytes", C.c_size_t)]


class AsarfError(RuntimeError):
    pass


_SIGS = {
    "asarf_last_error": (C.c_char_p, []),
    "asarf_version": (C.c_char_p, []),
    "asarf_default_options": (None, [C.POINTER(Options)]),
    "asarf_plan_create": (C.c_int, [C.POINTER(SceneC), C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "asarf_plan_destroy": (None, [C.c_void_p]),
    "asarf_plan_dims": (C.c_int, [C.c_void_p, C.POINTER(Dims)]),
    "asarf_focus": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "asarf_focus_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "asarf_convert_asar_blocks": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_void_p]),
    "asarf_fbaq4_index": (C.c_int32, [C.c_int32, C.c_int32]),
    "asarf_condition_slc": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_float, C.c_void_p,
                                      C.c_void_p]),
    "asarf_condition_detected": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_float, C.c_void_p,
                                           C.c_void_p]),
    "asarf_focus_host_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "asarf_plan_wait": (C.c_int, [C.c_void_p]),
    "asarf_plan_slc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "asarf_plan_results": (C.c_int, [C.c_void_p, C.POINTER(Results), C.c_void_p]),
    "asarf_plan_enable_timing": (C.c_int, [C.c_void_p, C.c_int32]),
    "asarf_plan_kernel_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_int32),
                                          C.POINTER(C.c_char_p)]),
    "asarf_interpolate_orbit": (C.c_int, [C.POINTER(Osv), C.c_int32, C.c_int64, C.POINTER(Osv)]),
    "asarf_geolocate": (C.c_int, [C.POINTER(C.c_double * 3)] * 3 + [C.c_double, C.POINTER(C.c_double * 3)]),
    "asarf_polyfit": (C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int32, C.c_int32,
                                C.POINTER(C.c_double)]),
    "asarf_estimate_processing_velocity": (C.c_int, [C.POINTER(SceneC), C.POINTER(C.c_double * 3)]),
    "asarf_generate_chirp": (C.c_int, [C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_int32,
                                       C.POINTER(C.c_float)]),
    "asarf_srgr_polynomial": (C.c_int, [C.POINTER(SceneC), C.c_double, C.c_int32, C.c_int32, C.c_double,
                                        C.POINTER(C.c_double * 5), C.POINTER(C.c_int32)]),
    "asarf_fft_size_above": (C.c_int32, [C.c_int32]),
    "asarf_raw_statistics_noalloc": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                               C.c_int32, C.c_int64, C.c_int32, C.c_double, C.c_void_p,
                                               C.c_void_p]),
    "asarf_batch_create": (C.c_int, [C.POINTER(SceneC), C.c_int32, C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]),
    "asarf_batch_destroy": (None, [C.c_void_p]),
    "asarf_batch_plan": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]),
    "asarf_batch_branch": (C.c_int, [C.c_void_p, C.c_int32]),
    "asarf_batch_focus": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p,
                                    C.POINTER(C.c_void_p), C.c_void_p]),
    "asarf_lpt_assign": (C.c_int, [C.POINTER(C.c_int64), C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "asarf_strip_create": (C.c_int, [C.POINTER(SceneC), C.c_int32, C.c_int32, C.c_void_p, C.POINTER(C.c_void_p)]),
    "asarf_strip_destroy": (None, [C.c_void_p]),
    "asarf_strip_get_dims": (C.c_int, [C.c_void_p, C.POINTER(StripDims)]),
    "asarf_strip_block": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                    C.POINTER(C.c_int32), C.POINTER(C.c_void_p)]),
    "asarf_focus_strip": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "asarf_strip_slc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "asarf_strip_errors": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.c_void_p]),
    # per-stage entry points
    "asarf_convert_ers_samples": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int32,
                                            C.c_void_p, C.c_int64, C.c_int32, C.c_void_p]),
    "asarf_raw_data_correction": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int64,
                                            C.POINTER(IqResults), C.c_void_p]),
    "asarf_zero_nans": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "asarf_doppler_centroid": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                         C.POINTER(C.c_double * 3), C.c_void_p]),
    "asarf_range_compression": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_float),
                                          C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.c_void_p]),
    "asarf_range_doppler": (C.c_int, [C.POINTER(RdaParams), C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                      C.c_int32, C.c_void_p]),
    "asarf_azimuth_multilook": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_void_p,
                                          C.POINTER(C.c_int32), C.c_void_p]),
    "asarf_range_spreading_loss": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                             C.c_void_p]),
    "asarf_srgr": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double * 5), C.c_double, C.c_int32,
                             C.c_void_p, C.c_void_p]),
    "asarf_srgr_index": (C.c_int, [C.POINTER(C.c_double * 5), C.c_double, C.c_int32, C.c_void_p, C.c_void_p,
                                   C.c_void_p]),
}

_cache: dict[str, C.CDLL] = {}


def load_library(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load libasarf.so (or another build of the same C ABI).  Raises if it is missing:
    the product has no fallback path."""
    p = str(Path(path) if path is not None else LIB_PATH)
    if p in _cache:
        return _cache[p]
    if not Path(p).exists():
        raise AsarfError(f"native library not built: {p} (run asar-focus_b200/build.py)")
    lib = C.CDLL(p)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _cache[p] = lib
    return lib


def check(lib: C.CDLL, rc: int, what: str) -> None:
    if rc != 0:
        msg = lib.asarf_last_error().decode(errors="replace")
        raise AsarfError(f"{what} failed ({rc}): {msg}")
