"""Per-stage calls: the reference's ``sar/`` functions one by one over the C ABI.

Each function takes and returns data in the reference's layout, so a caller that keeps the
reference's own pipeline (main.cc) can swap a single stage.  Images are
``DevicePaddedImage`` (cuda_util/device_padded_image.cuh:13-27): a complex64
[y_stride][x_stride] array with the data block [0, y_size) x [0, x_size) at the top left.
Arrays are torch CUDA tensors for the product library; the host-emulation test build of
the same ABI takes numpy arrays instead.  Every call synchronises its stream before it
returns, as the reference functions do.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import load_library

__all__ = ["DevicePaddedImage", "convert_ers_samples", "raw_data_correction", "zero_nans",
           "calculate_doppler_centroid", "range_compression", "range_doppler_algorithm",
           "azimuth_multilook", "range_spreading_loss_correction", "srgr_interpolation", "srgr_index", "srgr_polynomial"]


def _ptr(x) -> int:
    if x is None:
        return 0
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return int(x.data_ptr())


def _stream(x) -> int:
    if isinstance(x, np.ndarray) or x is None:
        return 0
    import torch
    return int(torch.cuda.current_stream(x.device).cuda_stream)


def _check_contig(x, what: str) -> None:
    ok = x.flags["C_CONTIGUOUS"] if isinstance(x, np.ndarray) else x.is_contiguous()
    if not ok:
        raise ValueError(f"{what} must be contiguous")


@dataclass
class DevicePaddedImage:
    """Padded complex image (DevicePaddedImage of the reference): ``data`` has shape
    (y_stride, x_stride), complex64."""
    data: object
    x_size: int
    y_size: int

    @property
    def x_stride(self) -> int:
        return int(self.data.shape[1])

    @property
    def y_stride(self) -> int:
        return int(self.data.shape[0])

    def __post_init__(self):
        _check_contig(self.data, "image")
        if len(self.data.shape) != 2 or self.x_size > self.x_stride or self.y_size > self.y_stride:
            raise ValueError("image block exceeds its padded shape")


def convert_ers_samples(raw, samples_per_line: int, img, range_size: int, swst=None, min_swst: int = 0,
                        lib=None) -> None:
    """ConvertErsImSamplesToComplexKernel (envisat_format/src/envisat_format_kernels.cu:116-134):
    ``raw`` uint8 [lines][line_bytes] -> rows [0, range_size) of complex ``img``."""
    lib = lib or load_library()
    _check_contig(raw, "raw")
    lines, line_bytes = int(raw.shape[0]), int(raw.shape[1])
    rc = lib.asarf_convert_ers_samples(_ptr(raw), line_bytes, int(samples_per_line), lines, _ptr(swst),
                                       int(min_swst), _ptr(img), int(img.shape[1]), int(range_size), _stream(img))
    _lib.check(lib, rc, "convert_ers_samples")


def convert_asar_blocks(raw, img, range_size: int, lut_i, lut_q, swst=None, min_swst: int = 0, lib=None) -> None:
    """ConvertAsarImBlocksToComplexKernel (envisat_format/src/envisat_format_kernels.cu:160-209):
    FBAQ4 records ``raw`` uint8 [records][record_bytes] -> rows [0, range_size) of complex
    ``img`` (NaN where a record holds no sample); ``lut_i`` / ``lut_q``: the 4096-entry tables
    (instrument-file order) in the same memory as ``img``."""
    lib = lib or load_library()
    _check_contig(raw, "raw")
    records, record_bytes = int(raw.shape[0]), int(raw.shape[1])
    rc = lib.asarf_convert_asar_blocks(_ptr(raw), record_bytes, records, _ptr(swst), int(min_swst), _ptr(lut_i),
                                       _ptr(lut_q), _ptr(img), int(img.shape[1]), int(range_size), _stream(img))
    _lib.check(lib, rc, "convert_asar_blocks")


def condition_slc(img, x_size: int, dest, record_header_bytes: int = 17, calibration: float = 1.0,
                  lib=None) -> None:
    """ConditionResultsSLC (envisat_format/src/envisat_format_kernels.cu:28-61, 95-106): complex
    ``img`` [rows][stride] (first x_size columns) -> IMS MDS records in ``dest``
    (rows x (header + 4 x_size) bytes)."""
    lib = lib or load_library()
    rows, stride = int(img.shape[0]), int(img.shape[1])
    rc = lib.asarf_condition_slc(_ptr(img), int(x_size), rows, stride, int(record_header_bytes), float(calibration),
                                 _ptr(dest), _stream(img))
    _lib.check(lib, rc, "condition_slc")


def condition_detected(img, dest, record_header_bytes: int = 17, calibration: float = 1.0, lib=None) -> None:
    """ConditionResultsDetected (envisat_format/src/envisat_format_kernels.cu:63-93, 108-114): float
    ``img`` [rows][cols] -> IMP MDS records in ``dest`` (rows x (header + 2 cols) bytes)."""
    lib = lib or load_library()
    rows, cols = int(img.shape[0]), int(img.shape[1])
    rc = lib.asarf_condition_detected(_ptr(img), cols, rows, int(record_header_bytes), float(calibration), _ptr(dest),
                                      _stream(img))
    _lib.check(lib, rc, "condition_detected")


def raw_data_correction(img: DevicePaddedImage, n_total_samples: int, lib=None) -> dict:
    """RawDataCorrection (sar/iq_correction.cu:188-274) in place; returns the SARResults
    fields it sets."""
    lib = lib or load_library()
    res = _lib.IqResults()
    rc = lib.asarf_raw_data_correction(_ptr(img.data), img.x_size, img.y_size, img.x_stride, img.y_stride,
                                       int(n_total_samples), C.byref(res), _stream(img.data))
    _lib.check(lib, rc, "raw_data_correction")
    return {k: float(getattr(res, k)) for k, _ in _lib.IqResults._fields_}


def zero_nans(img: DevicePaddedImage, lib=None) -> None:
    """DevicePaddedImage::ZeroNaNs (cuda_util/device_padded_image.cu:322-329)."""
    lib = lib or load_library()
    rc = lib.asarf_zero_nans(_ptr(img.data), img.x_stride, img.y_stride, _stream(img.data))
    _lib.check(lib, rc, "zero_nans")


def calculate_doppler_centroid(img: DevicePaddedImage, prf: float, lib=None) -> list[float]:
    """CalculateDopplerCentroid (sar/fractional_doppler_centroid.cu:98-139): quadratic
    Doppler-centroid polynomial over range pixels, highest power first."""
    lib = lib or load_library()
    poly = (C.c_double * 3)()
    rc = lib.asarf_doppler_centroid(_ptr(img.data), img.x_size, img.y_size, img.x_stride, float(prf),
                                    C.byref(poly), _stream(img.data))
    _lib.check(lib, rc, "doppler_centroid")
    return list(poly)


def range_compression(img: DevicePaddedImage, chirp_padded: np.ndarray, chirp_samples: int, lib=None) -> int:
    """RangeCompression (sar/range_compression.cu:57-111) in place; ``chirp_padded`` is the
    complex64 ChirpInfo::padded_windowed_data.  Updates and returns ``img.x_size``."""
    lib = lib or load_library()
    ch = np.ascontiguousarray(np.asarray(chirp_padded, dtype=np.complex64))
    new_x = C.c_int32(0)
    rc = lib.asarf_range_compression(_ptr(img.data), img.x_size, img.y_size, img.x_stride,
                                     ch.ctypes.data_as(C.POINTER(C.c_float)), int(ch.shape[0]), int(chirp_samples),
                                     C.byref(new_x), _stream(img.data))
    _lib.check(lib, rc, "range_compression")
    img.x_size = int(new_x.value)
    return img.x_size


def range_doppler_algorithm(prf: float, wavelength: float, range_spacing: float, slant_range_first: float,
                            az_bw_frac: float, vr_poly, dc_poly, src: DevicePaddedImage, out_data,
                            lib=None) -> DevicePaddedImage:
    """RangeDopplerAlgorithm (sar/range_doppler_algorithm.cu:312-407): ``src`` is consumed
    (its columns hold the azimuth spectrum afterwards); ``out_data`` has src's padded shape."""
    lib = lib or load_library()
    p = _lib.RdaParams()
    p.prf, p.wavelength, p.range_spacing = float(prf), float(wavelength), float(range_spacing)
    p.slant_range_first, p.az_bw_frac = float(slant_range_first), float(az_bw_frac)
    p.vr_poly = (C.c_double * 3)(*[float(v) for v in vr_poly])
    p.dc_poly = (C.c_double * 3)(*[float(v) for v in dc_poly])
    out = DevicePaddedImage(out_data, src.x_size, src.y_size)
    if out.x_stride != src.x_stride or out.y_stride != src.y_stride:
        raise ValueError("output image must have the source's padded shape")
    rc = lib.asarf_range_doppler(C.byref(p), _ptr(src.data), _ptr(out_data), src.x_size, src.y_size, src.x_stride,
                                 src.y_stride, _stream(src.data))
    _lib.check(lib, rc, "range_doppler")
    return out


def azimuth_multilook(slc, azimuth_spacing: float, out, lib=None) -> int:
    """AzimuthMultiLook (sar/az_multilook.cu:82-98): ``slc`` complex64 [y][x] contiguous,
    ``out`` float32 with room for round(y / ratio) rows; returns the output row count."""
    lib = lib or load_library()
    _check_contig(slc, "slc")
    out_y = C.c_int32(0)
    y, x = int(slc.shape[0]), int(slc.shape[1])
    ratio = np.float32(12.5 / float(azimuth_spacing))
    need = int(np.round(np.float32(y) / ratio)) + 1
    if int(np.prod(out.shape)) < (need - 1) * x:
        raise ValueError("multilook output too small")
    rc = lib.asarf_azimuth_multilook(_ptr(slc), x, y, float(azimuth_spacing), _ptr(out), C.byref(out_y),
                                     _stream(slc))
    _lib.check(lib, rc, "azimuth_multilook")
    return int(out_y.value)


def range_spreading_loss_correction(img, slant_range_first: float, range_spacing: float, reference_range: float,
                                    lib=None) -> None:
    """RangeSpreadingLossCorrection (sar/range_spreading_loss.cu:54-68) in place on float32 [az][rg]."""
    lib = lib or load_library()
    _check_contig(img, "image")
    rc = lib.asarf_range_spreading_loss(_ptr(img), int(img.shape[1]), int(img.shape[0]), float(slant_range_first),
                                        float(range_spacing), float(reference_range), _stream(img))
    _lib.check(lib, rc, "range_spreading_loss")


def srgr_interpolation(slant, grsr_poly, range_spacing: float, out, lib=None) -> None:
    """SrGrInterpolation (sar/srgr.cu:49-71): float32 [y][in_x] -> ``out`` float32 [y][out_x]."""
    lib = lib or load_library()
    _check_contig(slant, "slant image")
    _check_contig(out, "ground image")
    poly = (C.c_double * 5)(*[float(v) for v in grsr_poly])
    rc = lib.asarf_srgr(_ptr(slant), int(slant.shape[1]), int(slant.shape[0]), C.byref(poly), float(range_spacing),
                        int(out.shape[1]), _ptr(out), _stream(slant))
    _lib.check(lib, rc, "srgr")


def srgr_index(grsr_poly, range_spacing: float, start, frac, lib=None) -> None:
    """Per-column (index, fraction) of SrGrInterpolation into int32 ``start`` and float32 ``frac``."""
    lib = lib or load_library()
    poly = (C.c_double * 5)(*[float(v) for v in grsr_poly])
    rc = lib.asarf_srgr_index(C.byref(poly), float(range_spacing), int(start.shape[0]), _ptr(start), _ptr(frac),
                              _stream(start))
    _lib.check(lib, rc, "srgr_index")


def srgr_polynomial(scene, slant_first: float, range_size: int, azimuth_size: int, line_time_interval: float,
                    lib=None) -> tuple[list[float], int]:
    """Ground->slant polynomial and ground sample count of SlantRangeToGroundRangeInterpolation
    (sar/srgr.cu:73-121) for a prepared ``asarf.Scene``."""
    lib = lib or load_library()
    sc, keep = scene.to_c()
    poly = (C.c_double * 5)()
    ng = C.c_int32(0)
    rc = lib.asarf_srgr_polynomial(C.byref(sc), float(slant_first), int(range_size), int(azimuth_size),
                                   float(line_time_interval), C.byref(poly), C.byref(ng))
    del keep
    _lib.check(lib, rc, "srgr_polynomial")
    return list(poly), int(ng.value)
