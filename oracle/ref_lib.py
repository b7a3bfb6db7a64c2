"""ctypes binding of the reference build (oracle/_ref/libasar_ref.so, made by oracle/ref_build).

TEST INFRASTRUCTURE ONLY: the reference's own CUDA focusing code, run on the GPU to pin
the CPU oracle and to time the reference arm of the benchmark.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

REF_LIB = Path(__file__).resolve().parent / "_ref" / "libasar_ref.so"
# the same harness over the product's header-compatible drop-in (asar-focus_b200/dropin)
DROPIN_LIB = Path(__file__).resolve().parent / "_ref" / "libasar_dropin.so"


class RefOutputs(C.Structure):
    _fields_ = [
        ("dc_i", C.c_double), ("dc_q", C.c_double), ("iq_gain", C.c_double), ("phase_error", C.c_double),
        ("stddev_i", C.c_double), ("stddev_q", C.c_double), ("dc_poly", C.c_double * 3),
        ("grsr_poly", C.c_double * 5), ("first_line", C.c_int32), ("n_lines", C.c_int32),
        ("slc_cols", C.c_int32), ("out_rows", C.c_int32), ("out_cols", C.c_int32), ("max_aperture", C.c_int32),
        ("ms_total", C.c_double), ("ms_after_decode", C.c_double), ("ms_wall", C.c_double),
        ("error", C.c_char * 256), ("ims_stats", C.c_double * 4), ("imp_stats", C.c_double * 4),
    ]


_libs: dict = {}


def available(path: Path = REF_LIB) -> bool:
    return path.exists()


def load(path: Path = REF_LIB):
    if path not in _libs:
        if not path.exists():
            raise FileNotFoundError(f"reference build missing: {path} (make -C oracle/ref_build)")
        lib = C.CDLL(str(path))
        f = lib.ref_focus
        f.restype = C.c_int
        f.argtypes = [C.c_void_p, C.POINTER(C.c_double * 3), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                      C.POINTER(RefOutputs), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        if hasattr(lib, "ref_convert_asar"):
            g = lib.ref_convert_asar
            g.restype = C.c_int
            g.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                          C.c_void_p]
        for name in ("ref_condition_slc", "ref_condition_detected"):
            if hasattr(lib, name):
                h = getattr(lib, name)
                h.restype = C.c_int
                h.argtypes = [C.c_void_p, C.c_int32, C.c_int32] + ([C.c_int32] if name == "ref_condition_slc" else []) \
                    + [C.c_int32, C.c_float, C.c_void_p]
        if hasattr(lib, "ref_set_statistics"):
            lib.ref_set_statistics.restype = None
            lib.ref_set_statistics.argtypes = [C.c_int]
        _libs[path] = lib
    return _libs[path]


def set_statistics(on: bool, lib_path: Path = REF_LIB) -> None:
    """Have ref_focus also compute the product statistics main.cc writes (ims_stats, imp_stats)."""
    load(lib_path).ref_set_statistics(int(bool(on)))


def ref_condition_slc(img: np.ndarray, x_size: int, hdr: int, cal: float, lib_path: Path = REF_LIB) -> np.ndarray:
    """The reference's ConditionResultsSLC on a complex64 [rows, stride] image (XSize x_size):
    uint8 [rows, hdr + 4 x_size]."""
    lib = load(lib_path)
    img = np.ascontiguousarray(img, dtype=np.complex64)
    y, stride = img.shape
    out = np.empty((y, hdr + 4 * x_size), dtype=np.uint8)
    if lib.ref_condition_slc(img.ctypes.data, x_size, y, stride, hdr, cal, out.ctypes.data) != 0:
        raise RuntimeError("reference ConditionResultsSLC failed")
    return out


def ref_condition_detected(img: np.ndarray, hdr: int, cal: float, lib_path: Path = REF_LIB) -> np.ndarray:
    """The reference's ConditionResultsDetected on a float32 [rows, cols] image: uint8 [rows, hdr + 2 cols]."""
    lib = load(lib_path)
    img = np.ascontiguousarray(img, dtype=np.float32)
    y, x = img.shape
    out = np.empty((y, hdr + 2 * x), dtype=np.uint8)
    if lib.ref_condition_detected(img.ctypes.data, x, y, hdr, cal, out.ctypes.data) != 0:
        raise RuntimeError("reference ConditionResultsDetected failed")
    return out


def ref_convert_asar(raw: np.ndarray, swst, i_lut: np.ndarray, q_lut: np.ndarray, range_size: int,
                     lib_path: Path = REF_LIB) -> np.ndarray:
    """The reference's ConvertAsarImBlocksToComplex on host FBAQ4 records (NaN pre-filled
    image, main_flow.cc:537-540): complex64 [records, range_size]."""
    lib = load(lib_path)
    raw = np.ascontiguousarray(raw, dtype=np.uint8)
    na, rec = raw.shape
    sw = None if swst is None else np.ascontiguousarray(swst, dtype=np.uint16)
    ti = np.ascontiguousarray(i_lut, dtype=np.float32)
    tq = np.ascontiguousarray(q_lut, dtype=np.float32)
    out = np.empty((na, range_size), dtype=np.complex64)
    rc = lib.ref_convert_asar(raw.ctypes.data, rec, na, None if sw is None else sw.ctypes.data, ti.ctypes.data,
                              tq.ctypes.data, range_size, out.ctypes.data)
    if rc != 0:
        raise RuntimeError("reference ConvertAsarImBlocksToComplex failed")
    return out


def ref_focus(scene_c, vr_poly, raw: np.ndarray, swst=None, dumps: bool = False, out_capacity: int | None = None,
              d_raw_ptr: int = 0, lib_path: Path = REF_LIB):
    """Run the reference chain (main.cc's flow) on host raw bytes, through the reference's
    own stages (REF_LIB) or through the drop-in (DROPIN_LIB).  Returns (detected float32
    [rows, cols], outputs dict, dumps dict)."""
    lib = load(lib_path)
    raw = np.ascontiguousarray(raw, dtype=np.uint8)
    na, nr = scene_c.azimuth_size, scene_c.range_size
    nk = nr - scene_c.chirp_samples
    cap = out_capacity or (na * nr)
    out = np.empty(cap, dtype=np.float32)
    d = {}
    ptrs = [None, None, None, None]
    if dumps:
        d["corrected"] = np.empty((na, nr), dtype=np.complex64)
        d["rc"] = np.empty((na, nk), dtype=np.complex64)
        d["slc"] = np.empty(na * (nk - 16), dtype=np.complex64)
        d["ml"] = np.empty(na * (nk - 16), dtype=np.float32)
        ptrs = [d["corrected"].ctypes.data, d["rc"].ctypes.data, d["slc"].ctypes.data, d["ml"].ctypes.data]
    sw = None if swst is None else np.ascontiguousarray(swst, dtype=np.uint16)
    o = RefOutputs()
    vr = (C.c_double * 3)(*vr_poly)
    rc = lib.ref_focus(C.addressof(scene_c), vr, raw.ctypes.data, None if sw is None else sw.ctypes.data,
                       out.ctypes.data, cap, C.byref(o), *ptrs, d_raw_ptr or None)
    if rc != 0:
        raise RuntimeError(f"reference chain failed ({rc}): {o.error.decode(errors='replace')}")
    res = {f: (list(getattr(o, f)) if f in ("dc_poly", "grsr_poly", "ims_stats", "imp_stats") else getattr(o, f))
           for f, _ in o._fields_}
    det = out[: o.out_rows * o.out_cols].reshape(o.out_rows, o.out_cols)
    if dumps:
        d["slc"] = d["slc"][: o.n_lines * o.slc_cols].reshape(o.n_lines, o.slc_cols)
        d["ml"] = d["ml"][: o.out_rows * o.slc_cols].reshape(o.out_rows, o.slc_cols)
    return det, res, d
