"""asar-focus B200: range-Doppler SAR focusing on sm_100a.

Python host layer over the C ABI (include/asarf.h, libasarf.so).  The CUDA library is
the only execution path: importing works without it, but every call that needs it raises
``AsarfError`` when it is not built.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import AsarfError, load_library
from .scene import Scene

__all__ = ["FocusPlan", "Scene", "AsarfError", "load_library", "version", "fft_size_above"]


def version(lib=None) -> str:
    lib = lib or load_library()
    return lib.asarf_version().decode()


def fft_size_above(v: int, lib=None) -> int:
    """GetOptimalFFTSizes().upper_bound(v) of the reference (main.cc:217, 223)."""
    lib = lib or load_library()
    return int(lib.asarf_fft_size_above(int(v)))


def _ptr(x) -> int:
    if x is None:
        return 0
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return int(x.data_ptr())


class FocusPlan:
    """One planned scene shape (asarf_plan).  ``focus`` takes device tensors; ``focus_host``
    takes host arrays and does the copies inside (the end-to-end path)."""

    def __init__(self, scene: Scene, rc_fft_len: int = 0, ref_compat_stats: bool = True, lib=None,
                 lib_path=None, dc_poly=None):
        self.lib = lib or load_library(lib_path)
        self.scene = scene
        if scene.vr_poly is None or not scene.osv:
            scene.prepare(self.lib)
        self._sc, self._osv_keep = scene.to_c()
        opt = _lib.Options()
        self.lib.asarf_default_options(C.byref(opt))
        opt.rc_fft_len = int(rc_fft_len)
        opt.ref_compat_stats = int(bool(ref_compat_stats))
        if dc_poly is not None:
            opt.dc_poly_given = 1
            opt.dc_poly = (C.c_double * 3)(*[float(v) for v in dc_poly])
        h = C.c_void_p()
        _lib.check(self.lib, self.lib.asarf_plan_create(C.byref(self._sc), C.byref(opt), C.byref(h)), "plan_create")
        self._h = h
        d = _lib.Dims()
        _lib.check(self.lib, self.lib.asarf_plan_dims(self._h, C.byref(d)), "plan_dims")
        self.dims = {f: (list(getattr(d, f)) if f in ("out_rows", "out_cols", "vr_poly") else getattr(d, f))
                     for f, _ in d._fields_}

    def close(self):
        if getattr(self, "_h", None):
            self.lib.asarf_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def out_shape(self) -> tuple[int, int]:
        return self.dims["out_rows_max"], self.dims["out_cols_max"]

    def focus(self, raw, out, swst=None, min_swst: int = 0, stream: int = 0):
        """Asynchronous focus of device-resident raw bytes into ``out`` (float32
        [out_rows_max, out_cols_max]).  ``raw``/``out``/``swst`` expose data_ptr()."""
        _lib.check(self.lib, self.lib.asarf_focus(self._h, _ptr(raw), _ptr(swst), int(min_swst), _ptr(out),
                                                  C.c_void_p(stream)), "focus")
        return out

    def focus_host(self, raw: np.ndarray, swst: np.ndarray | None = None, stream: int = 0) -> np.ndarray:
        """Host raw bytes [Na, raw_line_bytes] uint8 -> host detected image (float32)."""
        raw = np.ascontiguousarray(raw, dtype=np.uint8)
        sw = None
        mn = 0
        if swst is not None:
            sw = np.ascontiguousarray(swst, dtype=np.uint16)
            mn = int(sw.min())
        out = np.empty(self.out_shape, dtype=np.float32)
        _lib.check(self.lib, self.lib.asarf_focus_host(self._h, raw.ctypes.data, _ptr(sw), mn, out.ctypes.data,
                                                       C.c_void_p(stream)), "focus_host")
        r = self.results(stream)
        return out[: r["out_rows"], : r["out_cols"]]

    def focus_host_ptr(self, raw_ptr: int, out_ptr: int, swst_ptr: int = 0, min_swst: int = 0, stream: int = 0):
        """asarf_focus_host on raw host pointers (e.g. pinned torch tensors); synchronous."""
        _lib.check(self.lib, self.lib.asarf_focus_host(self._h, raw_ptr, swst_ptr or None, int(min_swst), out_ptr,
                                                       C.c_void_p(stream)), "focus_host")

    def results(self, stream: int = 0) -> dict:
        r = _lib.Results()
        _lib.check(self.lib, self.lib.asarf_plan_results(self._h, C.byref(r), C.c_void_p(stream)), "plan_results")
        d = {}
        for f, _ in r._fields_:
            v = getattr(r, f)
            d[f] = list(v) if not isinstance(v, (int, float)) else v
        d["dc_block_hz"] = d["dc_block_hz"][: d["n_dc_blocks"]]
        return d

    def enable_timing(self, runs: int) -> None:
        """Record events between the kernels of the next ``runs`` focus calls."""
        _lib.check(self.lib, self.lib.asarf_plan_enable_timing(self._h, int(runs)), "enable_timing")

    def kernel_times(self) -> tuple[dict, int]:
        """({kernel: total ms over the recorded runs}, runs)."""
        ms = (C.c_float * 7)()
        names = (C.c_char_p * 7)()
        runs = C.c_int32()
        _lib.check(self.lib, self.lib.asarf_plan_kernel_times(self._h, ms, C.byref(runs), names), "kernel_times")
        return {names[k].decode(): float(ms[k]) for k in range(7)}, int(runs.value)

    def slc_into(self, dst, stream: int = 0):
        """Copy the subset complex image of the last run into ``dst`` (complex64
        [n_lines, slc_cols], device memory or, for a host build, host memory)."""
        _lib.check(self.lib, self.lib.asarf_plan_slc(self._h, C.c_void_p(_ptr(dst)), C.c_void_p(stream)), "plan_slc")
        return dst
