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

__all__ = ["FocusPlan", "FocusBatch", "FocusStrip", "Scene", "AsarfError", "load_library", "version", "fft_size_above",
           "lpt_assign"]


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
                 lib_path=None, dc_poly=None, product: int = 0, calibration: float = 1.0,
                 record_header_bytes: int = 17, sq_stats: bool = False, precision: int = 0,
                 absolute_phase: bool = False, az_n2: int = 0, az_tile_width: int = 0, strided_tile_width: int = 0,
                 keep_slc: bool = True, compiled_schedules: bool = True):
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
        opt.product = int(product)
        opt.calibration = float(calibration)
        opt.record_header_bytes = int(record_header_bytes)
        opt.sq_stats = int(bool(sq_stats))
        opt.precision = int(precision)
        opt.absolute_phase = int(bool(absolute_phase))
        opt.az_n2 = int(az_n2)
        opt.az_tile_width = int(az_tile_width)
        opt.strided_tile_width = int(strided_tile_width)
        opt.keep_slc = int(bool(keep_slc))
        opt.compiled_schedules = int(bool(compiled_schedules))
        self.product = int(product)
        h = C.c_void_p()
        _lib.check(self.lib, self.lib.asarf_plan_create(C.byref(self._sc), C.byref(opt), C.byref(h)), "plan_create")
        self._h = h
        d = _lib.Dims()
        _lib.check(self.lib, self.lib.asarf_plan_dims(self._h, C.byref(d)), "plan_dims")
        self.dims = {f: (list(getattr(d, f)) if f in ("out_rows", "out_cols", "vr_poly") else getattr(d, f))
                     for f, _ in d._fields_}

    @classmethod
    def _wrap(cls, lib, handle, scene, owner):
        """A view of a plan owned by someone else (a batch): never destroyed through this object."""
        self = cls.__new__(cls)
        self.lib, self.scene, self._h, self._owner = lib, scene, handle, owner
        self.product = _lib.PRODUCT_DETECTED
        d = _lib.Dims()
        _lib.check(lib, lib.asarf_plan_dims(handle, C.byref(d)), "plan_dims")
        self.dims = {f: (list(getattr(d, f)) if f in ("out_rows", "out_cols", "vr_poly") else getattr(d, f))
                     for f, _ in d._fields_}
        return self

    def close(self):
        if getattr(self, "_owner", None) is not None:
            self._h = None
            return
        if getattr(self, "_h", None):
            self.lib.asarf_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def out_shape(self) -> tuple:
        """Shape of the output buffer: float32 [out_rows_max, out_cols_max] for the detected
        image, uint8 [out_bytes_max] for level-1 MDS records."""
        if self.product:
            return (self.dims["out_bytes_max"],)
        return self.dims["out_rows_max"], self.dims["out_cols_max"]

    @property
    def out_dtype(self):
        return np.uint8 if self.product else np.float32

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
        out = np.empty(self.out_shape, dtype=self.out_dtype)
        _lib.check(self.lib, self.lib.asarf_focus_host(self._h, raw.ctypes.data, _ptr(sw), mn, out.ctypes.data,
                                                       C.c_void_p(stream)), "focus_host")
        r = self.results(stream)
        if self.product:
            return out[: r["records"] * r["record_bytes"]].reshape(r["records"], r["record_bytes"])
        return out[: r["out_rows"], : r["out_cols"]]

    def focus_host_ptr(self, raw_ptr: int, out_ptr: int, swst_ptr: int = 0, min_swst: int = 0, stream: int = 0):
        """asarf_focus_host on raw host pointers (e.g. pinned torch tensors); synchronous."""
        _lib.check(self.lib, self.lib.asarf_focus_host(self._h, raw_ptr, swst_ptr or None, int(min_swst), out_ptr,
                                                       C.c_void_p(stream)), "focus_host")

    def focus_host_async(self, raw_ptr: int, out_ptr: int, swst_ptr: int = 0, min_swst: int = 0, stream: int = 0):
        """asarf_focus_host_async: enqueue upload, focus and download and return at once
        (stream 0: the plan's own non-blocking stream).  Host buffers should be pinned and
        stay untouched until ``wait()``."""
        _lib.check(self.lib, self.lib.asarf_focus_host_async(self._h, raw_ptr, swst_ptr or None, int(min_swst),
                                                             out_ptr, C.c_void_p(stream)), "focus_host_async")

    def wait(self):
        """asarf_plan_wait: block until this plan's enqueued host runs have finished."""
        _lib.check(self.lib, self.lib.asarf_plan_wait(self._h), "plan_wait")

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


def lpt_assign(work, bins: int, lib=None) -> list[int]:
    """Longest-processing-time assignment of work items to bins (asarf_lpt_assign): the rule
    that deals batch segments to graph branches and to GPUs."""
    lib = lib or load_library()
    n = len(work)
    w = (C.c_int64 * n)(*[int(v) for v in work])
    out = (C.c_int32 * max(n, 1))()
    _lib.check(lib, lib.asarf_lpt_assign(w, n, int(bins), out), "lpt_assign")
    return [int(out[i]) for i in range(n)]


class FocusBatch:
    """Independent segments of uneven size focused together (asarf_batch): every segment's
    kernels in one CUDA graph with concurrent branches, replayed on later calls with the same
    buffers.  ``plans[i]`` is segment i's plan (dims, results, SLC)."""

    def __init__(self, scenes, branches: int = 4, ref_compat_stats: bool = True, lib=None, lib_path=None,
                 precision: int = 0, options=None):
        """``options``: per-segment dicts of launch shapes (az_n2, az_tile_width,
        strided_tile_width, rc_fft_len), e.g. from asarf.autotune.tune."""
        self.lib = lib or load_library(lib_path)
        self.scenes = list(scenes)
        n = len(self.scenes)
        for sc in self.scenes:
            if sc.vr_poly is None or not sc.osv:
                sc.prepare(self.lib)
        self._keep = [sc.to_c() for sc in self.scenes]
        arr = (_lib.SceneC * n)(*[k[0] for k in self._keep])
        opts = (_lib.Options * n)()
        for i in range(n):
            self.lib.asarf_default_options(C.byref(opts[i]))
            opts[i].ref_compat_stats = int(bool(ref_compat_stats))
            opts[i].precision = int(precision)
            for k, v in ((options[i] if options else None) or {}).items():
                if k in ("az_n2", "az_tile_width", "strided_tile_width", "rc_fft_len", "precision", "keep_slc",
                         "compiled_schedules"):
                    setattr(opts[i], k, int(v))
        h = C.c_void_p()
        _lib.check(self.lib, self.lib.asarf_batch_create(arr, n, C.cast(opts, C.c_void_p), int(branches), C.byref(h)),
                   "batch_create")
        self._h = h
        self.plans = []
        for i in range(n):
            ph = C.c_void_p()
            _lib.check(self.lib, self.lib.asarf_batch_plan(self._h, i, C.byref(ph)), "batch_plan")
            self.plans.append(FocusPlan._wrap(self.lib, ph, self.scenes[i], self))
        self.branches = [int(self.lib.asarf_batch_branch(self._h, i)) for i in range(n)]

    def close(self):
        if getattr(self, "_h", None):
            for p in self.plans:
                p.close()
            self.lib.asarf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def focus(self, raws, outs, swsts=None, min_swst=None, stream: int = 0):
        """Asynchronous focus of every segment: raws[i] (device raw bytes) -> outs[i] (float32
        [out_rows_max, out_cols_max] of plans[i])."""
        n = len(self.plans)
        r = (C.c_void_p * n)(*[_ptr(x) for x in raws])
        o = (C.c_void_p * n)(*[_ptr(x) for x in outs])
        sw = C.cast((C.c_void_p * n)(*[_ptr(x) for x in swsts]), C.c_void_p) if swsts is not None else None
        mn = C.cast((C.c_int32 * n)(*[int(v) for v in min_swst]), C.c_void_p) if min_swst is not None else None
        _lib.check(self.lib, self.lib.asarf_batch_focus(self._h, r, sw, mn, o, C.c_void_p(stream)), "batch_focus")
        return outs


class FocusStrip:
    """A long strip focused as overlapped azimuth blocks (asarf_strip): per-block statistics,
    Doppler estimate and Vr, one strip SLC, one multilook/RSL/SRGR pass over the strip."""

    def __init__(self, scene: Scene, block_lines: int = 16384, overlap: int = 1400, ref_compat_stats: bool = True,
                 lib=None, lib_path=None):
        self.lib = lib or load_library(lib_path)
        self.scene = scene
        if scene.vr_poly is None or not scene.osv:
            scene.prepare(self.lib)
        self._sc, self._osv_keep = scene.to_c()
        opt = _lib.Options()
        self.lib.asarf_default_options(C.byref(opt))
        opt.ref_compat_stats = int(bool(ref_compat_stats))
        self._opt = opt
        h = C.c_void_p()
        _lib.check(self.lib, self.lib.asarf_strip_create(C.byref(self._sc), int(block_lines), int(overlap),
                                                         C.cast(C.byref(opt), C.c_void_p), C.byref(h)), "strip_create")
        self._h = h
        d = _lib.StripDims()
        _lib.check(self.lib, self.lib.asarf_strip_get_dims(self._h, C.byref(d)), "strip_dims")
        self.dims = {f: getattr(d, f) for f, _ in d._fields_}
        self.blocks = []
        for k in range(self.dims["n_blocks"]):
            s0, lo, hi, ph = C.c_int32(), C.c_int32(), C.c_int32(), C.c_void_p()
            _lib.check(self.lib, self.lib.asarf_strip_block(self._h, k, C.byref(s0), C.byref(lo), C.byref(hi),
                                                            C.byref(ph)), "strip_block")
            self.blocks.append({"start": s0.value, "keep_lo": lo.value, "keep_hi": hi.value,
                                "plan": FocusPlan._wrap(self.lib, ph, scene, self)})

    def close(self):
        if getattr(self, "_h", None):
            for b in self.blocks:
                b["plan"].close()
            self.lib.asarf_strip_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def out_shape(self) -> tuple[int, int]:
        return self.dims["out_rows"], self.dims["out_cols"]

    def focus(self, raw, out, swst=None, min_swst: int = 0, stream: int = 0):
        _lib.check(self.lib, self.lib.asarf_focus_strip(self._h, _ptr(raw), _ptr(swst), int(min_swst), _ptr(out),
                                                        C.c_void_p(stream)), "focus_strip")
        return out

    def slc_into(self, dst, stream: int = 0):
        """Strip SLC, complex64 [slc_rows, slc_cols]."""
        _lib.check(self.lib, self.lib.asarf_strip_slc(self._h, C.c_void_p(_ptr(dst)), C.c_void_p(stream)), "strip_slc")
        return dst

    def errors(self, stream: int = 0) -> int:
        e = C.c_uint32()
        _lib.check(self.lib, self.lib.asarf_strip_errors(self._h, C.byref(e), C.c_void_p(stream)), "strip_errors")
        return int(e.value)
