"""Argument checks of the C ABI on CPU (host-emulation build): scenes that are empty, too
short or inconsistent, option values out of range, and bad pointers to the focus call are
rejected with ASARF_ERR_INVALID and a message, before any buffer is allocated or any kernel
runs.  The reference checks few of these inside its stages (std::logic_error "Range padding
and chirp size mismatch", sar/range_compression.cu:64; CHECK_BOOL asserts such as
sar/iq_correction.cu:181 and sar/az_multilook.cu:89); the plan checks the scene up front so
that a bad scene never reaches a kernel.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import asarf
from asarf import _lib
from asarf import scene as S

ERR_INVALID = -1


def _create(lib, sc, scene_fields=None, option_fields=None):
    """asarf_plan_create on a prepared scene with some fields overwritten: (status, message)."""
    s, keep = sc.to_c()
    for k, v in (scene_fields or {}).items():
        setattr(s, k, v)
    opt = _lib.Options()
    lib.asarf_default_options(C.byref(opt))
    for k, v in (option_fields or {}).items():
        setattr(opt, k, v)
    h = C.c_void_p()
    rc = lib.asarf_plan_create(C.byref(s), C.byref(opt), C.byref(h))
    msg = lib.asarf_last_error().decode(errors="replace")
    if rc == 0:
        lib.asarf_plan_destroy(h)
    del keep
    return rc, msg


@pytest.fixture(scope="module")
def tiny_scene(emu_lib):
    sc = S.tiny()
    sc.prepare(emu_lib)
    return sc


def test_valid_scene_is_accepted(emu_lib, tiny_scene):
    assert _create(emu_lib, tiny_scene)[0] == 0
    sc = S.tiny(azimuth_size=70)  # the shortest scene whose results window keeps 8 lines
    sc.prepare(emu_lib)
    assert _create(emu_lib, sc)[0] == 0


@pytest.mark.parametrize("fields, text", [
    ({"azimuth_size": 0}, "scene sizes must be positive"),
    ({"azimuth_size": 1}, "scene sizes must be positive"),
    ({"range_size": -5}, "scene sizes must be positive"),
    ({"samples_per_line": 0}, "scene sizes must be positive"),
    ({"samples_per_line": 769}, "exceeds range_size"),
    ({"raw_line_bytes": 1535}, "raw_line_bytes must be even"),
    ({"raw_line_bytes": 1000}, "raw_line_bytes must be even and >= 2*samples_per_line"),
    ({"raw_format": 7}, "unknown raw_format"),
    ({"chirp_samples": 0}, "chirp_samples"),
    ({"chirp_samples": 740}, "chirp_samples"),
    ({"prf": 0.0}, "must be positive"),
    ({"wavelength": float("nan")}, "must be positive"),
    ({"azimuth_spacing": -2.5}, "must be positive"),
    ({"n_osv": 1}, "at least two orbit state vectors"),
])
def test_inconsistent_scenes_are_rejected(emu_lib, tiny_scene, fields, text):
    rc, msg = _create(emu_lib, tiny_scene, scene_fields=fields)
    assert rc == ERR_INVALID, (fields, rc, msg)
    assert text in msg, msg


def test_fbaq_records_need_tables_and_room(emu_lib):
    sc = S.tiny_fbaq()
    sc.prepare(emu_lib)
    assert _create(emu_lib, sc)[0] == 0
    rc, msg = _create(emu_lib, sc, scene_fields={"fbaq_i_lut": None})
    assert rc == ERR_INVALID and "reconstruction tables" in msg
    rc, msg = _create(emu_lib, sc, scene_fields={"raw_line_bytes": 600})
    assert rc == ERR_INVALID and "cannot hold" in msg


def test_scene_shorter_than_one_aperture_is_rejected(emu_lib):
    # the synthetic aperture of this geometry is 62 lines: 66 lines leave a results window of
    # 4 lines, fewer than the 8 a focus needs
    sc = S.tiny(azimuth_size=66)
    sc.prepare(emu_lib)
    rc, msg = _create(emu_lib, sc)
    assert rc == ERR_INVALID and "results window leaves" in msg, msg


@pytest.mark.parametrize("fields, text", [
    ({"rc_fft_len": 512}, "range FFT length"),
    ({"rc_fft_len": 1033}, "range FFT length"),
    ({"az_n2": 7}, "az_n2"),
    ({"az_tile_width": 33}, "az_tile_width must be even"),
    ({"az_tile_width": 128}, "az_tile_width must be even and in [16, 64]"),
    ({"strided_tile_width": 24}, "strided_tile_width must be 16 or 32"),
    ({"product": 9}, "unknown product"),
    ({"record_header_bytes": -1}, "negative record header"),
])
def test_bad_options_are_rejected(emu_lib, tiny_scene, fields, text):
    rc, msg = _create(emu_lib, tiny_scene, option_fields=fields)
    assert rc == ERR_INVALID, (fields, rc, msg)
    assert text in msg, msg


def test_focus_rejects_null_and_misaligned_buffers(emu_lib, tiny_scene):
    plan = asarf.FocusPlan(tiny_scene, lib=emu_lib)
    lib = emu_lib
    raw = np.zeros(tiny_scene.azimuth_size * tiny_scene.raw_line_bytes + 2, np.uint8)
    out = np.zeros(plan.dims["out_bytes_max"] // 4 + 1, np.float32)
    rc = lib.asarf_focus(plan._h, None, None, 0, C.c_void_p(out.ctypes.data), None)
    assert rc == ERR_INVALID and "null argument" in lib.asarf_last_error().decode()
    rc = lib.asarf_focus(plan._h, C.c_void_p(raw.ctypes.data + 1), None, 0, C.c_void_p(out.ctypes.data), None)
    assert rc == ERR_INVALID and "2-byte aligned" in lib.asarf_last_error().decode()
    rc = lib.asarf_focus(None, C.c_void_p(raw.ctypes.data), None, 0, C.c_void_p(out.ctypes.data), None)
    assert rc == ERR_INVALID
    # a rejected call leaves the plan usable
    res = plan.results()
    assert res["errors"] == 0
    plan.close()
