"""The exact kernel bodies (host-emulation build) against the CPU oracle, on CPU.

Same code as the sm_100a kernels (bodies.cuh), run single-threaded; a kernel logic error
shows up here before any GPU time is spent.
"""
from __future__ import annotations

import numpy as np
import pytest

import asarf
from asarf import scene as S
from conftest import oracle_focus, rel_rmse, scene_and_raw

TOL_DETECTED = 1e-5  # relative RMSE of the detected intensity (float32 FFT vs FP64 oracle)


def _run(lib, sc, raw, ref_compat=True, rc_len=0, swst=None):
    plan = asarf.FocusPlan(sc, lib=lib, ref_compat_stats=ref_compat, rc_fft_len=rc_len)
    out = plan.focus_host(raw, swst)
    return plan, out, plan.results()


def _check(plan, out, res, ref):
    assert res["errors"] == 0
    assert res["first_line"] == ref.window["first_line"]
    assert out.shape == ref.detected.shape
    assert abs(res["dc_i"] - ref.iq.dc_i) <= 1e-6 * abs(ref.iq.dc_i)
    assert abs(res["dc_q"] - ref.iq.dc_q) <= 1e-6 * abs(ref.iq.dc_q)
    assert abs(res["iq_gain"] - ref.iq.iq_gain) <= 1e-6
    assert abs(res["phase_error"] - ref.iq.phase_error) <= 1e-5
    assert np.allclose(res["doppler_centroid_poly"][2], ref.dc_poly[2], rtol=1e-6, atol=1e-4)
    assert rel_rmse(out, ref.detected) < TOL_DETECTED


def test_tiny_matches_oracle(emu_lib):
    sc, raw, _ = scene_and_raw(emu_lib, S.tiny)
    plan, out, res = _run(emu_lib, sc, raw)
    _check(plan, out, res, oracle_focus(sc, raw))


def test_data_only_statistics(emu_lib):
    """ref_compat_stats=False: gain/phase sums over the data block only (no padding bias)."""
    sc, raw, _ = scene_and_raw(emu_lib, S.tiny)
    plan, out, res = _run(emu_lib, sc, raw, ref_compat=False)
    ref = oracle_focus(sc, raw, ref_compat=False)
    _check(plan, out, res, ref)
    assert abs(res["phase_error"]) < 5.0   # the true 2 deg skew, not the padding artefact


def test_negative_doppler_window_variant(emu_lib):
    """DC < 0 selects the other results-window variant (lines cut at the end)."""
    sc, raw, _ = scene_and_raw(emu_lib, S.tiny, dc_coeffs=(-350.0,), seed=11)
    plan, out, res = _run(emu_lib, sc, raw, ref_compat=False)
    ref = oracle_focus(sc, raw, ref_compat=False)
    assert ref.dc_poly[2] < 0 and res["variant"] == 1
    _check(plan, out, res, ref)


def tiny_nine(**kw):
    """The small scene on 1200 lines: azimuth FFT 1215 = 45 x 27, strided pass [9, 5]."""
    base = dict(azimuth_size=1200, seed=13)
    base.update(kw)
    return S.tiny(**base)


def test_strided_radix_nine_matches_oracle(emu_lib):
    sc, raw, _ = scene_and_raw(emu_lib, tiny_nine)
    plan, out, res = _run(emu_lib, sc, raw)
    assert plan.dims["n1"] == 45
    _check(plan, out, res, oracle_focus(sc, raw))


def test_range_fft_length_does_not_matter(emu_lib):
    """Any range FFT length >= range size gives the same compressed samples."""
    sc, raw, _ = scene_and_raw(emu_lib, S.tiny)
    _, a, _ = _run(emu_lib, sc, raw, rc_len=768)
    _, b, _ = _run(emu_lib, sc, raw, rc_len=1029)
    assert rel_rmse(a, b) < 1e-5


@pytest.mark.parametrize("ref_compat", [True, False])
def test_swst_shift_and_unwindowed_chirp(emu_lib, ref_compat):
    """Per-line SWST offsets (unfilled samples), a range size that is not a multiple of 32
    (the last Doppler block runs into the range padding) and the unwindowed replica."""
    na = 1024
    codes = (np.arange(na) // 300 * 22 + 600).astype(np.uint16)  # ERS codes step by multiples of 22
    sc, raw, _ = scene_and_raw(emu_lib, S.tiny, swst_codes=codes, range_size=768 + 4 * int(codes.max() - codes.min()),
                               apply_window=False, seed=21)
    assert sc.range_size % 32 != 0
    plan = asarf.FocusPlan(sc, lib=emu_lib, ref_compat_stats=ref_compat)
    out = plan.focus_host(raw, codes)
    res = plan.results()
    ref = oracle_focus(sc, raw, ref_compat=ref_compat)
    _check(plan, out, res, ref)


def test_detected_only_runs_equal_the_kept_slc_runs(emu_lib):
    """keep_slc = 0: the inverse azimuth pass writes |z|^2 rows and the multilook reads them;
    the detected image is bit-identical, and the complex SLC is not offered."""
    from asarf import _lib
    sc, raw, _ = scene_and_raw(emu_lib, S.tiny)
    full = asarf.FocusPlan(sc, lib=emu_lib).focus_host(raw)
    plan = asarf.FocusPlan(sc, lib=emu_lib, keep_slc=False)
    det = plan.focus_host(raw)
    assert np.array_equal(det, full)
    with pytest.raises(_lib.AsarfError):
        plan.slc_into(np.zeros((4, 4), dtype=np.complex64))


# (azimuth lines, az_n2, compiled_schedules bits): scenes whose transforms take each compiled
# instantiation -- blocks 125 = 5*5*5 and 168 = 8*7*3, strided 225 = 9*5*5 and 180 = 9*4*5
COMPILED_CASES = [(1990, 125, 2), (3590, 16, 1), (2010, 168, 2), (2870, 16, 1)]


@pytest.mark.parametrize("lines, n2, bits", COMPILED_CASES)
def test_compiled_schedules_equal_run_time_schedules(emu_lib, lines, n2, bits):
    """The compile-time transform schedules run the same operations in the same order as the
    run-time ones: identical images, and the compiled run matches the oracle."""
    sc, raw, _ = scene_and_raw(emu_lib, S.tiny, azimuth_size=lines, seed=3)
    outs = []
    for compiled in (True, False):
        plan = asarf.FocusPlan(sc, lib=emu_lib, az_n2=n2, compiled_schedules=compiled)
        assert plan.dims["compiled_schedules"] == (bits if compiled else 0)
        outs.append(plan.focus_host(raw))
        assert plan.results()["errors"] == 0
    assert np.array_equal(outs[0], outs[1])
    if lines == 1990:
        assert rel_rmse(outs[0], oracle_focus(sc, raw).detected) < TOL_DETECTED
