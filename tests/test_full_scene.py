"""Full-size scenes on a B200 against the FP64 oracle and the reference's own CUDA build.

* ERS-like 5616 x 28000 (5-bit I/Q, 20 x 20 point grid, Doppler linear in range, Vr from the
  orbit): the whole detected image and SLC against the oracle run on the whole scene with the
  reference's statistics (padding included), both precision forms; every point target's
  resolution, PSLR, ISLR and peak phase; and the image with the library's own Doppler
  estimate against the reference build.
* ASAR IM-like 5616 x 30000 (8-bit I/Q, quadratic Doppler): the same against the oracle with
  data-only statistics (the other statistics mode), and against the reference build.

* Both: the compile-time transform schedules against the run-time ones, bit for bit.

The oracle runs once per scene (about a minute on the host cores) and is shared by the
tests of that scene.
"""
from __future__ import annotations

import numpy as np
import pytest

import asarf
from asarf import _lib
from asarf import scene as S
from conftest import rel_rmse, scene_and_raw

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-5    # relative RMSE, plain FP32 form
TOL_SPLIT = 1e-4   # relative RMSE, split-precision form

_ORACLE: dict = {}


def _oracle(name, sc, raw, ref_compat):
    from oracle import rda
    key = (name, ref_compat)
    if key not in _ORACLE:
        _ORACLE.clear()  # one full-scene oracle run held at a time
        _ORACLE[key] = rda.focus(raw, sc.to_dict(), ref_compat=ref_compat)
    return _ORACLE[key]


def _focus(lib, sc, raw, **kw):
    import torch
    plan = asarf.FocusPlan(sc, lib=lib, **kw)
    out = plan.focus_host(raw)
    res = plan.results()
    d = torch.empty((res["n_lines"], plan.dims["slc_cols"]), dtype=torch.complex64, device="cuda")
    plan.slc_into(d, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    slc = d.cpu().numpy()
    plan.close()
    return out, slc, res


def _irf_deviations(slc, ref_slc, truth, first):
    from oracle import irf
    worst = {"res": 0.0, "pslr": 0.0, "islr": 0.0, "phase": 0.0}
    n = 0
    for (xt, yt) in truth["targets"]:
        y, x = yt - first, xt - 8
        if not (40 <= y < slc.shape[0] - 40 and 40 <= x < slc.shape[1] - 40):
            continue
        lo, hi = int(max(0, y - 400)), int(min(slc.shape[0], y + 400))
        blk = np.abs(ref_slc[lo:hi, int(x) - 6:int(x) + 7])
        py, px = np.unravel_index(np.argmax(blk), blk.shape)
        a = irf.analyse(slc, lo + py, int(x) - 6 + px)
        b = irf.analyse(ref_slc, lo + py, int(x) - 6 + px)
        if not a or not b:
            continue
        d = irf.compare(a, b)
        worst["res"] = max(worst["res"], d["res_az_rel"], d["res_rg_rel"])
        worst["pslr"] = max(worst["pslr"], d["pslr_az_db"], d["pslr_rg_db"])
        worst["islr"] = max(worst["islr"], d["islr_db"])
        worst["phase"] = max(worst["phase"], d["phase_rad"])
        n += 1
    return n, worst


def _check_against_oracle(gpu_lib, factory, ref_compat):
    sc, raw, truth = scene_and_raw(gpu_lib, factory, device="cuda")
    ref = _oracle(factory.__name__, sc, raw, ref_compat)
    for precision, tol in ((_lib.PRECISION_FP32, TOL_FP32), (_lib.PRECISION_SPLIT, TOL_SPLIT)):
        out, slc, res = _focus(gpu_lib, sc, raw, ref_compat_stats=ref_compat, precision=precision)
        assert res["errors"] == 0
        assert res["first_line"] == ref.window["first_line"]
        assert out.shape == ref.detected.shape
        assert rel_rmse(out, ref.detected) < tol, precision
        assert rel_rmse(slc, ref.slc) < tol, precision
        n, worst = _irf_deviations(slc, ref.slc, truth, res["first_line"])
        assert n >= 300, n
        assert worst["res"] < 0.01 and worst["pslr"] < 0.1 and worst["islr"] < 0.2 and worst["phase"] < 1e-3, \
            (precision, worst)


def test_ers_full_scene_matches_oracle(gpu_lib):
    _check_against_oracle(gpu_lib, S.ers_full, ref_compat=True)


def test_asar_full_scene_matches_oracle_data_only_statistics(gpu_lib):
    _check_against_oracle(gpu_lib, S.asar_im, ref_compat=False)


def _check_against_reference_build(gpu_lib, factory, max_bad_cols):
    """Own Doppler estimate (exact integer lag sums) against the reference's float ACCC: the
    estimates differ by ~1e-5 Hz, which moves the Doppler-bin rounding of at most a few
    range columns; every other column agrees to float noise."""
    from oracle import ref_lib
    if not ref_lib.available():
        pytest.fail("reference build oracle/_ref/libasar_ref.so missing")
    sc, raw, _ = scene_and_raw(gpu_lib, factory, device="cuda")
    scc, keep = sc.to_c()
    det, r, _ = ref_lib.ref_focus(scc, sc.vr_poly, raw)
    out, _, res = _focus(gpu_lib, sc, raw)
    assert (r["first_line"], r["n_lines"]) == (res["first_line"], res["n_lines"])
    assert out.shape == det.shape
    x = np.arange(0, sc.range_size, 64)
    assert np.max(np.abs(np.polyval(res["doppler_centroid_poly"], x) - np.polyval(r["dc_poly"], x))) < 1e-3
    a = out.astype(np.float64)
    b = det.astype(np.float64)
    col_err = np.sqrt(np.sum((a - b) ** 2, axis=0) / np.maximum(np.sum(b ** 2, axis=0), 1e-30))
    bad = np.flatnonzero(col_err > 1e-4)
    assert bad.size <= max_bad_cols, bad
    good = np.setdiff1d(np.arange(out.shape[1]), bad)
    assert rel_rmse(out[:, good], det[:, good]) < TOL_FP32


def test_ers_full_scene_own_doppler_matches_reference_build(gpu_lib):
    _check_against_reference_build(gpu_lib, S.ers_full, max_bad_cols=64)


def test_asar_full_scene_matches_reference_build(gpu_lib):
    _check_against_reference_build(gpu_lib, S.asar_im, max_bad_cols=64)


@pytest.mark.parametrize("factory", [S.ers_full, S.asar_im])
def test_compiled_schedules_equal_run_time_schedules(gpu_lib, factory):
    """The compile-time instantiations of the azimuth transforms (strided 225 / 180, blocks 125
    / 168: both full scenes take both) run the run-time schedules' operations in the same order:
    image and SLC bit-identical with them switched off."""
    sc, raw, _ = scene_and_raw(gpu_lib, factory, device="cuda")
    runs = []
    for compiled in (True, False):
        plan = asarf.FocusPlan(sc, lib=gpu_lib, compiled_schedules=compiled)
        assert plan.dims["compiled_schedules"] == (3 if compiled else 0)
        plan.close()
        runs.append(_focus(gpu_lib, sc, raw, compiled_schedules=compiled))
    (out_a, slc_a, res_a), (out_b, slc_b, res_b) = runs
    assert res_a["errors"] == res_b["errors"] == 0
    assert np.array_equal(out_a, out_b)
    assert np.array_equal(slc_a, slc_b)
