"""sm_100a focusing path (C ABI, libasarf.so) against the CPU oracle and the reference's
own CUDA build, on a B200."""
from __future__ import annotations

import numpy as np
import pytest

import asarf
from asarf import scene as S
from conftest import oracle_focus, rel_rmse, scene_and_raw

pytestmark = pytest.mark.gpu

TOL_DETECTED = 1e-5   # relative RMSE of detected intensity
TOL_SLC = 1e-5        # relative RMSE of the complex SLC


def _focus(lib, sc, raw, **kw):
    swst = kw.pop("swst", None)
    plan = asarf.FocusPlan(sc, lib=lib, **kw)
    out = plan.focus_host(raw, swst)
    return plan, out, plan.results()


def _slc(plan, res):
    import torch
    d = torch.empty((res["n_lines"], plan.dims["slc_cols"]), dtype=torch.complex64, device="cuda")
    plan.slc_into(d, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return d.cpu().numpy()


def asar_small(**kw):
    """The ENVISAT ASAR IM-like parameter set (8-bit I/Q, 27.1 us / 16 MHz chirp, PRF 1652,
    quadratic Doppler) on a 4096-line cut."""
    base = dict(azimuth_size=4096, grid=(4, 4))
    base.update(kw)
    return S.asar_im(**base)


def tiny_nine(**kw):
    """The small scene on 1200 lines: azimuth FFT 1215 = 45 x 27, strided pass radices [9, 5]."""
    base = dict(azimuth_size=1200, seed=13)
    base.update(kw)
    return S.tiny(**base)


@pytest.mark.parametrize("factory", [S.tiny, S.ers_small, asar_small, tiny_nine])
def test_matches_oracle(gpu_lib, factory):
    sc, raw, _ = scene_and_raw(gpu_lib, factory)
    plan, out, res = _focus(gpu_lib, sc, raw)
    ref = oracle_focus(sc, raw)
    assert res["errors"] == 0
    assert res["first_line"] == ref.window["first_line"]
    assert abs(res["dc_i"] - ref.iq.dc_i) <= 1e-6 * ref.iq.dc_i
    assert abs(res["iq_gain"] - ref.iq.iq_gain) <= 1e-6
    assert abs(res["phase_error"] - ref.iq.phase_error) <= 1e-5
    assert np.allclose(res["doppler_centroid_poly"][2], ref.dc_poly[2], rtol=1e-6)
    assert out.shape == ref.detected.shape
    assert rel_rmse(out, ref.detected) < TOL_DETECTED
    assert rel_rmse(_slc(plan, res), ref.slc) < TOL_SLC


def test_variants_match_oracle(gpu_lib):
    """SWST shifts (unfilled samples), negative Doppler (other window variant), data-only
    statistics, unwindowed replica."""
    na = 1024
    codes = (np.arange(na) // 300 * 22 + 600).astype(np.uint16)
    sc, raw, _ = scene_and_raw(gpu_lib, S.tiny, swst_codes=codes,
                               range_size=768 + 4 * int(codes.max() - codes.min()), apply_window=False,
                               dc_coeffs=(-350.0,), seed=21)
    for ref_compat in (True, False):
        plan, out, res = _focus(gpu_lib, sc, raw, swst=codes, ref_compat_stats=ref_compat)
        ref = oracle_focus(sc, raw, ref_compat=ref_compat)
        assert res["errors"] == 0
        assert res["variant"] == (0 if ref.dc_poly[2] > 0 else 1)
        assert rel_rmse(out, ref.detected) < TOL_DETECTED


def test_point_target_quality_matches_oracle(gpu_lib):
    """IRF of every point target: resolution within 1 %, PSLR within 0.1 dB, ISLR within
    0.2 dB, peak phase within 1 mrad of the FP64 oracle."""
    from oracle import irf
    sc, raw, truth = scene_and_raw(gpu_lib, S.ers_small)
    plan, out, res = _focus(gpu_lib, sc, raw, ref_compat_stats=False)
    ref = oracle_focus(sc, raw, ref_compat=False)
    slc = _slc(plan, res)
    first = res["first_line"]
    n = 0
    for (xt, yt) in truth["targets"]:
        y, x = yt - first, xt - 8
        if not (40 <= y < slc.shape[0] - 40 and 40 <= x < slc.shape[1] - 40):
            continue
        # locate the focused peak in the oracle image (azimuth position depends on the DC convention)
        lo, hi = int(max(0, y - 400)), int(min(slc.shape[0], y + 400))
        blk = np.abs(ref.slc[lo:hi, int(x) - 6:int(x) + 7])
        py, px = np.unravel_index(np.argmax(blk), blk.shape)
        a = irf.analyse(slc, lo + py, int(x) - 6 + px)
        b = irf.analyse(ref.slc, lo + py, int(x) - 6 + px)
        if not a or not b:
            continue
        d = irf.compare(a, b)
        assert d["res_az_rel"] < 0.01 and d["res_rg_rel"] < 0.01, d
        assert d["pslr_az_db"] < 0.1 and d["pslr_rg_db"] < 0.1, d
        assert d["islr_db"] < 0.2, d
        assert d["phase_rad"] < 1e-3, d
        n += 1
    assert n >= 4


def test_host_api_equals_device_api_and_is_deterministic(gpu_lib):
    import torch
    sc, raw, _ = scene_and_raw(gpu_lib, S.tiny)
    plan = asarf.FocusPlan(sc, lib=gpu_lib)
    host = plan.focus_host(raw)
    raw_d = torch.from_numpy(raw).cuda()
    outs = []
    for _ in range(2):
        o = torch.zeros(plan.out_shape, dtype=torch.float32, device="cuda")
        plan.focus(raw_d, o, stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        outs.append(o.cpu().numpy()[: host.shape[0], : host.shape[1]])
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0], host)


@pytest.mark.parametrize("factory", [S.tiny, S.ers_small, asar_small])
def test_matches_reference_build(gpu_lib, factory):
    """Against the reference's own CUDA build (cuFFT) run on this GPU."""
    from oracle import ref_lib
    if not ref_lib.available():
        pytest.fail("reference build oracle/_ref/libasar_ref.so missing")
    sc, raw, _ = scene_and_raw(gpu_lib, factory)
    scc, keep = sc.to_c()
    det, r, _ = ref_lib.ref_focus(scc, sc.vr_poly, raw)
    plan, out, res = _focus(gpu_lib, sc, raw)
    assert (r["first_line"], r["n_lines"]) == (res["first_line"], res["n_lines"])
    assert np.allclose(r["dc_poly"], res["doppler_centroid_poly"], rtol=1e-5, atol=1e-6)
    assert abs(r["iq_gain"] - res["iq_gain"]) < 1e-6
    assert out.shape == det.shape
    assert rel_rmse(out, det) < TOL_DETECTED


def test_full_scene_matches_reference_build_given_its_doppler(gpu_lib):
    """ERS 5616 x 28000: the reference's float ACCC sums put its Doppler polynomial ~1e-5 Hz
    from the exact integer estimate, enough to move a few columns across a Doppler-bin
    rounding boundary; with the reference's own polynomial the images agree to float noise."""
    from oracle import ref_lib
    sc, raw, _ = scene_and_raw(gpu_lib, S.ers_full, device="cuda")
    scc, keep = sc.to_c()
    det, r, _ = ref_lib.ref_focus(scc, sc.vr_poly, raw)
    plan, out, res = _focus(gpu_lib, sc, raw, dc_poly=r["dc_poly"])
    est = res["doppler_centroid_estimate"]
    x = np.arange(0, sc.range_size, 64)
    assert np.max(np.abs(np.polyval(est, x) - np.polyval(r["dc_poly"], x))) < 1e-3  # Hz
    assert res["errors"] == 0
    assert out.shape == det.shape
    assert rel_rmse(out, det) < TOL_DETECTED


@pytest.mark.parametrize("factory", [S.ers_small, asar_small])
def test_detected_only_runs_equal_the_kept_slc_runs(gpu_lib, factory):
    """keep_slc = 0 (the benchmark's detected product): bit-identical image."""
    sc, raw, _ = scene_and_raw(gpu_lib, factory)
    full = asarf.FocusPlan(sc, lib=gpu_lib).focus_host(raw)
    det = asarf.FocusPlan(sc, lib=gpu_lib, keep_slc=False).focus_host(raw)
    assert np.array_equal(det, full)


@pytest.mark.parametrize("lines, n2, bits", [(1990, 125, 2), (3590, 16, 1), (2010, 168, 2), (2870, 16, 1)])
def test_compiled_schedules_equal_run_time_schedules(gpu_lib, lines, n2, bits):
    """Every compiled instantiation (blocks 125 / 168, strided 225 / 180) on the GPU: the same
    image as the run-time schedules, bit for bit."""
    sc, raw, _ = scene_and_raw(gpu_lib, S.tiny, azimuth_size=lines, seed=3)
    outs = []
    for compiled in (True, False):
        plan, out, res = _focus(gpu_lib, sc, raw, az_n2=n2, compiled_schedules=compiled)
        assert plan.dims["compiled_schedules"] == (bits if compiled else 0)
        assert res["errors"] == 0
        outs.append(out)
    assert np.array_equal(outs[0], outs[1])
