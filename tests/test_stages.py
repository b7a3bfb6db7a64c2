"""Per-stage entry points (the reference's sar/ functions one by one) against the oracle's
stage functions on the same inputs.

Each test runs twice: on the host-emulation build of the kernel bodies (CPU, numpy arrays)
and, under ``-m gpu``, on the CUDA library (torch CUDA tensors).  The last test chains all
stages as the reference's main flow does and compares the detected image with the
planned (fused) path and with the oracle's whole chain.
"""
from __future__ import annotations

import numpy as np
import pytest

from asarf import scene as S
from asarf import stages as st
from conftest import oracle_focus, rel_rmse, scene_and_raw
from oracle import geometry as geo
from oracle import rda


class Backend:
    def __init__(self, lib, gpu: bool):
        self.lib = lib
        self.gpu = gpu

    def dev(self, a: np.ndarray):
        if not self.gpu:
            return np.ascontiguousarray(a).copy()
        import torch
        return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")

    def host(self, x) -> np.ndarray:
        if not self.gpu:
            return np.asarray(x).copy()
        return x.cpu().numpy()

    def empty(self, shape, dtype):
        return self.dev(np.zeros(shape, dtype=dtype))


@pytest.fixture(params=["emu", pytest.param("gpu", marks=pytest.mark.gpu)])
def be(request):
    if request.param == "emu":
        return Backend(request.getfixturevalue("emu_lib"), False)
    return Backend(request.getfixturevalue("gpu_lib"), True)


def _scene(be, **kw):
    sc, raw, _ = scene_and_raw(be.lib, S.tiny, **kw)
    return sc, raw


def _padded_decoded(sc, raw):
    d = sc.to_dict()
    rg_pad, az_pad = geo.reference_padding(sc.range_size, sc.chirp_samples, sc.azimuth_size)
    data = rda.decode_ers(raw, sc.samples_per_line, d.get("swst"), sc.range_size)
    return rda.pad_image(data, rg_pad, az_pad)


def _corrected(sc, raw):
    img = _padded_decoded(sc, raw)
    iq = rda.raw_data_correction(img, sc.range_size, sc.azimuth_size, sc.samples_per_line * sc.azimuth_size)
    rda.zero_nans(img)
    return img, iq


def _same_nan(a, b):
    return np.array_equal(np.isnan(a.real), np.isnan(b.real)) and np.array_equal(np.isnan(a.imag), np.isnan(b.imag))


def test_convert_ers_samples(be):
    sc, raw = _scene(be)
    rg_pad, az_pad = geo.reference_padding(sc.range_size, sc.chirp_samples, sc.azimuth_size)
    swst = np.asarray(sc.swst_codes, dtype=np.uint16) if sc.swst_codes is not None else None
    img = be.empty((az_pad, rg_pad), np.complex64)
    st.convert_ers_samples(be.dev(raw), sc.samples_per_line, img, sc.range_size,
                           swst=None if swst is None else be.dev(swst),
                           min_swst=0 if swst is None else int(swst.min()), lib=be.lib)
    got = be.host(img)[: sc.azimuth_size, : sc.range_size]
    ref = rda.decode_ers(raw, sc.samples_per_line, None if swst is None else swst, sc.range_size)
    assert _same_nan(got, ref)
    m = ~np.isnan(ref)
    assert np.array_equal(got[m], ref[m])
    assert not np.any(be.host(img)[: sc.azimuth_size, sc.range_size:])


def test_convert_ers_samples_swst_shift(be):
    """Lines with a later sampling window start shift right by 4 samples per SWST code."""
    sc, raw = _scene(be)
    na = sc.azimuth_size
    swst = (100 + (np.arange(na) // 37) % 3).astype(np.uint16)
    nr = sc.samples_per_line + 4 * 2
    img = be.empty((na, nr + 8), np.complex64)
    st.convert_ers_samples(be.dev(raw), sc.samples_per_line, img, nr, swst=be.dev(swst), min_swst=100, lib=be.lib)
    got = be.host(img)[:, :nr]
    ref = rda.decode_ers(raw, sc.samples_per_line, swst, nr)
    assert _same_nan(got, ref)
    m = ~np.isnan(ref)
    assert np.array_equal(got[m], ref[m])


def test_raw_data_correction_and_zero_nans(be):
    sc, raw = _scene(be)
    img0 = _padded_decoded(sc, raw)
    ref = img0.copy()
    iq = rda.raw_data_correction(ref, sc.range_size, sc.azimuth_size, sc.samples_per_line * sc.azimuth_size)
    rda.zero_nans(ref)
    dimg = st.DevicePaddedImage(be.dev(img0), sc.range_size, sc.azimuth_size)
    res = st.raw_data_correction(dimg, sc.samples_per_line * sc.azimuth_size, lib=be.lib)
    st.zero_nans(dimg, lib=be.lib)
    assert res["dc_i"] == pytest.approx(iq.dc_i, rel=2e-7)
    assert res["dc_q"] == pytest.approx(iq.dc_q, rel=2e-7)
    assert res["stddev_i"] == pytest.approx(iq.stddev_i, rel=2e-7)
    assert res["stddev_q"] == pytest.approx(iq.stddev_q, rel=2e-7)
    assert res["iq_gain"] == pytest.approx(iq.iq_gain, rel=1e-7)
    assert res["phase_error"] == pytest.approx(iq.phase_error, abs=1e-4)
    got = be.host(dimg.data)
    assert not np.isnan(got).any()
    # the constants agree to float rounding, so the samples agree to a few ulp
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.max(np.abs(ref))
    assert not np.any(got[sc.azimuth_size:])


def test_doppler_centroid(be):
    sc, raw = _scene(be)
    img, _ = _corrected(sc, raw)
    poly_ref, _, _ = rda.doppler_centroid(img, sc.range_size, sc.azimuth_size, sc.prf)
    dimg = st.DevicePaddedImage(be.dev(img), sc.range_size, sc.azimuth_size)
    poly = st.calculate_doppler_centroid(dimg, sc.prf, lib=be.lib)
    assert np.allclose(poly, poly_ref, rtol=1e-6, atol=1e-9)
    assert poly[2] == pytest.approx(poly_ref[2], rel=1e-7, abs=1e-4)


def test_range_compression(be):
    sc, raw = _scene(be)
    img, _ = _corrected(sc, raw)
    rg_pad = img.shape[1]
    chirp = rda.generate_chirp(sc.chirp_kr, sc.range_sampling_rate, sc.chirp_samples, sc.apply_window, rg_pad)
    dimg = st.DevicePaddedImage(be.dev(img), sc.range_size, sc.azimuth_size)
    ref = img.copy()
    nk_ref = rda.range_compression(ref, sc.azimuth_size, sc.range_size, chirp, sc.chirp_samples)
    nk = st.range_compression(dimg, chirp, sc.chirp_samples, lib=be.lib)
    assert nk == nk_ref == dimg.x_size
    got = be.host(dimg.data)
    na = sc.azimuth_size
    assert rel_rmse(got[:na, :nk], ref[:na, :nk]) < 2e-6
    assert not np.any(got[:na, nk:])


def test_range_compression_rejects_chirp_size(be):
    sc, raw = _scene(be)
    img, _ = _corrected(sc, raw)
    chirp = np.zeros(img.shape[1] - 2, np.complex64)
    dimg = st.DevicePaddedImage(be.dev(img), sc.range_size, sc.azimuth_size)
    with pytest.raises(Exception, match="Range padding and chirp size mismatch"):
        st.range_compression(dimg, chirp, sc.chirp_samples, lib=be.lib)


def _rc_image(sc, raw):
    img, _ = _corrected(sc, raw)
    chirp = rda.generate_chirp(sc.chirp_kr, sc.range_sampling_rate, sc.chirp_samples, sc.apply_window, img.shape[1])
    dc_poly, _, _ = rda.doppler_centroid(img, sc.range_size, sc.azimuth_size, sc.prf)
    nk = rda.range_compression(img, sc.azimuth_size, sc.range_size, chirp, sc.chirp_samples)
    return img, nk, dc_poly


def test_range_doppler(be):
    sc, raw = _scene(be)
    img, nk, dc_poly = _rc_image(sc, raw)
    na = sc.azimuth_size
    args = rda.RdaArgs(sc.prf, sc.wavelength, sc.az_bw_frac, sc.range_spacing, sc.slant_range_first, dc_poly,
                       np.asarray(sc.vr_poly))
    ref = rda.range_doppler(img.copy(), nk, na, args)
    src = st.DevicePaddedImage(be.dev(img), nk, na)
    out = st.range_doppler_algorithm(sc.prf, sc.wavelength, sc.range_spacing, sc.slant_range_first, sc.az_bw_frac,
                                     sc.vr_poly, dc_poly, src, be.empty(img.shape, np.complex64), lib=be.lib)
    got = be.host(out.data)
    assert rel_rmse(got[:na, :nk], ref[:na, :nk]) < 1e-5
    assert not np.any(got[na:]) and not np.any(got[:, nk:])


def test_multilook_rsl_srgr(be):
    sc, raw = _scene(be)
    ref = oracle_focus(sc, raw)
    slc = np.ascontiguousarray(ref.slc)
    ml_ref, _ = rda.azimuth_multilook(slc, sc.azimuth_spacing)
    ny_max = int(np.ceil(slc.shape[0] / float(np.float32(12.5 / sc.azimuth_spacing)))) + 1
    ml = be.empty((ny_max, slc.shape[1]), np.float32)
    ny = st.azimuth_multilook(be.dev(slc), sc.azimuth_spacing, ml, lib=be.lib)
    assert ny == ml_ref.shape[0]
    got = be.host(ml)[:ny]
    assert rel_rmse(got, ml_ref) < 1e-6

    # range spreading loss on the reference's multilooked image: float product, bit-exact gains
    sub_first = sc.slant_range_first + ref.window["near"] * sc.range_spacing
    ml_d = be.dev(ml_ref)
    st.range_spreading_loss_correction(ml_d, sub_first, sc.range_spacing, geo.REFERENCE_RANGE, lib=be.lib)
    rsl = geo.rsl_table(ml_ref.shape[1], sub_first, sc.range_spacing)
    assert np.allclose(be.host(ml_d), (ml_ref * rsl[None, :]).astype(np.float32), rtol=2e-7, atol=0)

    # SRGR: index map bit-exact, interpolation to float rounding
    ng = ref.detected.shape[1]
    start = be.empty((ng,), np.int32)
    frac = be.empty((ng,), np.float32)
    st.srgr_index(ref.grsr_poly, sc.range_spacing, start, frac, lib=be.lib)
    assert np.array_equal(be.host(start), ref.srgr_start)
    assert np.array_equal(be.host(frac), ref.srgr_frac)
    det = be.empty(ref.detected.shape, np.float32)
    st.srgr_interpolation(be.dev(ref.ml), ref.grsr_poly, sc.range_spacing, det, lib=be.lib)
    assert rel_rmse(be.host(det), ref.detected) < 1e-6


def test_stage_chain_matches_planned_path(be):
    """decode -> correction -> ZeroNaNs -> DC -> RC -> RDA -> window -> multilook -> RSL ->
    SRGR through the per-stage calls, as main.cc strings them, equals the planned path."""
    import asarf

    sc, raw = _scene(be)
    d = sc.to_dict()
    na, nr, nc = sc.azimuth_size, sc.range_size, sc.chirp_samples
    rg_pad, az_pad = geo.reference_padding(nr, nc, na)
    img = be.empty((az_pad, rg_pad), np.complex64)
    st.convert_ers_samples(be.dev(raw), sc.samples_per_line, img, nr, lib=be.lib)
    p = st.DevicePaddedImage(img, nr, na)
    res = st.raw_data_correction(p, sc.samples_per_line * na, lib=be.lib)
    st.zero_nans(p, lib=be.lib)
    dc_poly = st.calculate_doppler_centroid(p, sc.prf, lib=be.lib)
    chirp = np.empty(rg_pad, np.complex64)
    chirp[:] = rda.generate_chirp(sc.chirp_kr, sc.range_sampling_rate, nc, sc.apply_window, rg_pad)
    nk = st.range_compression(p, chirp, nc, lib=be.lib)
    out = st.range_doppler_algorithm(sc.prf, sc.wavelength, sc.range_spacing, sc.slant_range_first, sc.az_bw_frac,
                                     sc.vr_poly, dc_poly, p, be.empty((az_pad, rg_pad), np.complex64), lib=be.lib)
    ap = geo.calc_aperture_pixels(sc.carrier_frequency, d["vr_poly_init"], [], sc.prf, sc.az_bw_frac,
                                  sc.slant_range_first, sc.range_spacing, nr, nc)
    win = geo.results_window(dc_poly[2], sc.lines_before, sc.lines_after, max(ap))
    first, last = win["first_line"], na - win["drop_end"]
    slc_h = be.host(out.data)[first:last, win["near"]: nk - win["far"]]
    slc = be.dev(np.ascontiguousarray(slc_h))
    ny_max = int(np.ceil(slc_h.shape[0] / float(np.float32(12.5 / sc.azimuth_spacing)))) + 1
    ml = be.empty((ny_max, slc_h.shape[1]), np.float32)
    ny = st.azimuth_multilook(slc, sc.azimuth_spacing, ml, lib=be.lib)
    ml_h = np.ascontiguousarray(be.host(ml)[:ny])
    ml = be.dev(ml_h)
    sub_first = sc.slant_range_first + win["near"] * sc.range_spacing
    st.range_spreading_loss_correction(ml, sub_first, sc.range_spacing, geo.REFERENCE_RANGE, lib=be.lib)

    plan = asarf.FocusPlan(sc, lib=be.lib)
    planned = plan.focus_host(raw)
    pr = plan.results()
    assert pr["first_line"] == first
    ng = planned.shape[1]
    ratio = float(np.float32(12.5 / sc.azimuth_spacing))
    grsr, ng2 = st.srgr_polynomial(sc, sub_first, slc_h.shape[1], ny, (1.0 / sc.prf) * ratio, lib=be.lib)
    assert ng2 == ng
    det = be.empty((ny, ng), np.float32)
    st.srgr_interpolation(ml, grsr, sc.range_spacing, det, lib=be.lib)
    det_h = be.host(det)
    assert det_h.shape == planned.shape
    assert rel_rmse(det_h, planned) < 1e-5
    assert rel_rmse(det_h, oracle_focus(sc, raw).detected) < 1e-5
    assert res["iq_gain"] == pytest.approx(pr["iq_gain"], rel=1e-6)
