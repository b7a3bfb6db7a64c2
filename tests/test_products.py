"""Level-1 products: the IMS (complex SLC) and IMP (detected) MDS record encodings of
ConditionResultsSLC / ConditionResultsDetected (envisat_format/src/envisat_format_kernels.cu:28-114),
as per-stage entry points and fused into the focus run (asarf_options.product), and the
product statistics main.cc writes into the SQ ADS (CalculateStatistics /
CalculateStatisticsImaged, main_flow.cc:666-676; asarf_options.sq_stats).

CPU: the host-emulation build against the oracle's restatement (IMS bit-exact; IMP exact up to
the last-ulp difference of the two log10 implementations, which moves a count only where
10 log10 lands on an integer); the fused products equal the per-stage conditioning of the
plan's own float image / SLC byte for byte; the statistics match the oracle's on the plan's own
image and SLC.  GPU: the CUDA kernels against the reference's own conditioning functions
compiled from its sources, bit for bit, special values included; the fused products and the
statistics on the device, the latter also against the reference chain's own statistics.
"""
from __future__ import annotations

import numpy as np
import pytest

import asarf
from asarf import scene as S
from asarf import stages as st
from conftest import scene_and_raw
from oracle import rda

HDR = 17
CAL = 3.7


def _special_complex(rng, y=23, stride=61, x=57):
    img = (rng.standard_normal((y, stride)) * 4000 + 1j * rng.standard_normal((y, stride)) * 4000).astype(np.complex64)
    img[0, :6] = [np.nan, 1e9, -1e9, 8855.9, -8855.9, 0.26]
    img[1, :4] = [complex(np.nan, 1.0), complex(-0.27, np.nan), complex(8856.5, -8856.6), complex(-0.0, 0.0)]
    return img, x


def _special_float(rng, y=19, x=53):
    img = (rng.exponential(1.0, (y, x)) * 10.0 ** rng.uniform(-4, 6, (y, x))).astype(np.float32)
    img[0, :8] = [0.0, -1.0, np.nan, np.inf, 1.0 / CAL, 10.0 / CAL, 1e30, 100.0 / CAL]
    return img


def _dev(gpu, a):
    if not gpu:
        return np.ascontiguousarray(a).copy()
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _host(gpu, x):
    return np.asarray(x).copy() if not gpu else x.cpu().numpy()


@pytest.fixture(params=["emu", pytest.param("gpu", marks=pytest.mark.gpu)])
def be(request):
    if request.param == "emu":
        return request.getfixturevalue("emu_lib"), False
    return request.getfixturevalue("gpu_lib"), True


def test_condition_slc_matches_oracle(be):
    lib, gpu = be
    img, x = _special_complex(np.random.default_rng(1))
    dest = _dev(gpu, np.full((img.shape[0], HDR + 4 * x), 0xAB, dtype=np.uint8))
    st.condition_slc(_dev(gpu, img), x, dest, HDR, CAL, lib=lib)
    got = _host(gpu, dest)
    ref = rda.condition_slc(img[:, :x], CAL, HDR)
    assert np.array_equal(got, ref)
    assert not got[:, :HDR].any()


def test_condition_detected_matches_oracle(be):
    lib, gpu = be
    img = _special_float(np.random.default_rng(2))
    dest = _dev(gpu, np.full((img.shape[0], HDR + 2 * img.shape[1]), 0xAB, dtype=np.uint8))
    st.condition_detected(_dev(gpu, img), dest, HDR, CAL, lib=lib)
    got = _host(gpu, dest)
    ref = rda.condition_detected(img, CAL, HDR)
    assert not got[:, :HDR].any()
    g = got[:, HDR:].reshape(img.shape[0], -1, 2).astype(np.int64)
    r = ref[:, HDR:].reshape(img.shape[0], -1, 2).astype(np.int64)
    gv, rv = g[..., 0] | g[..., 1] << 8, r[..., 0] | r[..., 1] << 8
    assert np.abs(gv - rv).max() <= 1 and np.count_nonzero(gv != rv) <= 2
    assert list(gv[0, :4]) == [0, 0, 0, 65535]


def _detected_and_slc(lib, gpu, sc, raw):
    det = asarf.FocusPlan(sc, lib=lib)
    if gpu:
        import torch
        d_raw = torch.from_numpy(raw).cuda()
        out = torch.zeros(det.out_shape, dtype=torch.float32, device="cuda")
        det.focus(d_raw, out)
        torch.cuda.synchronize()
        res = det.results()
        image = out[: res["out_rows"], : res["out_cols"]].contiguous()
        slc = torch.empty((res["n_lines"], det.dims["slc_cols"]), dtype=torch.complex64, device="cuda")
        det.slc_into(slc)
        torch.cuda.synchronize()
    else:
        image = np.ascontiguousarray(det.focus_host(raw))
        res = det.results()
        slc = np.empty((res["n_lines"], det.dims["slc_cols"]), dtype=np.complex64)
        det.slc_into(slc)
    return det, res, image, slc


def test_fused_products_equal_per_stage_conditioning(be):
    lib, gpu = be
    sc, raw, _ = scene_and_raw(lib, S.tiny)
    det, res, image, slc = _detected_and_slc(lib, gpu, sc, raw)
    want_imp = _dev(gpu, np.zeros((res["out_rows"], HDR + 2 * res["out_cols"]), dtype=np.uint8))
    st.condition_detected(image, want_imp, HDR, CAL, lib=lib)
    want_ims = _dev(gpu, np.zeros((res["n_lines"], HDR + 4 * det.dims["slc_cols"]), dtype=np.uint8))
    st.condition_slc(slc, det.dims["slc_cols"], want_ims, HDR, CAL, lib=lib)
    imp = asarf.FocusPlan(sc, lib=lib, product=1, calibration=CAL)
    ims = asarf.FocusPlan(sc, lib=lib, product=2, calibration=CAL)
    got_imp = imp.focus_host(raw)
    got_ims = ims.focus_host(raw)
    assert imp.results()["record_bytes"] == HDR + 2 * res["out_cols"]
    assert ims.results()["records"] == res["n_lines"]
    assert np.array_equal(got_imp, _host(gpu, want_imp))
    assert np.array_equal(got_ims, _host(gpu, want_ims))
    assert imp.dims["out_bytes_max"] >= got_imp.size and ims.dims["out_bytes_max"] >= got_ims.size


def test_product_statistics_match_oracle(be):
    lib, gpu = be
    sc, raw, _ = scene_and_raw(lib, S.tiny)
    det, res, image, slc = _detected_and_slc(lib, gpu, sc, raw)
    image, slc = _host(gpu, image), _host(gpu, slc)
    want_imp = rda.product_statistics_imp(image, slc, CAL)
    want_ims = rda.product_statistics_ims(slc, CAL)
    for product, want in ((0, want_imp), (1, want_imp), (2, want_ims)):
        p = asarf.FocusPlan(sc, lib=lib, product=product, calibration=CAL, sq_stats=True)
        p.focus_host(raw)
        got = np.array(p.results()["sq_stats"])
        assert np.allclose(got, want, rtol=2e-6, atol=1e-9), (product, got, want)
    # the IMP form includes SLC floats: its mean differs from the image's own mean
    assert abs(want_imp[0] / CAL - float(image.mean())) > 1e-4 * abs(float(image.mean()))


def test_unknown_product_rejected(emu_lib):
    sc, raw, _ = scene_and_raw(emu_lib, S.tiny)
    with pytest.raises(asarf.AsarfError):
        asarf.FocusPlan(sc, lib=emu_lib, product=5)


@pytest.mark.gpu
def test_conditioning_matches_reference_kernels(gpu_lib):
    import torch
    from oracle import ref_lib
    if not ref_lib.available():
        pytest.fail("reference build oracle/_ref/libasar_ref.so missing")
    rng = np.random.default_rng(5)
    img, x = _special_complex(rng, y=64, stride=530, x=517)
    dest = torch.zeros((img.shape[0], HDR + 4 * x), dtype=torch.uint8, device="cuda")
    st.condition_slc(torch.from_numpy(img).cuda(), x, dest, HDR, CAL, lib=gpu_lib)
    assert np.array_equal(dest.cpu().numpy(), ref_lib.ref_condition_slc(img, x, HDR, CAL))
    fimg = _special_float(rng, y=71, x=1031)
    fdest = torch.zeros((fimg.shape[0], HDR + 2 * fimg.shape[1]), dtype=torch.uint8, device="cuda")
    st.condition_detected(torch.from_numpy(fimg).cuda(), fdest, HDR, CAL, lib=gpu_lib)
    assert np.array_equal(fdest.cpu().numpy(), ref_lib.ref_condition_detected(fimg, HDR, CAL))


@pytest.mark.gpu
def test_product_statistics_match_reference_chain(gpu_lib):
    from oracle import ref_lib
    if not ref_lib.available():
        pytest.fail("reference build oracle/_ref/libasar_ref.so missing")
    sc, raw, _ = scene_and_raw(gpu_lib, S.ers_small)
    ref_lib.set_statistics(True)
    try:
        scc, keep = sc.to_c()
        _, r, _ = ref_lib.ref_focus(scc, sc.vr_poly, raw)
    finally:
        ref_lib.set_statistics(False)
    imp = asarf.FocusPlan(sc, lib=gpu_lib, product=1, sq_stats=True)
    ims = asarf.FocusPlan(sc, lib=gpu_lib, product=2, sq_stats=True)
    imp.focus_host(raw)
    ims.focus_host(raw)
    # the reference sums in float per block: agreement to its rounding
    got_imp, got_ims = np.array(imp.results()["sq_stats"]), np.array(ims.results()["sq_stats"])
    assert np.allclose(got_imp, r["imp_stats"], rtol=1e-4, atol=1e-5 * np.abs(got_imp).max())
    # IMS means are near zero: compare them on the scale of the deviations
    assert np.allclose(got_ims, r["ims_stats"], rtol=1e-4, atol=1e-5 * np.abs(got_ims).max())
