"""ENVISAT ASAR FBAQ4 records: the decode fused into the statistics and range-compression
kernels, and the per-stage decode entry point.

Pins: the reference's only known-answer test for this path, the Fbaq4Index table of
envisat_format/unit-test/envisat_parse_util_test.cc:24-85 (code -> level for block 1), checked
against the library, the oracle and the simulator's encoder; the oracle's vectorised decode
against a literal record walk of ConvertAsarImBlocksToComplexKernel; and, on the GPU, the
reference's own ConvertAsarImBlocksToComplex (compiled from its sources) against the oracle
bit for bit, and the reference's whole chain on FBAQ4 records against the fused path.

CPU: the host-emulation build against the oracle (decode bit-exact, statistics and image to
the float32 tolerance of the ERS path).  GPU: the same on the CUDA library, plus run-to-run
reproducibility of the FP64 statistics (fixed-order fold, no atomics).
"""
from __future__ import annotations

import numpy as np
import pytest

import asarf
from asarf import fbaq
from asarf import scene as S
from asarf import stages as st
from conftest import oracle_focus, rel_rmse, scene_and_raw
from oracle import rda

TOL_DETECTED = 1e-5

# Fbaq4Index(1, code) of the reference's unit test: the 4-bit code read as sign-magnitude,
# codes 1111 .. 1000 -> levels 0 .. 7, codes 0000 .. 0111 -> levels 8 .. 15
KAT_LEVEL = {0b1111: 0, 0b1110: 1, 0b1101: 2, 0b1100: 3, 0b1011: 4, 0b1010: 5, 0b1001: 6, 0b1000: 7,
             0b0000: 8, 0b0001: 9, 0b0010: 10, 0b0011: 11, 0b0100: 12, 0b0101: 13, 0b0110: 14, 0b0111: 15}


def _fbaq_scene(lib, factory=S.tiny_fbaq, **kw):
    """A scene with SWST changes and records of different lengths (one partial last block,
    one record shorter by several blocks, one empty record)."""
    base = factory()
    na = base.azimuth_size
    codes = (300 + 3 * ((np.arange(na) // 97) % 4)).astype(np.uint16)
    spl = base.range_size - int(codes.max() - codes.min())
    counts = np.full(na, spl, dtype=np.int64)
    counts[5] = spl - 40
    counts[na // 2] = spl - 3 * 63
    counts[na // 3] = 0
    kw = dict(dict(swst_codes=codes, record_samples=counts), **kw)
    sc, raw, _ = scene_and_raw(lib, factory, **kw)
    return sc, raw


def test_fbaq4_index_known_answers(emu_lib):
    prod = asarf.load_library()
    for code, level in KAT_LEVEL.items():
        want = 256 * level + 1
        assert prod.asarf_fbaq4_index(1, code) == want
        assert emu_lib.asarf_fbaq4_index(1, code) == want
        assert rda.fbaq4_index(1, code) == want
        assert fbaq.table_index(1, code) == want
    blocks, codes = np.meshgrid(np.arange(256), np.arange(16), indexing="ij")
    lib_idx = np.array([[prod.asarf_fbaq4_index(int(b), int(c)) for c in range(16)] for b in range(256)])
    assert np.array_equal(lib_idx, rda.fbaq4_index(blocks, codes))
    assert np.array_equal(fbaq.level_of_code(fbaq.code_of_level(np.arange(16))), np.arange(16))


def _decode_record_walk(raw, swst, range_size, ti, tq):
    """ConvertAsarImBlocksToComplexKernel transcribed as a loop over (record, byte)."""
    na, rec = raw.shape
    out = np.full(na * range_size, complex(np.nan, np.nan), dtype=np.complex64)
    mn = int(min(swst))
    for y in range(na):
        length = int(raw[y, 0]) | (int(raw[y, 1]) << 8)
        for x in range(2, rec):
            j = x - 2
            if j >= length or j % 64 == 0:
                continue
            b = j // 64
            bid = int(raw[y, 2 + 64 * b])
            cw = int(raw[y, x])
            ii, qi = rda.fbaq4_index(bid, cw >> 4), rda.fbaq4_index(bid, cw & 15)
            k = j - (b + 1) + (int(swst[y]) - mn) + y * range_size
            if k < out.size:
                out[k] = complex(ti[ii], tq[qi])
    return out.reshape(na, range_size)


def test_oracle_decode_matches_record_walk():
    rng = np.random.default_rng(3)
    na, spl, rs = 9, 200, 210
    rec = 2 + fbaq.block_bytes(spl)
    raw = rng.integers(0, 256, size=(na, rec), dtype=np.uint8)
    lengths = [fbaq.block_bytes(spl), 0, 1, 64, 65, 130, fbaq.block_bytes(150), rec - 2, rec + 40]
    for y, length in enumerate(lengths):
        raw[y, 0], raw[y, 1] = length & 0xFF, length >> 8
    swst = np.array([5, 5, 6, 9, 5, 7, 15, 5, 5], dtype=np.uint16)
    ti, tq = fbaq.synthetic_tables(1.01)
    got = rda.decode_asar_fbaq(raw, swst, rs, ti, tq)
    ref = _decode_record_walk(raw, swst, rs, ti, tq)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert fbaq.record_samples(fbaq.block_bytes(150)) == 150 and fbaq.record_samples(65) == 63


class _Be:
    def __init__(self, lib, gpu):
        self.lib, self.gpu = lib, gpu

    def dev(self, a):
        if not self.gpu:
            return np.ascontiguousarray(a).copy()
        import torch
        return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")

    def host(self, x):
        return np.asarray(x).copy() if not self.gpu else x.cpu().numpy()


@pytest.fixture(params=["emu", pytest.param("gpu", marks=pytest.mark.gpu)])
def be(request):
    if request.param == "emu":
        return _Be(request.getfixturevalue("emu_lib"), False)
    return _Be(request.getfixturevalue("gpu_lib"), True)


def test_convert_asar_blocks_bit_exact(be):
    sc, raw = _fbaq_scene(be.lib)
    ti, tq = sc.fbaq_tables
    swst = np.asarray(sc.swst_codes, dtype=np.uint16)
    rs = sc.range_size
    img = be.dev(np.zeros((sc.azimuth_size, rs + 24), dtype=np.complex64))
    st.convert_asar_blocks(be.dev(raw), img, rs, be.dev(ti), be.dev(tq), swst=be.dev(swst), min_swst=int(swst.min()),
                           lib=be.lib)
    got = be.host(img)
    ref = rda.decode_asar_fbaq(raw, swst, rs, ti, tq)
    assert np.array_equal(got[:, :rs].view(np.uint32), ref.view(np.uint32))
    assert not np.any(got[:, rs:])
    # the empty record decodes to NaN only
    assert np.all(np.isnan(got[sc.azimuth_size // 3, :rs].real))


def test_focus_matches_oracle(be):
    sc, raw = _fbaq_scene(be.lib)
    swst = np.asarray(sc.swst_codes, dtype=np.uint16)
    plan = asarf.FocusPlan(sc, lib=be.lib)
    out = plan.focus_host(raw, swst)
    res = plan.results()
    ref = oracle_focus(sc, raw)
    assert res["errors"] == 0
    assert res["first_line"] == ref.window["first_line"]
    assert abs(res["dc_i"] - ref.iq.dc_i) <= 1e-6 * abs(ref.iq.dc_i)
    assert abs(res["dc_q"] - ref.iq.dc_q) <= 1e-6 * abs(ref.iq.dc_q)
    assert abs(res["iq_gain"] - ref.iq.iq_gain) <= 1e-6
    assert abs(res["phase_error"] - ref.iq.phase_error) <= 1e-5
    assert abs(res["stddev_i"] - ref.iq.stddev_i) <= 1e-6 * ref.iq.stddev_i
    assert np.allclose(res["doppler_centroid_poly"], ref.dc_poly, rtol=1e-6, atol=1e-6)
    assert out.shape == ref.detected.shape
    assert rel_rmse(out, ref.detected) < TOL_DETECTED


def test_plan_rejects_bad_fbaq_scenes(emu_lib):
    import ctypes as C
    sc, _ = _fbaq_scene(emu_lib)
    c, keep = sc.to_c()
    h = C.c_void_p()
    c.raw_line_bytes = 2 + fbaq.block_bytes(sc.samples_per_line) - 1
    assert emu_lib.asarf_plan_create(C.byref(c), None, C.byref(h)) == -1
    assert b"FBAQ4" in emu_lib.asarf_last_error()
    c, keep = sc.to_c()
    c.fbaq_q_lut = None
    assert emu_lib.asarf_plan_create(C.byref(c), None, C.byref(h)) == -1
    assert b"tables" in emu_lib.asarf_last_error()
    c, keep = sc.to_c()
    c.raw_format = 7
    assert emu_lib.asarf_plan_create(C.byref(c), None, C.byref(h)) == -1


@pytest.mark.gpu
def test_gpu_statistics_reproducible_and_larger_scene(gpu_lib):
    import torch
    sc, raw, _ = scene_and_raw(gpu_lib, S.ers_small, raw_format="fbaq4", seed=1006)
    plan = asarf.FocusPlan(sc, lib=gpu_lib)
    d_raw = torch.from_numpy(raw).cuda()
    outs, results = [], []
    for _ in range(3):
        o = torch.zeros(plan.out_shape, dtype=torch.float32, device="cuda")
        plan.focus(d_raw, o, stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        outs.append(o.cpu().numpy())
        results.append(plan.results())
    assert all(np.array_equal(outs[0], o) for o in outs[1:])
    assert all(results[0] == r for r in results[1:])
    ref = oracle_focus(sc, raw)
    r = results[0]
    assert r["errors"] == 0
    assert abs(r["iq_gain"] - ref.iq.iq_gain) <= 1e-6
    assert np.allclose(r["doppler_centroid_poly"], ref.dc_poly, rtol=1e-6, atol=1e-6)
    det = outs[0][: r["out_rows"], : r["out_cols"]]
    assert rel_rmse(det, ref.detected) < TOL_DETECTED


@pytest.mark.gpu
def test_reference_decode_pins_oracle(gpu_lib):
    from oracle import ref_lib
    if not ref_lib.available():
        pytest.fail("reference build oracle/_ref/libasar_ref.so missing")
    sc, raw = _fbaq_scene(gpu_lib)
    ti, tq = sc.fbaq_tables
    swst = np.asarray(sc.swst_codes, dtype=np.uint16)
    got = ref_lib.ref_convert_asar(raw, swst, ti, tq, sc.range_size)
    ref = rda.decode_asar_fbaq(raw, swst, sc.range_size, ti, tq)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
def test_fbaq_matches_reference_build(gpu_lib):
    from oracle import ref_lib
    if not ref_lib.available():
        pytest.fail("reference build oracle/_ref/libasar_ref.so missing")
    sc, raw = _fbaq_scene(gpu_lib)
    swst = np.asarray(sc.swst_codes, dtype=np.uint16)
    plan = asarf.FocusPlan(sc, lib=gpu_lib)
    out = plan.focus_host(raw, swst)
    res = plan.results()
    c, keep = sc.to_c()
    det, r, _ = ref_lib.ref_focus(c, sc.vr_poly, raw, swst=swst)
    assert (r["first_line"], r["n_lines"]) == (res["first_line"], res["n_lines"])
    assert abs(r["iq_gain"] - res["iq_gain"]) < 1e-6
    assert np.allclose(r["dc_poly"], res["doppler_centroid_poly"], rtol=1e-5, atol=1e-6)
    assert det.shape == out.shape
    assert rel_rmse(out, det) < TOL_DETECTED
