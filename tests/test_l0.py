"""ERS IM level-0 packets: the host forecast (record-number gaps filled from the previous
packet, sensing-time window) against the oracle's restatement of FetchErsL0ImForecastMeta,
the unpack kernel (measurement bytes, SWST / PRI codes, header checks) against the
oracle's ParseErsLevel0ImPackets, and packets -> unpack -> focus against focusing the raw
lines directly.
"""
from __future__ import annotations

import numpy as np
import pytest

from asarf import _lib, l0
from oracle import l0 as ol0

T0_US = 8_765 * 86_400_000_000 + 40_000 * 1_000_000   # some day in 2024, 11:06:40
PRI_US = 595


def _packets(n=40, gaps=((10, 3), (25, 1)), seed=3, **kw):
    """n packets with record-number jumps: at packet i the number skips by k (k packets missing)."""
    rng = np.random.default_rng(seed)
    raw = rng.integers(0, 32, size=(n, l0.MEASUREMENT_BYTES), dtype=np.uint8)
    rec = np.arange(n, dtype=np.int64) + 1000
    for i, k in gaps:
        rec[i:] += k
    times = T0_US + rec * PRI_US
    swst = (rng.integers(0, 3, size=n) + 600).astype(np.uint16)
    pri = np.full(n, 2820, dtype=np.uint16)
    return l0.write_packets(raw, swst, pri, rec, times, **kw), raw, swst, times


@pytest.mark.parametrize("window", [(0, 10**9, 0, 0), (5, 30, 0, 0), (5, 30, 2, 3), (0, 15, 100, 100)])
def test_forecast_matches_oracle(emu_lib, window):
    blob, _, _, times = _packets()
    lo, hi, before, after = window
    start = l0.mjd(T0_US + (1000 + lo) * PRI_US)
    stop = l0.mjd(T0_US + (1000 + hi) * PRI_US)
    offs, ts, b, a = l0.forecast(blob, start, stop, before, after, lib=emu_lib)
    fc, rb, ra = ol0.forecast(blob, start, stop, before, after)
    assert list(offs) == [o for o, _ in fc]
    assert ts == [t for _, t in fc]
    assert (b, a) == (rb, ra)


def test_forecast_fills_missing_packets_with_the_previous_one(emu_lib):
    blob, _, _, _ = _packets(n=20, gaps=((7, 4),))
    offs, _, _, _ = l0.forecast(blob, (0, 0, 0), (10**6, 0, 0), 0, 0, lib=emu_lib)
    assert len(offs) == 24
    assert list(offs[6:11]) == [6 * l0.MDSR_BYTES] * 5  # packet 6 stands in for the 4 missing ones
    assert offs[11] == 7 * l0.MDSR_BYTES


def test_forecast_rejects_the_reference_error_cases(emu_lib):
    blob, _, _, _ = _packets(n=10, gaps=((5, 901),))
    with pytest.raises(_lib.AsarfError):
        l0.forecast(blob, (0, 0, 0), (10**6, 0, 0), 0, 0, lib=emu_lib)
    assert b"more than threshold 900" in emu_lib.asarf_last_error()
    bad, _, _, _ = _packets(n=4, gaps=(), isp_length=11464)
    with pytest.raises(_lib.AsarfError):
        l0.forecast(bad, (0, 0, 0), (10**6, 0, 0), 0, 0, lib=emu_lib)
    assert b"ISP length shall be 11465" in emu_lib.asarf_last_error()


def test_unpack_emulated_matches_oracle(emu_lib):
    blob, _, _, _ = _packets()
    offs, _, _, _ = l0.forecast(blob, (0, 0, 0), (10**6, 0, 0), 0, 0, lib=emu_lib)
    n = len(offs)
    raw = np.zeros((n, l0.MEASUREMENT_BYTES), dtype=np.uint8)
    swst = np.zeros(n, dtype=np.uint16)
    pri = np.zeros(n, dtype=np.uint16)
    err = np.zeros(1, dtype=np.uint32)
    l0.unpack(blob, offs, n, raw, swst, pri, err, lib=emu_lib)
    ref = ol0.parse(blob, offs)
    assert np.array_equal(raw, ref["raw"]) and np.array_equal(swst, ref["swst"]) and np.array_equal(pri, ref["pri"])
    assert int(err[0]) == ref["errors"] == 0
    marked = l0.write_packets(raw[:3], swst[:3], pri[:3], np.arange(3), np.arange(3), aux_marker=0x55)
    l0.unpack(marked, np.arange(3, dtype=np.int64) * l0.MDSR_BYTES, 3, raw[:3], None, None, err, lib=emu_lib)
    assert int(err[0]) == l0.ERR_AUX_MARKER


@pytest.mark.gpu
def test_unpack_on_gpu_feeds_the_focus(gpu_lib):
    """Packets of the ERS 5616-sample lines (one 3-packet gap) -> GPU unpack -> focus, against
    the oracle's parse and against focusing the parsed raw lines."""
    import torch
    import asarf
    from asarf import scene as S
    from asarf import sim
    from conftest import scene_and_raw
    sc, raw_lines, _ = scene_and_raw(gpu_lib, S.ers_full, azimuth_size=2048, grid=(4, 2), device="cuda")
    n = raw_lines.shape[0]
    rec = np.arange(n, dtype=np.int64) + 1
    rec[1000:] += 3
    swst = np.full(n, 600, dtype=np.uint16)
    blob = l0.write_packets(raw_lines, swst, np.full(n, 2820, np.uint16), rec, T0_US + rec * PRI_US)
    offs, _, _, _ = l0.forecast(blob, (0, 0, 0), (10**6, 0, 0), 0, 0, lib=gpu_lib)
    lines = len(offs)
    assert lines == n + 3
    d_blob = torch.from_numpy(blob).cuda()
    d_offs = torch.from_numpy(offs).cuda()
    d_raw = torch.zeros((lines, l0.MEASUREMENT_BYTES), dtype=torch.uint8, device="cuda")
    d_swst = torch.zeros(lines, dtype=torch.int16, device="cuda")
    d_pri = torch.zeros(lines, dtype=torch.int16, device="cuda")
    d_err = torch.zeros(1, dtype=torch.int32, device="cuda")
    l0.unpack(d_blob, d_offs, lines, d_raw, d_swst, d_pri, d_err, lib=gpu_lib,
              stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ref = ol0.parse(blob, offs)
    assert int(d_err.item()) == 0
    assert np.array_equal(d_raw.cpu().numpy(), ref["raw"])
    assert np.array_equal(d_swst.cpu().numpy().view(np.uint16), ref["swst"])
    assert np.array_equal(d_pri.cpu().numpy().view(np.uint16), ref["pri"])
    # the unpacked lines focus exactly as the parsed host lines do
    from dataclasses import replace
    sc2 = replace(sc, azimuth_size=lines)
    sc2.prepare(gpu_lib)
    plan = asarf.FocusPlan(sc2, lib=gpu_lib)
    out_d = torch.zeros(plan.out_shape, dtype=torch.float32, device="cuda")
    plan.focus(d_raw, out_d, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    host = plan.focus_host(ref["raw"])
    r = plan.results()
    assert r["errors"] == 0
    assert np.array_equal(out_d.cpu().numpy()[: host.shape[0], : host.shape[1]], host)


# ---------------------------------------------------------------- ENVISAT ASAR IM
RSR = 19.207680e6       # ASAR IM range sampling rate (instrument file)
ASAR_PRI = 11628        # PRI code (PRF = RSR / code = 1652 Hz)


def _asar_packets(n=60, seed=5, noise=(0, 1, 30), cal=(20, 21, 45), short=(33,)):
    """n packets of FBAQ4 records: noise packets at the given indices (and first, before any
    echo), calibration packets elsewhere, some records shorter than the rest."""
    rng = np.random.default_rng(seed)
    nbytes = 2 + 64 * 10 + 20
    rec = np.zeros((n, nbytes), dtype=np.uint8)
    for i in range(n):
        ln = nbytes - 2 - (130 if i in short else 0)
        rec[i, 0], rec[i, 1] = ln & 0xFF, ln >> 8
        rec[i, 2:2 + ln] = rng.integers(0, 256, size=ln, dtype=np.uint8)
    flags = np.full(n, l0.FLAG_ECHO, dtype=np.uint8)
    flags[list(noise)] = l0.FLAG_NOISE
    flags[list(cal)] = l0.FLAG_CAL
    times = T0_US + np.arange(n, dtype=np.int64) * 605
    swst = (rng.integers(0, 4, size=n) + 900).astype(np.uint16)
    pri = np.full(n, ASAR_PRI, dtype=np.uint16)
    blob, num = l0.write_asar_packets(rec, swst, pri, times, flags)
    return blob, num, rec, flags, times


@pytest.mark.parametrize("window", [(0, 10**9, 0, 0), (5, 40, 0, 0), (5, 40, 2, 3), (23, 50, 1, 100)])
def test_asar_forecast_matches_oracle(emu_lib, window):
    blob, num, _, _, _ = _asar_packets()
    lo, hi, before, after = window
    start = l0.mjd(T0_US + lo * 605)
    stop = l0.mjd(T0_US + hi * 605)
    offs, ts, b, a = l0.asar_forecast(blob, num, start, stop, before, after, lib=emu_lib)
    fc, rb, ra = ol0.asar_forecast(blob, num, start, stop, before, after)
    assert list(offs) == [o for o, _ in fc]
    assert ts == [t for _, t in fc]
    assert (b, a) == (rb, ra)


def test_asar_forecast_skips_noise_and_leading_packets(emu_lib):
    blob, num, _, flags, _ = _asar_packets()
    offs, _, _, _ = l0.asar_forecast(blob, num, (0, 0, 0), (10**6, 0, 0), 0, 0, lib=emu_lib)
    # packets 0, 1 (noise, before the first echo) and 30 (noise) are not lines
    assert len(offs) == num - 3


def test_asar_lines_and_unpack_match_oracle(emu_lib):
    blob, num, rec, flags, _ = _asar_packets()
    offs, _, _, _ = l0.asar_forecast(blob, num, (0, 0, 0), (10**6, 0, 0), 0, 0, lib=emu_lib)
    src, times, record_bytes, most = l0.asar_lines(blob, offs, RSR, lib=emu_lib)
    ref = ol0.asar_parse(blob, offs, RSR)
    assert record_bytes == ref["record_bytes"] == rec.shape[1]
    assert most == ref["max_samples"]
    assert times == ref["times"]
    lines = len(offs)
    out = np.full((lines, record_bytes), 0xEE, dtype=np.uint8)
    swst = np.zeros(lines, dtype=np.uint16)
    pri = np.zeros(lines, dtype=np.uint16)
    err = np.zeros(1, dtype=np.uint32)
    l0.asar_unpack(blob, src, lines, record_bytes, out, swst, pri, err, lib=emu_lib)
    assert int(err[0]) == 0
    assert np.array_equal(out, ref["records"]) and np.array_equal(swst, ref["swst"])
    assert np.array_equal(pri, ref["pri"])
    # a calibration line repeats the previous line, one PRI later
    k = int(np.flatnonzero(offs == _offset_of(blob, num, 20))[0])
    assert np.array_equal(out[k], out[k - 1])
    us = int(np.float64(np.float32(1.0) / (np.float32(RSR) / np.float32(ASAR_PRI))) * 1e6)
    assert times[k] == ol0._add_micros(times[k - 1], us)


def _offset_of(blob, num, i):
    o = 0
    for _ in range(i):
        o += 39 + ((int(blob[o + 24]) << 8) | int(blob[o + 25]))
    return o


def test_asar_rejects_the_reference_error_cases(emu_lib):
    blob, num, rec, flags, times = _asar_packets()
    bad, n2 = l0.write_asar_packets(rec, np.zeros(num, np.uint16), np.full(num, ASAR_PRI, np.uint16), times, flags,
                                    datafield_length=30)
    with pytest.raises(_lib.AsarfError):
        l0.asar_forecast(bad, n2, (0, 0, 0), (10**6, 0, 0), 0, 0, lib=emu_lib)
    assert b"Date Field Header Length should be 29" in emu_lib.asarf_last_error()
    wm, n3 = l0.write_asar_packets(rec, np.zeros(num, np.uint16), np.full(num, ASAR_PRI, np.uint16), times, flags,
                                   mode_id=0x55)
    offs, _, _, _ = l0.asar_forecast(wm, n3, (0, 0, 0), (10**6, 0, 0), 0, 0, lib=emu_lib)
    with pytest.raises(_lib.AsarfError):
        l0.asar_lines(wm, offs, RSR, lib=emu_lib)
    assert b"Expected only IM mode packets" in emu_lib.asarf_last_error()
    # a window whose first line after trimming is a calibration packet, with the walk ending on
    # an echo packet: the reference's consistency check throws
    with pytest.raises(_lib.AsarfError):
        l0.asar_forecast(blob, num, l0.mjd(T0_US + 20 * 605), (10**6, 0, 0), 0, 0, lib=emu_lib)
    assert b"Programming error detected" in emu_lib.asarf_last_error()
    with pytest.raises(ValueError):
        ol0.asar_forecast(blob, num, l0.mjd(T0_US + 20 * 605), (10**6, 0, 0), 0, 0)
    # a data set cut inside the last echo packet's sample blocks
    offs, _, _, _ = l0.asar_forecast(blob, num, (0, 0, 0), (10**6, 0, 0), 0, 0, lib=emu_lib)
    with pytest.raises(_lib.AsarfError):
        l0.asar_lines(blob[:-10], offs, RSR, lib=emu_lib)
    assert b"end past the data set" in emu_lib.asarf_last_error()
    # the unpack kernel flags a block length beyond the record
    offs, _, _, _ = l0.asar_forecast(blob, num, (0, 0, 0), (10**6, 0, 0), 0, 0, lib=emu_lib)
    src, _, record_bytes, _ = l0.asar_lines(blob, offs, RSR, lib=emu_lib)
    err = np.zeros(1, dtype=np.uint32)
    out = np.zeros((len(offs), record_bytes - 8), dtype=np.uint8)
    l0.asar_unpack(blob, src, len(offs), record_bytes - 8, out, None, None, err, lib=emu_lib)
    assert int(err[0]) == l0.ERR_LENGTH


@pytest.mark.gpu
def test_asar_unpack_on_gpu_feeds_the_focus(gpu_lib):
    """ASAR IM FBAQ4 packets (noise and calibration packets interleaved) -> forecast -> GPU
    unpack -> focus, against the oracle's parse and against focusing the host records."""
    import torch
    import asarf
    from asarf import scene as S
    from conftest import scene_and_raw
    from dataclasses import replace
    sc, recs, _ = scene_and_raw(gpu_lib, S.asar_fbaq, azimuth_size=2048, grid=(4, 2))
    n = recs.shape[0]
    # noise packet first, then echoes with two calibration packets and one noise packet inserted
    order = [0] + list(range(n))
    flags = [l0.FLAG_NOISE] + [l0.FLAG_ECHO] * n
    for at, kind in ((700, l0.FLAG_CAL), (701, l0.FLAG_CAL), (1500, l0.FLAG_NOISE)):
        order.insert(at, order[at - 1])
        flags.insert(at, kind)
    order = np.asarray(order)
    swst = np.full(len(order), 900, dtype=np.uint16)
    times = T0_US + np.arange(len(order), dtype=np.int64) * 605
    blob, num = l0.write_asar_packets(recs[order], swst, np.full(len(order), ASAR_PRI, np.uint16), times,
                                      np.asarray(flags, dtype=np.uint8))
    offs, _, _, _ = l0.asar_forecast(blob, num, (0, 0, 0), (10**6, 0, 0), 0, 0, lib=gpu_lib)
    src, _, record_bytes, _ = l0.asar_lines(blob, offs, RSR, lib=gpu_lib)
    lines = len(offs)
    assert lines == n + 2 and record_bytes == sc.raw_line_bytes
    d_blob = torch.from_numpy(blob).cuda()
    d_src = torch.from_numpy(src).cuda()
    d_rec = torch.full((lines, record_bytes), 0xEE, dtype=torch.uint8, device="cuda")
    d_swst = torch.zeros(lines, dtype=torch.int16, device="cuda")
    d_pri = torch.zeros(lines, dtype=torch.int16, device="cuda")
    d_err = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    l0.asar_unpack(d_blob, d_src, lines, record_bytes, d_rec, d_swst, d_pri, d_err, lib=gpu_lib, stream=stream)
    torch.cuda.synchronize()
    ref = ol0.asar_parse(blob, offs, RSR)
    assert int(d_err.item()) == 0
    assert np.array_equal(d_rec.cpu().numpy(), ref["records"])
    assert np.array_equal(d_swst.cpu().numpy().view(np.uint16), ref["swst"])
    assert np.array_equal(d_pri.cpu().numpy().view(np.uint16), ref["pri"])
    sc2 = replace(sc, azimuth_size=lines)
    sc2.prepare(gpu_lib)
    plan = asarf.FocusPlan(sc2, lib=gpu_lib)
    out_d = torch.zeros(plan.out_shape, dtype=torch.float32, device="cuda")
    plan.focus(d_rec, out_d, stream=stream)
    torch.cuda.synchronize()
    host = plan.focus_host(ref["records"])
    assert plan.results()["errors"] == 0
    assert np.array_equal(out_d.cpu().numpy()[: host.shape[0], : host.shape[1]], host)
