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
