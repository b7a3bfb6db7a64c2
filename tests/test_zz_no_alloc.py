"""The allocation-free statistics entry point (asarf_raw_statistics_noalloc) against the
planned path's statistics, on the GPU, through the C ABI.

It serves callers that cannot allocate device memory (graph capture in progress, a host
application owning the device memory, real-time ingest); it uses one fixed static scratch
array per device, so two consecutive calls on different scenes also check that the
second call does not see the first call's sums.  This file is collected last so that a
failure here leaves every other test already run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import asarf
from asarf import _lib
from asarf import scene as S
from asarf import sim

pytestmark = pytest.mark.gpu


def _planned_stats(lib, sc, raw_d, out_shape_stream):
    import torch
    plan = asarf.FocusPlan(sc, lib=lib)
    out = torch.empty(plan.out_shape, dtype=torch.float32, device="cuda")
    plan.focus(raw_d, out, stream=out_shape_stream)
    torch.cuda.synchronize()
    return plan, plan.results()


def _noalloc(lib, sc, raw_d, stride, stream):
    import torch
    buf = torch.zeros(C.sizeof(_lib.RawStats), dtype=torch.uint8, device="cuda")
    rc = lib.asarf_raw_statistics_noalloc(raw_d.data_ptr(), sc.raw_line_bytes, sc.samples_per_line, sc.range_size,
                                          sc.azimuth_size, None, 0, sc.samples_per_line * sc.azimuth_size, stride,
                                          sc.prf, buf.data_ptr(), C.c_void_p(stream))
    _lib.check(lib, rc, "raw_statistics_noalloc")
    torch.cuda.synchronize()
    host = buf.cpu().numpy().tobytes()
    return _lib.RawStats.from_buffer_copy(host)


def test_noalloc_statistics_match_planned_path_on_consecutive_calls():
    import torch
    lib = asarf.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    scenes = [S.tiny(), S.tiny(dc_coeffs=(-250.0,), seed=33, range_size=1032)]
    for sc in scenes:  # two calls in a row, different scenes, same static scratch
        sc.prepare(lib)
        raw, _ = sim.simulate(sc, device="cpu")
        raw_d = torch.from_numpy(raw).cuda()
        plan, res = _planned_stats(lib, sc, raw_d, stream)
        got = _noalloc(lib, sc, raw_d, plan.dims["rg_pad_ref"], stream)
        assert got.errors == 0
        for f in ("dc_i", "dc_q", "stddev_i", "stddev_q"):
            assert getattr(got, f) == res[f], f
        assert abs(got.iq_gain / res["iq_gain"] - 1) < 1e-12
        assert abs(got.phase_error - res["phase_error"]) < 1e-9
        assert got.n_dc_blocks == res["n_dc_blocks"]
        assert np.allclose(got.doppler_centroid_poly[:], res["doppler_centroid_estimate"], rtol=1e-12, atol=1e-12)
        assert np.allclose(got.dc_block_hz[: got.n_dc_blocks], res["dc_block_hz"], rtol=1e-12, atol=1e-9)


def test_noalloc_rejects_sizes_outside_its_limits():
    import torch
    lib = asarf.load_library()
    raw_d = torch.zeros(64 * 64, dtype=torch.uint8, device="cuda")
    out = torch.zeros(C.sizeof(_lib.RawStats), dtype=torch.uint8, device="cuda")
    rc = lib.asarf_raw_statistics_noalloc(raw_d.data_ptr(), 32, 16, 16, 64, None, 0, 0, 0, 1680.0, out.data_ptr(),
                                          None)
    assert rc == -1
    assert b"sizes out of range" in lib.asarf_last_error()
