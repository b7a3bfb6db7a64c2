"""Long strips as overlapped azimuth blocks (asarf_strip).

Checked against the oracle's restatement of the same scheme (each block focused as its own
scene, kept lines assembled, one multilook/RSL/SRGR pass), with a Doppler centroid that
drifts along azimuth; and every block's share of the strip SLC is bit-identical to the
same lines focused by that block alone.
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

import asarf
from asarf import scene as S
from conftest import rel_rmse, scene_and_raw
from oracle import rda

BLOCK, OVERLAP = 1024, 320


def _strip_scene(lib):
    return scene_and_raw(lib, S.tiny, azimuth_size=3000, dc_kind="sin", dc_drift=120.0, seed=77, grid=(2, 6))[:2]


def _host(x):
    return x if isinstance(x, np.ndarray) else x.cpu().numpy()


def _run(lib, sc, raw, gpu: bool, block=BLOCK, overlap=OVERLAP):
    strip = asarf.FocusStrip(sc, block_lines=block, overlap=overlap, lib=lib)
    d = strip.dims
    if gpu:
        import torch
        raw_d = torch.from_numpy(raw).cuda()
        out = torch.zeros(strip.out_shape, dtype=torch.float32, device="cuda")
        slc = torch.zeros((d["slc_rows"], d["slc_cols"]), dtype=torch.complex64, device="cuda")
        st = torch.cuda.current_stream().cuda_stream
        strip.focus(raw_d, out, stream=st)
        strip.slc_into(slc, stream=st)
        torch.cuda.synchronize()
    else:
        out = np.zeros(strip.out_shape, dtype=np.float32)
        slc = np.zeros((d["slc_rows"], d["slc_cols"]), dtype=np.complex64)
        strip.focus(raw, out)
        strip.slc_into(slc)
    assert strip.errors() == 0
    return strip, _host(out), _host(slc)


def _check(lib, gpu: bool, sc=None, raw=None, block=BLOCK, overlap=OVERLAP, n_blocks=4):
    if sc is None:
        sc, raw = _strip_scene(lib)
    strip, det, slc = _run(lib, sc, raw, gpu, block, overlap)
    d = strip.dims
    assert d["n_blocks"] == n_blocks
    ap = d["max_aperture"]
    starts, lo, hi, first = rda.strip_layout(sc.azimuth_size, block, overlap, ap)
    assert [b["start"] for b in strip.blocks] == starts
    assert [b["keep_lo"] for b in strip.blocks] == lo and [b["keep_hi"] for b in strip.blocks] == hi
    assert d["first_line"] == first
    # the Doppler estimate follows the azimuth drift from block to block
    dcs = [b["plan"].results()["doppler_centroid_poly"][2] for b in strip.blocks]
    assert max(dcs) - min(dcs) > 50.0
    ref_det, ref_slc = rda.focus_strip(raw, sc.to_dict(), block, overlap)
    assert slc.shape == ref_slc.shape and det.shape == ref_det.shape
    assert rel_rmse(slc, ref_slc) < 1e-5
    assert rel_rmse(det, ref_det) < 1e-5
    # each block's share equals that block focused on its own (its own results window)
    for b in strip.blocks:
        s = b["start"]
        bs = replace(sc, azimuth_size=block, first_line_time_us=sc.first_line_time_us +
                     int(np.floor(s * sc.line_time_interval * 1e6 + 0.5)), lines_before=0, lines_after=0,
                     swst_codes=None)
        plan = asarf.FocusPlan(bs, lib=lib)
        plan.focus_host(np.ascontiguousarray(raw[s:s + block]))
        r = plan.results()
        if gpu:
            import torch
            own = torch.zeros((r["n_lines"], plan.dims["slc_cols"]), dtype=torch.complex64, device="cuda")
            plan.slc_into(own, stream=torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            own = own.cpu().numpy()
        else:
            own = plan.slc_into(np.zeros((r["n_lines"], plan.dims["slc_cols"]), dtype=np.complex64))
        a, z = max(b["keep_lo"], r["first_line"]), min(b["keep_hi"], r["first_line"] + r["n_lines"])
        assert z - a > 100
        mine = slc[s + a - first: s + z - first]
        theirs = own[a - r["first_line"]: z - r["first_line"]]
        assert np.array_equal(mine, theirs)


def test_strip_blocks_emu(emu_lib):
    _check(emu_lib, gpu=False)


@pytest.mark.gpu
def test_strip_blocks_gpu(gpu_lib):
    _check(gpu_lib, gpu=True)


@pytest.mark.gpu
def test_strip_with_the_long_strip_blocking_gpu(gpu_lib):
    """The long-strip workload's own blocking (16384-line blocks overlapping by 1400, ASAR-like
    8-bit, Doppler drifting +-100 Hz) on a 36000-line strip (3 blocks): against the oracle's
    restatement, and every block's share bit-identical to the block focused alone."""
    sc, raw, _ = scene_and_raw(gpu_lib, S.asar_strip, azimuth_size=36000, grid=(8, 12), device="cuda")
    _check(gpu_lib, True, sc, raw, block=16384, overlap=1400, n_blocks=3)
