"""Absolute-phase mode (asarf_options.absolute_phase): the azimuth matched filter also carries
exp(j 4 pi R0 / lambda) per range column (R0 the column's slant range, FP64, reduced modulo
2 pi before the cast) and exp(j pi dc_off^2 / Ka), so a focused point target keeps its own
phase instead of -4 pi R0 / lambda.  The reference has no such term; its convention stays the
default.

* CPU (host emulation of the kernel bodies) and GPU: SLC against the oracle in the same mode
  (relative RMSE, and the phase at every point target within 1 mrad).
* Physics: the simulated targets all have the same reflectivity phase, so in this mode their
  focused phases agree across range (spread well under a radian), while in the reference
  convention they are spread over the circle by 4 pi R0 / lambda.
"""
from __future__ import annotations

import numpy as np
import pytest

import asarf
from asarf import scene as S
from conftest import rel_rmse, scene_and_raw


def _oracle(sc, raw, absolute):
    from oracle import rda
    return rda.focus(raw, sc.to_dict(), ref_compat=False, absolute_phase=absolute)


def _target_phases(slc, ref_slc, truth, first):
    from oracle import irf
    got, want = [], []
    for (xt, yt) in truth["targets"]:
        y, x = yt - first, xt - 8
        if not (40 <= y < slc.shape[0] - 40 and 40 <= x < slc.shape[1] - 40):
            continue
        lo, hi = int(max(0, y - 400)), int(min(slc.shape[0], y + 400))
        blk = np.abs(ref_slc[lo:hi, int(x) - 6:int(x) + 7])
        py, px = np.unravel_index(np.argmax(blk), blk.shape)
        a = irf.analyse(slc, lo + py, int(x) - 6 + px)
        b = irf.analyse(ref_slc, lo + py, int(x) - 6 + px)
        if a and b:
            got.append(a["phase"])
            want.append(b["phase"])
    return np.array(got), np.array(want)


def _circular_spread(ph):
    return float(np.abs(np.angle(np.exp(1j * (ph - np.angle(np.mean(np.exp(1j * ph))))))).max())


def _slc(plan, res, on_gpu: bool):
    shape = (res["n_lines"], plan.dims["slc_cols"])
    if on_gpu:
        import torch
        d = torch.empty(shape, dtype=torch.complex64, device="cuda")
        plan.slc_into(d, stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        return d.cpu().numpy()
    out = np.empty(shape, dtype=np.complex64)  # the host emulation's "device" memory is host memory
    plan.slc_into(out)
    return out


def _check(lib, factory, tol, on_gpu):
    sc, raw, truth = scene_and_raw(lib, factory)
    plan = asarf.FocusPlan(sc, lib=lib, ref_compat_stats=False, absolute_phase=True)
    plan.focus_host(raw)
    res = plan.results()
    assert res["errors"] == 0
    slc = _slc(plan, res, on_gpu)
    ref = _oracle(sc, raw, True)
    assert rel_rmse(slc, ref.slc) < tol
    got, want = _target_phases(slc, ref.slc, truth, res["first_line"])
    assert got.size >= 4
    assert np.abs(np.angle(np.exp(1j * (got - want)))).max() < 1e-3
    return got, sc, raw, truth


def test_absolute_phase_emulated_kernels_match_oracle(emu_lib):
    _check(emu_lib, S.tiny, 1e-5, on_gpu=False)


@pytest.mark.gpu
def test_absolute_phase_matches_oracle_and_flattens_target_phase(gpu_lib):
    got, sc, raw, truth = _check(gpu_lib, S.ers_small, 1e-5, on_gpu=True)
    assert _circular_spread(got) < 0.5
    conv = _oracle(sc, raw, False)
    ph, _ = _target_phases(conv.slc, conv.slc, truth, conv.window["first_line"])
    assert _circular_spread(ph) > 1.0
