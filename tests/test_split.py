"""Split-precision form of the range-Doppler block (asarf_options.precision = SPLIT) on a B200.

The forward contiguous azimuth transform of length n2 = R * m runs as m-point DFT tiles on
the tensor cores (tcgen05, bf16 hi + lo operands, three products, FP32 accumulation) and
one FP32 radix-R pass.  Checked against the FP64 oracle at the stated tolerances for the
float output: intensity and SLC relative RMSE below 1e-4, and per point target resolution
within 1 %, PSLR within 0.1 dB, ISLR within 0.2 dB and peak phase within 1 mrad.  The
window, Doppler and IQ decisions are those of the plain form (the transform feeds none of
them), and the error flags stay clear.
"""
from __future__ import annotations

import numpy as np
import pytest

import asarf
from asarf import _lib
from asarf import scene as S
from conftest import oracle_focus, rel_rmse, scene_and_raw

pytestmark = pytest.mark.gpu

TOL_SPLIT = 1e-4  # relative RMSE of intensity and of the complex SLC against the FP64 oracle


def asar_small(**kw):
    """ASAR IM-like parameters on a 4096-line cut (azimuth FFT 4116 = 84 x 49)."""
    base = dict(azimuth_size=4096, grid=(4, 4))
    base.update(kw)
    return S.asar_im(**base)


def _slc(plan, res):
    import torch
    d = torch.empty((res["n_lines"], plan.dims["slc_cols"]), dtype=torch.complex64, device="cuda")
    plan.slc_into(d, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return d.cpu().numpy()


def _run(lib, sc, raw, precision, **kw):
    plan = asarf.FocusPlan(sc, lib=lib, precision=precision, **kw)
    out = plan.focus_host(raw)
    res = plan.results()
    return plan, out, res


@pytest.mark.parametrize("factory", [S.tiny, S.ers_small, asar_small])
def test_split_matches_oracle(gpu_lib, factory):
    sc, raw, _ = scene_and_raw(gpu_lib, factory)
    plan, out, res = _run(gpu_lib, sc, raw, _lib.PRECISION_SPLIT)
    assert plan.dims["precision"] == _lib.PRECISION_SPLIT, plan.dims
    assert plan.dims["split_radix"] * plan.dims["split_m"] == plan.dims["n2"]
    ref = oracle_focus(sc, raw)
    assert res["errors"] == 0
    assert res["first_line"] == ref.window["first_line"]
    assert out.shape == ref.detected.shape
    assert rel_rmse(out, ref.detected) < TOL_SPLIT
    assert rel_rmse(_slc(plan, res), ref.slc) < TOL_SPLIT


def test_split_and_plain_forms_agree(gpu_lib):
    sc, raw, _ = scene_and_raw(gpu_lib, S.ers_small)
    p32, o32, r32 = _run(gpu_lib, sc, raw, _lib.PRECISION_FP32)
    psp, osp, rsp = _run(gpu_lib, sc, raw, _lib.PRECISION_SPLIT)
    assert p32.dims["precision"] == _lib.PRECISION_FP32
    for k in ("first_line", "n_lines", "variant", "out_rows", "out_cols"):
        assert r32[k] == rsp[k], k
    assert rel_rmse(osp, o32) < TOL_SPLIT


def test_split_point_target_quality_matches_oracle(gpu_lib):
    from oracle import irf
    sc, raw, truth = scene_and_raw(gpu_lib, S.ers_small)
    plan, out, res = _run(gpu_lib, sc, raw, _lib.PRECISION_SPLIT, ref_compat_stats=False)
    ref = oracle_focus(sc, raw, ref_compat=False)
    slc = _slc(plan, res)
    first = res["first_line"]
    n = 0
    for (xt, yt) in truth["targets"]:
        y, x = yt - first, xt - 8
        if not (40 <= y < slc.shape[0] - 40 and 40 <= x < slc.shape[1] - 40):
            continue
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
