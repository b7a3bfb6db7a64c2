"""The header-compatible drop-in (asar-focus_b200/dropin/sar_dropin.cu): the reference's
sar/ functions with their own C++ signatures over DevicePaddedImage / CudaWorkspace /
SARMetadata, implemented on libasarf.

The harness that replays main.cc's flow is compiled once against the reference's own sar/
GPU stages (oracle/_ref/libasar_ref.so) and once against the drop-in
(oracle/_ref/libasar_dropin.so); the two builds differ only in which implementation of
those functions they link.  The drop-in run must give the reference run's image and the
planned path's image.
"""
from __future__ import annotations

import numpy as np
import pytest

import asarf
from asarf import scene as S
from conftest import rel_rmse, scene_and_raw

pytestmark = pytest.mark.gpu


def test_dropin_library_exports_the_reference_signatures():
    from oracle import ref_lib
    assert ref_lib.available(ref_lib.DROPIN_LIB), "drop-in build missing (make -C oracle/ref_build)"


@pytest.mark.parametrize("factory", [S.tiny, S.ers_small])
def test_main_flow_on_dropin_matches_reference_and_planned_path(gpu_lib, factory):
    from oracle import ref_lib
    sc, raw, _ = scene_and_raw(gpu_lib, factory)
    scc, keep = sc.to_c()
    det_ref, r_ref, _ = ref_lib.ref_focus(scc, sc.vr_poly, raw)
    det_new, r_new, d_new = ref_lib.ref_focus(scc, sc.vr_poly, raw, dumps=True, lib_path=ref_lib.DROPIN_LIB)
    assert (r_new["first_line"], r_new["n_lines"], r_new["out_rows"], r_new["out_cols"]) == \
        (r_ref["first_line"], r_ref["n_lines"], r_ref["out_rows"], r_ref["out_cols"])
    assert abs(r_new["iq_gain"] - r_ref["iq_gain"]) < 1e-6
    assert np.allclose(r_new["dc_poly"], r_ref["dc_poly"], rtol=1e-5, atol=1e-6)
    assert np.allclose(r_new["grsr_poly"], r_ref["grsr_poly"], rtol=1e-9, atol=1e-9)  # FP64 fits, metres
    assert rel_rmse(det_new, det_ref) < 1e-5
    plan = asarf.FocusPlan(sc, lib=gpu_lib)
    out = plan.focus_host(raw)
    assert out.shape == det_new.shape
    assert rel_rmse(det_new, out) < 1e-5
