"""The CPU oracle against golden outputs of the reference's own focusing code.

The fixtures (tests/golden/ref_*.npz) were produced by tests/golden/make_golden.py: the
reference's sar/ + cuda_util/ sources compiled for sm_100a and run on a B200 over scenes
simulated on the CPU from fixed seeds.  Here the same raw bytes are regenerated (SHA-256
checked) and the oracle must reproduce the reference: IQ statistics and the IQ-corrected
samples bit-for-bit, the range-compressed and detected samples to float32 noise.
"""
from __future__ import annotations

import hashlib
from pathlib import Path

import numpy as np
import pytest

import asarf
from asarf import scene as S
from asarf import sim
from conftest import rel_rmse

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("name,factory", [("tiny", S.tiny), ("ers_small", S.ers_small)])
def test_oracle_reproduces_reference_build(name, factory):
    from oracle import rda
    g = np.load(GOLDEN / f"ref_{name}.npz")
    lib = asarf.load_library()
    sc = factory()
    sc.prepare(lib)
    raw, _ = sim.simulate(sc, device="cpu")
    digest = np.frombuffer(hashlib.sha256(raw.tobytes()).digest(), dtype=np.uint8)
    assert np.array_equal(digest, g["raw_sha256"]), "synthetic raw bytes differ from the fixture's"
    assert np.allclose(sc.vr_poly, g["vr_poly"], rtol=0, atol=0)
    ref = rda.focus(raw, sc.to_dict(), keep_intermediate=True)
    dc_i, dc_q, gain, phase, sd_i, sd_q = g["stats"]
    assert ref.iq.dc_i == dc_i and ref.iq.dc_q == dc_q
    assert ref.iq.stddev_i == sd_i and ref.iq.stddev_q == sd_q
    # the reference reduces the gain / phase sums in float: its reported values carry ~1e-8
    # relative noise; the float constants it applies (and so the corrected samples) agree exactly
    assert abs(ref.iq.iq_gain / gain - 1) < 1e-7 and abs(ref.iq.phase_error - phase) < 1e-4
    x = np.arange(0, sc.range_size, 32)
    assert np.max(np.abs(np.polyval(ref.dc_poly, x) - np.polyval(g["dc_poly"], x))) < 1e-3
    first, n_lines, slc_cols, out_rows, out_cols, max_ap = (int(v) for v in g["window"])
    assert ref.window["first_line"] == first and ref.slc.shape == (n_lines, slc_cols)
    assert ref.detected.shape == (out_rows, out_cols) and max(ref.extra["aperture"]) == max_ap
    rows = g["corrected_head"].shape[0]
    # IQ correction arithmetic: with the reference's own float constants (its gain and
    # quadrature terms come from float-reduced sums; sin = sin(phase), cos = 1 - sin^2)
    # the oracle's correction reproduces the reference's samples bit for bit
    delta = np.sin(np.deg2rad(phase))
    dec = rda.decode_ers(raw[:rows], sc.samples_per_line, None, sc.range_size)
    mine = rda.apply_iq_correction(dec, dc_i, dc_q, np.float32(gain), np.float32(delta), np.float32(1 - delta * delta))
    assert np.array_equal(mine, g["corrected_head"])
    # and the oracle's own constants are within one float32 ulp of the reference's
    assert abs(np.float32(ref.iq.sin_corr) - np.float32(delta)) <= np.spacing(np.float32(delta))
    assert rel_rmse(ref.extra["corrected"][:rows], g["corrected_head"]) < 1e-6
    assert rel_rmse(ref.extra["rc"][:rows], g["rc_head"]) < 2e-6
    assert rel_rmse(ref.detected[:rows], g["detected_head"]) < 1e-5
    s1 = ref.detected.astype(np.float64).sum()
    assert abs(s1 / g["detected_sum"][0] - 1) < 1e-5
