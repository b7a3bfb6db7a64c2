"""Host FP64 geometry of the library (C++) against the oracle's restatement (numpy)."""
from __future__ import annotations

import ctypes as C

import numpy as np

import asarf
from asarf import scene as S
from oracle import geometry as geo
from oracle import rda


def _scene(lib, factory=S.ers_full, **kw):
    sc = factory(**kw)
    sc.prepare(lib)
    return sc


def test_interpolate_and_geolocate():
    lib = asarf.load_library()
    sc = _scene(lib)
    osv = [geo.Osv(*o) for o in sc.osv]
    t = sc.first_line_time_us + 7_654_321
    o_ref = geo.interpolate_orbit(osv, t)
    arr = (asarf._lib.Osv * len(sc.osv))(*[asarf._lib.Osv(a, (C.c_double * 3)(*p), (C.c_double * 3)(*v))
                                           for a, p, v in sc.osv])
    o = asarf._lib.Osv()
    assert lib.asarf_interpolate_orbit(arr, len(sc.osv), t, C.byref(o)) == 0
    assert np.allclose(o.pos[:], o_ref.pos, rtol=0, atol=1e-6)
    assert np.allclose(o.vel[:], o_ref.vel, rtol=0, atol=1e-9)
    out = (C.c_double * 3)()
    r = 850000.0
    assert lib.asarf_geolocate((C.c_double * 3)(*o.vel), (C.c_double * 3)(*o.pos),
                               (C.c_double * 3)(*sc.center_point), r, out) == 0
    g = geo.geolocate(o_ref.vel, o_ref.pos, sc.center_point, r)
    assert np.allclose(out[:], g, atol=1e-5)
    # zero Doppler, requested slant range, on the ellipsoid
    d = np.array(out[:]) - np.array(o.pos[:])
    assert abs(np.dot(d, o.vel[:])) / np.linalg.norm(d) / np.linalg.norm(o.vel[:]) < 1e-9
    assert abs(np.linalg.norm(d) - r) < 1e-4


def test_processing_velocity_estimate():
    lib = asarf.load_library()
    sc = _scene(lib)
    d = sc.to_dict()
    ref = geo.estimate_processing_velocity([geo.Osv(*o) for o in sc.osv], d["first_line_time_us"],
                                           d["line_time_interval"], d["center_point"], d["slant_range_first"],
                                           d["range_spacing"], d["carrier_frequency"], d["vr_poly_init"], d["prf"],
                                           d["az_bw_frac"], d["range_size"], d["chirp_samples"], d["azimuth_size"])
    x = np.arange(0, sc.range_size, 97)
    assert np.allclose(np.polyval(sc.vr_poly, x), np.polyval(ref, x), rtol=1e-9)
    assert 6900 < sc.vr_poly[2] < 7200


def test_srgr_polynomial_and_index_map():
    lib = asarf.load_library()
    sc = _scene(lib, S.ers_small)
    c, keep = sc.to_c()
    poly = (C.c_double * 5)()
    ng = C.c_int32()
    nx = sc.range_size - sc.chirp_samples - 16
    first = sc.slant_range_first + 8 * sc.range_spacing
    lti = (1.0 / sc.prf) * 5.0
    assert lib.asarf_srgr_polynomial(C.byref(c), first, nx, 700, lti, poly, C.byref(ng)) == 0
    ref, ng_ref = geo.srgr_polynomial([geo.Osv(*o) for o in sc.osv], sc.first_line_time_us, lti, 700,
                                      sc.center_point, first, sc.range_spacing, nx)
    assert ng.value == ng_ref
    gd = np.linspace(0, ng_ref * 12.5, 50)
    assert np.allclose(np.polyval(poly[:], gd), np.polyval(ref, gd), atol=1e-6)
    # the two FP64 fits differ only in rounding noise (the constant term is ~5e-5 m); the
    # float32 index maps they produce select the same slant samples
    start, frac = geo.srgr_index_map(ref, sc.range_spacing, ng_ref)
    start2, frac2 = geo.srgr_index_map(poly[:], sc.range_spacing, ng_ref)
    assert np.array_equal(start, start2)
    assert np.max(np.abs(frac - frac2)) < 1e-5
    assert start[0] == 0 and np.all(np.diff(start) >= 0) and start[-1] + 1 < nx


def test_chirp_replica_matches_oracle():
    lib = asarf.load_library()
    for window in (True, False):
        sc = S.ers_small(apply_window=window)
        out = np.empty(2 * 2800, dtype=np.float32)
        assert lib.asarf_generate_chirp(sc.chirp_kr, sc.range_sampling_rate, sc.chirp_samples, int(window), 2800,
                                        out.ctypes.data_as(C.POINTER(C.c_float))) == 0
        c = out[0::2] + 1j * out[1::2]
        ref = rda.generate_chirp(sc.chirp_kr, sc.range_sampling_rate, sc.chirp_samples, window, 2800)
        assert np.array_equal(c.astype(np.complex64), ref)


def test_float32_fma_emulation_is_exact():
    from fractions import Fraction
    rng = np.random.default_rng(5)
    a = rng.normal(0, 100, 2000).astype(np.float32)
    b = rng.normal(0, 1e-3, 2000).astype(np.float32)
    c = rng.normal(0, 1, 2000).astype(np.float32)
    v = rda.fmaf(a, b, c)
    for i in range(0, 2000, 37):
        assert v[i] == geo.fmaf(a[i], b[i], c[i])
    # a halfway case where binary64 rounding then binary32 rounding would differ
    x = np.float32(1.0 + 2 ** -23)
    y = np.float32(1.0 + 2 ** -23)
    z = np.float32(-1.0)
    exact = Fraction(float(x)) * Fraction(float(y)) + Fraction(float(z))
    assert geo.fmaf(x, y, z) == np.float32(float(exact))


def test_blackman_window_is_numpy_blackman16():
    assert np.array_equal(rda.blackman16(), np.blackman(16).astype(np.float32))
