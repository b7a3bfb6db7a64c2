"""FP64 host-side geometry of the focusing path (oracle restatement).

Each function cites the reference function it restates.  Times are integer
microseconds (the reference uses ``boost::posix_time::ptime`` with microsecond
resolution).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from fractions import Fraction

import numpy as np

SOL = 299792458.0
REFERENCE_RANGE = 800000.0          # envisat_format/include/asar_constants.h:37
GROUND_SPACING = np.float32(12.5)   # sar/srgr.cu:84 (IMP fixed 12.5 m), sar/az_multilook.cu:83
RCMC_WINDOW = 16                    # sar/range_doppler_algorithm.cu:29, focussing_details.h


@dataclass
class Osv:
    time_us: int
    pos: tuple
    vel: tuple


def optimal_fft_sizes(limit: int = 131072) -> list[int]:
    """All 2^a 3^b 5^c 7^d <= limit, sorted (cuda_util/cufft_plan.cc:147-181)."""
    out = set()
    p2 = 1
    while p2 <= limit:
        p3 = p2
        while p3 <= limit:
            p5 = p3
            while p5 <= limit:
                p7 = p5
                while p7 <= limit:
                    out.add(p7)
                    p7 *= 7
                p5 *= 5
            p3 *= 3
        p2 *= 2
    return sorted(out)


_SIZES = optimal_fft_sizes()


def fft_upper_bound(v: int) -> int:
    """std::map::upper_bound: smallest size STRICTLY greater than v (main.cc:217, 223)."""
    for s in _SIZES:
        if s > v:
            return s
    raise ValueError(f"no FFT size above {v}")


def reference_padding(range_size: int, chirp_samples: int, azimuth_size: int) -> tuple[int, int]:
    """(rg_pad, az_pad) as main.cc:215-228 computes them."""
    return fft_upper_bound(range_size + chirp_samples), fft_upper_bound(azimuth_size)


def interpolate_orbit(osv: list[Osv], time_us: int) -> Osv:
    """Lagrange interpolation over all state vectors (sar/orbit_state_vector.cc:23-48)."""
    t0 = osv[0].time_us
    tp = (time_us - t0) * 1e-6
    n = len(osv)
    pos = [0.0, 0.0, 0.0]
    vel = [0.0, 0.0, 0.0]
    for i in range(n):
        mult = 1.0
        xi = (osv[i].time_us - t0) * 1e-6
        for j in range(n):
            if i == j:
                continue
            xj = (osv[j].time_us - t0) * 1e-6
            mult *= (tp - xj) / (xi - xj)
        for k in range(3):
            pos[k] += mult * osv[i].pos[k]
            vel[k] += mult * osv[i].vel[k]
    return Osv(time_us, tuple(pos), tuple(vel))


def azimuth_time_us(first_line_time_us: int, line_time_interval: float, idx: int) -> int:
    """CalcAzimuthTime (sar/sar_metadata.h:90-93): uint32 microseconds, truncated."""
    us = int(line_time_interval * idx * 1e6)
    us &= 0xFFFFFFFF
    return first_line_time_us + us


def geolocate(vel, pos, init_guess, slant_range: float) -> np.ndarray:
    """Zero-Doppler Newton geolocation on the ellipsoid (util/src/geo_tools.cc:27-85)."""
    a = 6378137.0
    b = 6356752.314245
    res = np.array(init_guess, dtype=np.float64)
    v = np.array(vel, dtype=np.float64)
    p = np.array(pos, dtype=np.float64)
    for it in range(1, 102):
        pv = res - p
        A = np.empty((3, 3))
        A[0] = v
        A[1] = 2.0 * pv
        A[2] = [2 * res[0] / (a * a), 2 * res[1] / (a * a), 2 * res[2] / (b * b)]
        B = np.array([v @ pv, pv @ pv - slant_range * slant_range,
                      (res[0] / a) ** 2 + (res[1] / a) ** 2 + (res[2] / b) ** 2 - 1.0])
        dx = np.linalg.solve(A, -B)
        res = res + dx
        if np.linalg.norm(dx) < 1e-6:
            return res
    raise RuntimeError("geolocation did not converge")


def polyfit(x, y, degree: int) -> np.ndarray:
    """Least squares via Householder QR, highest power first (util/src/math_utils.cc:23-44)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    a = np.vander(x, degree + 1, increasing=True)
    q, r = np.linalg.qr(a)
    c = np.linalg.solve(r, q.T @ y)
    return c[::-1].copy()


def polyval(p, x: float) -> float:
    """Horner in FP64 (util/include/math_utils.h:55-63)."""
    v = 0.0
    for e in p:
        v = v * x + e
    return v


def calc_ka(carrier_frequency, vr_poly, slant_first, range_spacing, px: int) -> float:
    """CalcKa (sar/sar_metadata.h:110-115)."""
    vr = polyval(vr_poly, px)
    r0 = slant_first + px * range_spacing
    return (2 * carrier_frequency * vr * vr) / (SOL * r0)


def calc_aperture_pixels_at(carrier_frequency, vr_poly, dc_poly, prf, az_bw_frac, slant_first,
                            range_spacing, px: int) -> int:
    """CalcAperturePixels (sar/sar_metadata.h:117-124); empty dc_poly evaluates to 0."""
    ka = calc_ka(carrier_frequency, vr_poly, slant_first, range_spacing, px)
    fmax = polyval(dc_poly, px) + (prf * az_bw_frac) / 2
    pixels = (fmax / ka) * prf
    return int(_round_half_away(pixels))


def calc_aperture_pixels(carrier_frequency, vr_poly, dc_poly, prf, az_bw_frac, slant_first,
                         range_spacing, range_size, chirp_samples) -> list[int]:
    """CalcAperturePixels over 10 range steps (sar/sar_metadata.h:126-141)."""
    range_end = range_size - chirp_samples
    step = range_end // 10
    out = []
    for px in range(0, range_end, step):
        out.append(calc_aperture_pixels_at(carrier_frequency, vr_poly, dc_poly, prf, az_bw_frac,
                                           slant_first, range_spacing, px))
    return out


def _round_half_away(v: float) -> float:
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)


def estimate_vr_at_range(osv, first_line_time_us, lti, center_point, slant_first, range_spacing,
                         carrier_frequency, vr_poly, dc_poly, prf, az_bw_frac, az_idx, range_idx) -> float:
    """EstimateVrAtRange (sar/processing_velocity_estimation.cc:56-101)."""
    r0 = slant_first + range_idx * range_spacing
    aperture = calc_aperture_pixels_at(carrier_frequency, vr_poly, dc_poly, prf, az_bw_frac,
                                       slant_first, range_spacing, range_idx)
    n = 9
    c_osv = interpolate_orbit(osv, azimuth_time_us(first_line_time_us, lti, az_idx))
    earth = geolocate(c_osv.vel, c_osv.pos, center_point, r0)
    step = int(aperture / (n - 1))
    xs = np.empty(n)
    ys = np.empty(n)
    for i in range(n):
        idx = az_idx + (i - n // 2) * step
        o = interpolate_orbit(osv, azimuth_time_us(first_line_time_us, lti, idx))
        d = np.array(o.pos) - earth
        ys[i] = d @ d - r0 * r0
        xs[i] = (c_osv.time_us - o.time_us) * 1e-6
    a = np.stack([np.ones(n), xs * xs], axis=1)
    sol = np.linalg.lstsq(a, ys, rcond=None)[0]
    return math.sqrt(sol[1])


def estimate_processing_velocity(osv, first_line_time_us, lti, center_point, slant_first, range_spacing,
                                 carrier_frequency, vr_poly_init, prf, az_bw_frac, range_size,
                                 chirp_samples, azimuth_size) -> np.ndarray:
    """EstimateProcessingVelocity (sar/processing_velocity_estimation.cc:105-148).

    The aperture length inside uses the Vr polynomial held in the metadata at call time
    (the initial guess) and an empty Doppler polynomial, as main.cc:251-252 calls it.
    """
    az_idx = azimuth_size // 2
    range_end = range_size - chirp_samples
    step = range_end // 10
    vr, idx = [], []
    for r in range(0, range_end, step):
        vr.append(estimate_vr_at_range(osv, first_line_time_us, lti, center_point, slant_first,
                                       range_spacing, carrier_frequency, vr_poly_init, [], prf,
                                       az_bw_frac, az_idx, r))
        idx.append(r)
    return polyfit(idx, vr, 2)


def results_window(dc_const: float, lines_before: int, lines_after: int, max_aperture: int) -> dict:
    """CalcResultsWindow (main_flow.cc:155-201) for a 16-tap RCMC window."""
    w = dict(near=RCMC_WINDOW // 2, far=RCMC_WINDOW // 2, before_start=lines_before,
             after_start=0, before_stop=0, after_stop=lines_after)
    if dc_const > 0:
        if lines_before < max_aperture:
            w["after_start"] = max_aperture - lines_before
    else:
        if lines_after < max_aperture:
            w["before_stop"] = max_aperture - lines_after
    w["first_line"] = w["before_start"] + w["after_start"]
    w["drop_end"] = w["before_stop"] + w["after_stop"]
    return w


def rsl_table(range_size: int, slant_first: float, range_spacing: float,
              reference_range: float = REFERENCE_RANGE) -> np.ndarray:
    """Range spreading loss column gains (sar/range_spreading_loss.cu:42-52)."""
    i = np.arange(range_size, dtype=np.float64)
    r = slant_first + i * range_spacing
    ratio = reference_range / r
    return (1.0 / np.sqrt(ratio ** 3)).astype(np.float32)


def srgr_polynomial(osv, first_line_time_us, lti, azimuth_size, center_point, slant_first,
                    range_spacing, range_size):
    """Slant->ground mapping fit of SlantRangeToGroundRangeInterpolation (sar/srgr.cu:73-121).

    Returns (grsr_poly float64[5] highest power first, output ground samples Ng).
    """
    n = 100
    t = azimuth_time_us(first_line_time_us, lti, azimuth_size // 2)
    o = interpolate_orbit(osv, t)
    first = geolocate(o.vel, o.pos, center_point, slant_first)
    gd, sr = [], []
    for i in range(n):
        r = slant_first + (i * (range_size // 100)) * range_spacing
        g = geolocate(o.vel, o.pos, center_point, r)
        gd.append(float(np.linalg.norm(g - first)))
        sr.append(r - slant_first)
    ng = int(gd[-1] / float(GROUND_SPACING))
    return polyfit(gd, sr, 4), ng


def _f32(v) -> Fraction:
    return Fraction(float(np.float32(v)))


def _round_f32(q: Fraction) -> np.float32:
    """Correctly round an exact rational to float32 (round to nearest, ties to even)."""
    f = np.float32(float(q))          # float(q) is correctly rounded to binary64
    # binary64 -> binary32 can double-round; fix up by comparing exact neighbours
    lo = np.nextafter(f, np.float32(-np.inf))
    hi = np.nextafter(f, np.float32(np.inf))
    best = f
    best_err = abs(Fraction(float(f)) - q)
    for c in (lo, hi):
        if not np.isfinite(c):
            continue
        e = abs(Fraction(float(c)) - q)
        if e < best_err or (e == best_err and (int(c.view(np.uint32)) & 1) == 0):
            best, best_err = c, e
    return np.float32(best)


def fmaf(a, b, c) -> np.float32:
    """Exact float32 fused multiply-add."""
    return _round_f32(_f32(a) * _f32(b) + _f32(c))


def divf(a, b) -> np.float32:
    return _round_f32(_f32(a) / _f32(b))


def mulf(a, b) -> np.float32:
    return _round_f32(_f32(a) * _f32(b))


def srgr_index_map(grsr_poly, range_spacing: float, ng: int):
    """Per ground column: (range_start int32, dx float32) of SrGrInterpolation (sar/srgr.cu:49-71).

    Float32 Horner with one rounding per fused multiply-add (nvcc contracts ``r *= x; r += e``),
    IEEE division by the float slant spacing, truncation to int.
    """
    p = [np.float32(c) for c in grsr_poly]
    dr = np.float32(range_spacing)
    start = np.empty(ng, dtype=np.int32)
    frac = np.empty(ng, dtype=np.float32)
    for x in range(ng):
        gdist = mulf(np.float32(x), GROUND_SPACING)
        r = np.float32(0.0)
        for e in p:
            r = fmaf(r, gdist, e)
        idx = divf(r, dr)
        s = int(np.trunc(np.float64(idx)))
        start[x] = s
        frac[x] = np.float32(idx) - np.float32(s)
    return start, frac
